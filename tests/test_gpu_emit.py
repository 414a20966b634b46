"""The whole P-frame encode on the device (vp8a.encode_p_frame: analysis,
§14 reconstruction, §9.4 loop-filter search, §15 filter pass) followed by
the bitstream writer, decoded by the decoder restatement: the decoder must
rebuild the device's decisions, its reconstruction and its filtered
picture exactly (the lockstep of tests/encoder_pframe_auto_loop_filter.rs
in oxideav-vp8), and the bytes must equal those written from the oracle's
own analysis and reconstruction of the same frame."""
import numpy as np
import pytest

import vp8a
from vp8a import abi, synth

pytestmark = pytest.mark.gpu

IDS = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]


def sequence(w, h, seed, n_refs):
    frames, _ = synth.make_sequence(w, h, 5, seed=seed, pieces=3, occluders=2)
    refs = [vp8a.pad_to_mb(*frames[k]) for k in (2, 0, 4)][:n_refs]
    return frames[3], refs


def decode(oracle, w, h, refs, ids, bits):
    d = oracle.CapturingDecoder(w, h)
    d.prime([refs[ids.index(i)] if i in ids else refs[0] for i in IDS])
    return d.decode(bits)


@pytest.mark.parametrize("w,h,seed,n_refs,qi,parts", [(176, 144, 1, 3, 40, 1), (320, 240, 2, 3, 20, 4),
                                                      (72, 40, 3, 2, 60, 2), (17, 33, 4, 1, 100, 1)])
def test_encode_p_frame_lockstep(ctx, oracle, w, h, seed, n_refs, qi, parts):
    src, refs = sequence(w, h, seed, n_refs)
    ids = IDS[:n_refs]
    bits, filtered, info = vp8a.encode_p_frame(ctx, src, refs, ids, qi, n_partitions=parts)
    got = decode(oracle, w, h, refs, ids, bits)
    dec = info["decisions"]
    assert np.array_equal(got["dec"]["ref_frame"], dec["ref_frame"])
    assert np.array_equal(got["dec"]["mode"], dec["mode"])
    assert np.array_equal(got["dec"]["mv"].view(np.int32), dec["mv"].view(np.int32))
    for a, b in zip(got["pre"], info["recon"]):
        assert np.array_equal(a, b)
    for a, b in zip(got["post"], filtered):
        assert np.array_equal(a, b)
    assert got["cfg"].loop_filter_level == info["level"] and got["cfg"].sharpness_level == info["sharpness"]

    # The same frame from the oracle's analysis and reconstruction.
    odec = np.asarray(oracle.analyse_inter_frame(src, refs, ids, vp8a.rd_lambda(qi))).reshape(-1)
    orec = tuple(np.zeros_like(p) for p in refs[0])
    ocf, _, _ = oracle.reconstruct_inter_frame(src, refs, ids, odec, abi.quant_indices(qi), orec)
    hdr = abi.frame_header(w, h, abi.quant_indices(qi), n_partitions=parts, loop_filter_level=info["level"],
                           sharpness_level=info["sharpness"])
    assert vp8a.write_inter_frame(hdr, odec, ocf) == bits


def test_encode_p_frame_fixed_level_and_simple_filter(ctx, oracle):
    src, refs = sequence(96, 64, 7, 2)
    ids = IDS[:2]
    bits, filtered, info = vp8a.encode_p_frame(ctx, src, refs, ids, 30, loop_filter_level=24, sharpness_level=3,
                                               simple=True, auto_lf=False)
    assert info["level"] == 24
    got = decode(oracle, 96, 64, refs, ids, bits)
    assert got["cfg"].simple == 1
    for a, b in zip(got["post"], filtered):
        assert np.array_equal(a, b)


def test_device_trellis_frame_decodes_in_lockstep(oracle):
    # A P frame reconstructed with the device trellis (TrellisStrength 1.0,
    # the reference's default) is written and decoded by the decoder
    # restatement primed with the references: same decisions and
    # reconstruction, and fewer bytes than with plain rounding.
    from vp8a import abi, synth

    frames, _ = synth.make_sequence(176, 144, 5, seed=23, pieces=3, occluders=2)
    refs = [vp8a.pad_to_mb(*frames[k]) for k in (2, 0, 4)]
    ids = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]
    sizes = {}
    with vp8a.Context(0) as c:
        for strength in (0.0, 1.0):
            c.set_trellis_strength(strength)
            bits, filt, det = vp8a.encode_p_frame(c, frames[3], refs, ids, 44)
            d = oracle.CapturingDecoder(176, 144)
            d.prime(refs)
            back = d.decode(bits)
            assert np.array_equal(back["dec"]["mode"], det["decisions"]["mode"])
            assert all(np.array_equal(a, b) for a, b in zip(back["pre"], det["recon"]))
            sizes[strength] = len(bits)
    assert sizes[1.0] < sizes[0.0]
