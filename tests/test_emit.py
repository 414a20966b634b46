"""The inter-frame bitstream writer (vp8a_write_inter_frame, host code in
the library) against the decoder restatement: a frame written from the
oracle's analysis decisions and quantised coefficients must decode to
exactly those decisions, that reconstruction and that loop-filtered
picture (the encoder/decoder lockstep of
tests/encoder_pframe_auto_loop_filter.rs in oxideav-vp8). The decoder is
primed with the analysis's references and a key frame's default entropy
state. No GPU is involved: the writer runs on the host."""
import numpy as np
import pytest

import vp8a
from vp8a import abi, synth

IDS = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]


def analysed(w, h, seed, qi=40, n_refs=3, segments=None):
    frames, _ = synth.make_sequence(w, h, 5, seed=seed, pieces=3, occluders=2)
    refs = [vp8a.pad_to_mb(*frames[k]) for k in (2, 0, 4)][:n_refs]
    src = frames[3]
    return frames, refs, src


def encode_and_decode(oracle, w, h, seed, qi=40, n_refs=3, n_partitions=1, level=20, sharpness=2, simple=False,
                      segment_quant=None, segment_lf=None, token_updates=None, fit_skip=False, lf_deltas=None,
                      trellis_strength=0.0):
    frames, refs, src = analysed(w, h, seed, n_refs=n_refs)
    ids = IDS[:n_refs]
    dec = np.asarray(oracle.analyse_inter_frame(src, refs, ids, vp8a.rd_lambda(qi))).reshape(-1)
    quant = abi.quant_indices(qi)
    recon = tuple(np.zeros_like(p) for p in refs[0])
    n = dec.size
    seg = None
    if segment_quant is not None:
        seg = np.random.default_rng(seed).integers(0, 4, n).astype(np.int8)
    lf_info = np.zeros(n, abi.MB_LF_INFO_DTYPE)
    cf, fl, _ = oracle.reconstruct_inter_frame(src, refs, ids, dec, quant, recon, mb_segment=seg,
                                               segment_quant=segment_quant, lf_info=lf_info,
                                               trellis_strength=trellis_strength)
    kw = {}
    if segment_quant is not None:
        kw.update(segmentation=1, segment_quant=list(segment_quant))
        if segment_lf is not None:
            kw.update(segment_lf_present=1, segment_lf=list(segment_lf))
    if lf_deltas is not None:
        kw.update(lf_delta_enabled=1, lf_delta_update=1, lf_ref_delta_present=0xF, lf_mode_delta_present=0xF,
                  lf_ref_delta=lf_deltas[0], lf_mode_delta=lf_deltas[1])
    hdr = abi.frame_header(w, h, quant, n_partitions=n_partitions, filter_type=int(simple), loop_filter_level=level,
                           sharpness_level=sharpness, fit_skip_prob=int(fit_skip), **kw)
    bits = vp8a.write_inter_frame(hdr, dec, cf, mb_segment=seg, token_prob_updates=token_updates)
    d = oracle.CapturingDecoder(w, h)
    slots = [refs[ids.index(i)] if i in ids else refs[0] for i in IDS]
    d.prime(slots)
    got = d.decode(bits)
    return dict(dec=dec, cf=cf, fl=fl, recon=recon, lf_info=lf_info, got=got, bits=bits, seg=seg)


def check_lockstep(r, oracle):
    dec, got = r["dec"], r["got"]
    assert not got["key"]
    gd = got["dec"]
    assert np.array_equal(gd["ref_frame"], dec["ref_frame"])
    assert np.array_equal(gd["mode"], dec["mode"])
    assert np.array_equal(gd["mv"].view(np.int32), dec["mv"].view(np.int32))
    split = dec["mode"] == abi.MODE_SPLIT
    assert np.array_equal(gd["split_mvs"][split].view(np.int32), dec["split_mvs"][split].view(np.int32))
    for a, b in zip(got["pre"], r["recon"]):
        assert np.array_equal(a, b)
    assert np.array_equal(got["lf"]["has_coeffs"], r["lf_info"]["has_coeffs"])
    if got["filtered"]:
        post = oracle.filter_frame(r["recon"], r["lf_info"], got["cfg"])
        for a, b in zip(got["post"], post):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("w,h,seed", [(176, 144, 1), (72, 40, 2), (17, 33, 3), (160, 16, 4)])
def test_round_trip_matches_the_analysis(oracle, w, h, seed):
    r = encode_and_decode(oracle, w, h, seed)
    check_lockstep(r, oracle)
    # The analysis produced splits and every mode here (not a trivial frame).
    if (w, h) == (176, 144):
        assert (r["dec"]["mode"] == abi.MODE_SPLIT).any() and (r["dec"]["mode"] == abi.MODE_NEW).any()


@pytest.mark.parametrize("n_partitions", [2, 4, 8])
def test_token_partitions(oracle, n_partitions):
    one = encode_and_decode(oracle, 176, 144, 5)
    r = encode_and_decode(oracle, 176, 144, 5, n_partitions=n_partitions)
    check_lockstep(r, oracle)
    # The same tokens, split by rows: the size grows by the partitions'
    # flush bytes and the size table only.
    assert abs(len(r["bits"]) - len(one["bits"])) <= 8 * n_partitions


def test_segmentation_deltas_and_simple_filter(oracle):
    r = encode_and_decode(oracle, 96, 80, 6, segment_quant=[-10, 5, 30, 0], segment_lf=[0, 3, -8, 12])
    check_lockstep(r, oracle)
    r = encode_and_decode(oracle, 96, 80, 7, simple=True, sharpness=5, lf_deltas=([2, -3, 4, -5], [1, -2, 3, -4]))
    check_lockstep(r, oracle)


def test_token_probability_updates_and_fitted_skip(oracle):
    upd = np.zeros(1056, np.uint8)
    rng = np.random.default_rng(8)
    idx = rng.choice(1056, 40, replace=False)
    upd[idx] = rng.integers(1, 256, 40)
    r = encode_and_decode(oracle, 128, 96, 8, token_updates=upd, fit_skip=True, qi=90)
    check_lockstep(r, oracle)


def test_low_and_high_quantisers(oracle):
    # qi 4: large coefficients (DCT_cat6 tokens); qi 127: mostly skipped MBs.
    for qi in (4, 127):
        r = encode_and_decode(oracle, 64, 48, 9, qi=qi, n_refs=2)
        check_lockstep(r, oracle)
    assert np.abs(encode_and_decode(oracle, 64, 48, 9, qi=4)["cf"]).max() > 66


def test_header_errors():
    dec = np.zeros(4, abi.MB_DECISION_DTYPE)
    dec["ref_frame"] = abi.REF_LAST
    cf = np.zeros((4, 400), np.int16)
    q = abi.quant_indices(40)
    cases = [
        (abi.frame_header(0, 32, q), abi.E_INVALID_DIMENSIONS),
        (abi.frame_header(32, 32, abi.quant_indices(128)), abi.E_QUANT_INDEX_OUT_OF_RANGE),
        (abi.frame_header(32, 32, q, loop_filter_level=64), abi.E_LOOP_FILTER_LEVEL_OUT_OF_RANGE),
        (abi.frame_header(32, 32, q, sharpness_level=8), abi.E_SHARPNESS_LEVEL_OUT_OF_RANGE),
        (abi.frame_header(32, 32, q, n_partitions=3), abi.E_INVALID_DCT_PARTITION_COUNT),
        (abi.frame_header(32, 32, q, copy_buffer_to_golden=3), abi.E_INVALID_COPY_BUFFER_SELECTOR),
        (abi.frame_header(32, 32, q, refresh_golden_frame=1, copy_buffer_to_golden=1),
         abi.E_INVALID_COPY_BUFFER_SELECTOR),
        (abi.frame_header(32, 32, q, lf_delta_enabled=1, lf_ref_delta=[64, 0, 0, 0]),
         abi.E_LOOP_FILTER_DELTA_OUT_OF_RANGE),
    ]
    for hdr, want in cases:
        with pytest.raises(vp8a.Vp8aError) as e:
            vp8a.write_inter_frame(hdr, dec, cf)
        assert e.value.status == want
    bad = cf.copy()
    bad[1, 20] = 2115
    with pytest.raises(vp8a.Vp8aError) as e:
        vp8a.write_inter_frame(abi.frame_header(32, 32, q), dec, bad)
    assert e.value.status == abi.E_COEFFICIENT_OUT_OF_RANGE
    intra = dec.copy()
    intra["ref_frame"][2] = abi.REF_INTRA
    with pytest.raises(vp8a.Vp8aError) as e:
        vp8a.write_inter_frame(abi.frame_header(32, 32, q), intra, cf)
    assert e.value.status == abi.E_INVALID_ARGUMENT
    # An all-ZEROMV, all-skip frame is a few bytes.
    assert len(vp8a.write_inter_frame(abi.frame_header(32, 32, q), dec, cf)) < 80


@pytest.mark.parametrize("strength,segments", [(1.0, False), (3.0, True), (8.0, False)])
def test_trellis_frames_decode_in_lockstep(oracle, strength, segments):
    # The §13 trellis chooses other levels than plain rounding; the frame
    # written from them must still decode to the same reconstruction, and it
    # costs fewer bytes.
    kw = dict(segment_quant=[-6, 0, 9, 20]) if segments else {}
    r = encode_and_decode(oracle, 176, 144, 11, qi=44, trellis_strength=strength, **kw)
    check_lockstep(r, oracle)
    plain = encode_and_decode(oracle, 176, 144, 11, qi=44, **kw)
    assert not np.array_equal(r["cf"], plain["cf"])
    assert len(r["bits"]) < len(plain["bits"])
