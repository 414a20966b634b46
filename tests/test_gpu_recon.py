"""Parity: the device §14 inter reconstruction (vp8a_reconstruct_inter_frame,
trellis off) reproduces the oracle's chosen-mode step of pick_mb_for_ref
(src/encoder.rs:8704-8800) byte for byte — reconstruction planes, the
quantised MbCoeffs and the skip / has-coeffs flags — on real analysis
decisions, odd picture sizes (edge-replicated source MBs), segment
quantisers, quantiser deltas, both filter sets, intra MBs, device buffers
and unaligned plane pitches."""
import numpy as np
import pytest

import vp8a
from vp8a import abi, synth

pytestmark = pytest.mark.gpu


def frame_case(w, h, seed):
    frames, _ = synth.make_sequence(w, h, 7, seed=seed, pieces=5, occluders=4)
    k = 3
    refs = [vp8a.pad_to_mb(*frames[k - 1]), vp8a.pad_to_mb(*frames[0]), vp8a.pad_to_mb(*frames[k + 1])]
    return frames[k], refs


def run_both(ctx, oracle, frame, refs, ids, dec, quant, fill=7, **kw):
    got = tuple(np.full(p.shape, fill, np.uint8) for p in refs[0])
    want = tuple(np.full(p.shape, fill, np.uint8) for p in refs[0])
    n = got[0].shape[0] // 16 * (got[0].shape[1] // 16)
    glf = np.full(n, 0x55, np.uint8).repeat(abi.MB_LF_INFO_DTYPE.itemsize).view(abi.MB_LF_INFO_DTYPE)
    wlf = glf.copy()
    gcf, gfl = vp8a.reconstruct_inter_frame(ctx, frame, refs, ids, dec, quant, got, lf_info=glf, **kw)
    wcf, wfl, _ = oracle.reconstruct_inter_frame(frame, refs, ids, dec, quant, want, lf_info=wlf, **kw)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    assert np.array_equal(gfl, wfl)
    assert np.array_equal(glf.view(np.uint8), wlf.view(np.uint8))
    bad = np.argwhere((gcf != wcf).any(axis=1)).reshape(-1)
    assert bad.size == 0, f"coefficients differ in {bad.size} MBs, first {bad[:5]}"
    return got, gcf, gfl


@pytest.mark.parametrize("w,h,seed,qi", [(320, 240, 31, 44), (1920, 1080, 7, 44), (320, 240, 31, 4),
                                         (320, 240, 31, 120)])
def test_reconstruct_from_analysis(ctx, oracle, w, h, seed, qi):
    frame, refs = frame_case(w, h, seed)
    ids = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]
    dec = vp8a.analyse_inter_frame(ctx, frame, refs, ids, vp8a.rd_lambda(qi))
    _, cf, fl = run_both(ctx, oracle, frame, refs, ids, dec, abi.quant_indices(qi))
    # The case must exercise both skipped and coded MBs.
    assert (fl & abi.MB_SKIP).any() or qi < 20
    assert (fl & abi.MB_HAS_COEFFS).any()


@pytest.mark.parametrize("w,h", [(72, 40), (17, 33), (160, 16), (16, 160)])
def test_reconstruct_odd_sizes(ctx, oracle, w, h):
    frames, _ = synth.make_sequence(w, h, 4, seed=w * 3 + h, pieces=3, occluders=2)
    refs = [vp8a.pad_to_mb(*frames[1]), vp8a.pad_to_mb(*frames[0]), vp8a.pad_to_mb(*frames[3])]
    ids = [1, 2, 3]
    dec = vp8a.analyse_inter_frame(ctx, frames[2], refs, ids, vp8a.rd_lambda(30))
    run_both(ctx, oracle, frames[2], refs, ids, dec, abi.quant_indices(30, y_dc=-3, y2_dc=5, y2_ac=-7, uv_dc=9,
                                                                        uv_ac=-2))


def random_case(rng, mb_cols, mb_rows):
    w, h = mb_cols * 16 - 5, mb_rows * 16 - 3
    frame = (rng.integers(0, 256, (h, w), dtype=np.uint8),
             rng.integers(0, 256, ((h + 1) // 2, (w + 1) // 2), dtype=np.uint8),
             rng.integers(0, 256, ((h + 1) // 2, (w + 1) // 2), dtype=np.uint8))
    # References near the source so the residuals are realistic, plus noise.
    pad = vp8a.pad_to_mb(*frame)
    refs = [tuple(np.clip(p.astype(int) + rng.integers(-12, 13, p.shape), 0, 255).astype(np.uint8) for p in pad)
            for _ in range(2)]
    n = mb_cols * mb_rows
    dec = np.zeros(n, abi.MB_DECISION_DTYPE)
    dec["ref_frame"] = rng.choice([abi.REF_INTRA, abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF], n)
    dec["mode"] = rng.choice([abi.MODE_ZERO, abi.MODE_NEW, abi.MODE_SPLIT], n)
    m = rng.integers(-20, 21, (n, 2))
    dec["mv"]["row"], dec["mv"]["col"] = m[:, 0], m[:, 1]
    sm = rng.integers(-20, 21, (n, 16, 2))
    dec["split_mvs"]["row"], dec["split_mvs"]["col"] = sm[..., 0], sm[..., 1]
    return frame, refs, dec


@pytest.mark.parametrize("filter_set,full_pixel,segment_abs", [(abi.FILTER_SIXTAP, False, False),
                                                               (abi.FILTER_BILINEAR, True, True)])
def test_reconstruct_mixed_decisions_and_segments(ctx, oracle, filter_set, full_pixel, segment_abs):
    rng = np.random.default_rng(41 + filter_set)
    frame, refs, dec = random_case(rng, 11, 7)
    ids = [abi.REF_GOLDEN, abi.REF_LAST]
    seg = rng.integers(-1, 4, dec.size).astype(np.int8)
    sq = [90, 10, 127, 0] if segment_abs else [-20, 15, 100, -100]
    _, cf, fl = run_both(ctx, oracle, frame, refs, ids, dec, abi.quant_indices(44, uv_ac=3), mb_segment=seg,
                         segment_quant=sq, segment_abs=segment_abs, full_pixel=full_pixel, filter_set=filter_set)
    skipped = np.isin(dec["ref_frame"], [abi.REF_INTRA, abi.REF_ALTREF])
    assert (fl[skipped] == 0).all() and not cf[skipped].any()
    assert (fl[~skipped] & abi.MB_HAS_COEFFS).any()


def test_reconstruct_device_buffers_unaligned_pitch(ctx, oracle):
    import torch

    rng = np.random.default_rng(5)
    frame, refs, dec = random_case(rng, 9, 5)
    ids = [abi.REF_LAST, abi.REF_GOLDEN]
    quant = abi.quant_indices(60)
    want = tuple(np.full(p.shape, 9, np.uint8) for p in refs[0])
    wcf, wfl, _ = oracle.reconstruct_inter_frame(frame, refs, ids, dec, quant, want)

    def strided(p, fill=None):
        d = torch.full((p.shape[0], p.shape[1] + 3), 9, dtype=torch.uint8, device="cuda")
        if fill is None:
            d[:, : p.shape[1]] = torch.from_numpy(np.ascontiguousarray(p)).cuda()
        return d[:, : p.shape[1]]

    dframe = [strided(p) for p in frame]
    drefs = [[strided(p) for p in r] for r in refs]
    drec = [strided(p, fill=9) for p in refs[0]]
    ddec = torch.from_numpy(dec.view(np.uint8).copy()).cuda()
    dcf = torch.zeros((dec.size, 400), dtype=torch.int16, device="cuda")
    dfl = torch.zeros(dec.size, dtype=torch.uint8, device="cuda")
    vp8a.reconstruct_inter_frame(ctx, dframe, drefs, ids, ddec, quant, drec, coeffs=dcf, flags=dfl)
    ctx.synchronize()
    for g, w in zip(drec, want):
        assert np.array_equal(g.cpu().numpy(), w)
    assert np.array_equal(dcf.cpu().numpy(), wcf)
    assert np.array_equal(dfl.cpu().numpy(), wfl)


def test_reconstruct_errors(ctx):
    rng = np.random.default_rng(1)
    frame, refs, dec = random_case(rng, 3, 2)
    rec = tuple(np.zeros_like(p) for p in refs[0])
    with pytest.raises(vp8a.Vp8aError) as e:
        vp8a.reconstruct_inter_frame(ctx, frame, refs, [1, 2], dec, abi.quant_indices(128), rec)
    assert e.value.status == abi.E_QUANT_INDEX_OUT_OF_RANGE
    small = tuple(p[:16, :16] for p in frame[:1]) + tuple(p[:8, :8] for p in frame[1:])
    with pytest.raises(vp8a.Vp8aError) as e:
        vp8a.reconstruct_inter_frame(ctx, small, refs, [1, 2], dec, abi.quant_indices(40), rec)
    assert e.value.status == abi.E_REFERENCE_DIMENSIONS_MISMATCH



@pytest.mark.parametrize("strength,qi,segments", [(1.0, 44, False), (1.0, 10, False), (3.5, 80, True),
                                                  (8.0, 44, False), (0.5, 127, True)])
def test_reconstruct_with_the_trellis(oracle, strength, qi, segments):
    # The §13 trellis (TrellisStrength > 0) on every block: the device's
    # levels, reconstruction and flags equal the oracle's, whole-MB and
    # SPLITMV MBs alike, with segment quantisers (each its own lambda).
    frame, refs = frame_case(320, 240, 31)
    ids = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]
    kw = {}
    if segments:
        kw = dict(mb_segment=np.random.default_rng(qi).integers(-1, 4, 300).astype(np.int8),
                  segment_quant=[-10, 0, 7, 25])
    with vp8a.Context(0) as c:
        dec = vp8a.analyse_inter_frame(c, frame, refs, ids, vp8a.rd_lambda(qi))
        assert (dec["mode"] == abi.MODE_SPLIT).any()
        plain_cf, _ = vp8a.reconstruct_inter_frame(c, frame, refs, ids, dec, abi.quant_indices(qi),
                                                   tuple(np.zeros_like(p) for p in refs[0]), **kw)
        c.set_trellis_strength(strength)
        got = tuple(np.full(p.shape, 7, np.uint8) for p in refs[0])
        want = tuple(np.full(p.shape, 7, np.uint8) for p in refs[0])
        gcf, gfl = vp8a.reconstruct_inter_frame(c, frame, refs, ids, dec, abi.quant_indices(qi), got, **kw)
    wcf, wfl, _ = oracle.reconstruct_inter_frame(frame, refs, ids, dec, abi.quant_indices(qi), want,
                                                 trellis_strength=strength, threads=8, **kw)
    bad = np.argwhere((gcf != wcf).any(axis=1)).reshape(-1)
    assert bad.size == 0, f"coefficients differ in {bad.size} MBs, first {bad[:5]}"
    assert np.array_equal(gfl, wfl)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    assert not np.array_equal(gcf, plain_cf)
    assert np.count_nonzero(gcf) < np.count_nonzero(plain_cf)
