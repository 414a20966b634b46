"""Parity: the device §18 inter prediction (vp8a_predict_inter_mb,
vp8a_predict_split_mv, vp8a_predict_inter_frame) reproduces the oracle's
predict_inter_mb / predict_split_mv (src/motion_comp.rs:1986, :2228)
byte for byte: both filter sets, full-pixel on and off, vectors reaching
past every plane edge, i16 wrap of the doubled vectors, host and device
buffers, unaligned outputs, and whole frames of real analysis decisions."""
import ctypes as C

import numpy as np
import pytest

import vp8a
from vp8a import abi, synth
from vp8a.frames import planes, ptr

pytestmark = pytest.mark.gpu


def random_ref(rng, mb_cols, mb_rows):
    y = rng.integers(0, 256, (mb_rows * 16, mb_cols * 16), dtype=np.uint8)
    u = rng.integers(0, 256, (mb_rows * 8, mb_cols * 8), dtype=np.uint8)
    v = rng.integers(0, 256, (mb_rows * 8, mb_cols * 8), dtype=np.uint8)
    return y, u, v


def random_mvs(rng, n, extreme=False):
    mvs = rng.integers(-1023, 1024, (n, 2))
    small = rng.random(n) < 0.5  # many vectors near the MB, most fetches in-plane
    mvs[small] = rng.integers(-24, 25, (int(small.sum()), 2))
    if extreme:  # i16 extremes: the doubling wraps, offsets leave the plane
        k = max(1, n // 8)
        mvs[:k] = rng.choice([-32768, -32767, -16385, 16384, 32767], (k, 2))
    return mvs


def positions(rng, n, mb_cols, mb_rows):
    xy = np.stack([rng.integers(0, mb_cols, n), rng.integers(0, mb_rows, n)], axis=1)
    xy[: max(1, n // 10)] = [mb_cols + 3, mb_rows + 1]  # MBs past the grid clamp like any fetch
    return xy


@pytest.mark.parametrize("filter_set", [abi.FILTER_SIXTAP, abi.FILTER_BILINEAR])
@pytest.mark.parametrize("full_pixel", [False, True])
def test_predict_inter_mb_batch(ctx, oracle, filter_set, full_pixel):
    rng = np.random.default_rng(11 + 2 * filter_set + full_pixel)
    ref = random_ref(rng, 7, 5)
    n = 777
    xy = positions(rng, n, 7, 5)
    mvs = random_mvs(rng, n, extreme=True)
    got = vp8a.predict_inter_mb(ctx, ref, xy, mvs, full_pixel, filter_set)
    want = oracle.predict_inter_mb(ref, xy, mvs, full_pixel, filter_set)
    bad = np.argwhere((got != want).any(axis=1)).reshape(-1)
    assert bad.size == 0, f"{bad.size} MBs differ, first {bad[:5]} mvs {mvs[bad[:3]]}"


@pytest.mark.parametrize("filter_set", [abi.FILTER_SIXTAP, abi.FILTER_BILINEAR])
@pytest.mark.parametrize("full_pixel", [False, True])
def test_predict_split_mv_batch(ctx, oracle, filter_set, full_pixel):
    rng = np.random.default_rng(23 + 2 * filter_set + full_pixel)
    ref = random_ref(rng, 6, 4)
    n = 333
    xy = positions(rng, n, 6, 4)
    mvs = random_mvs(rng, 16 * n, extreme=True)
    got = vp8a.predict_split_mv(ctx, ref, xy, mvs, full_pixel, filter_set)
    want = oracle.predict_split_mv(ref, xy, mvs, full_pixel, filter_set)
    bad = np.argwhere((got != want).any(axis=1)).reshape(-1)
    assert bad.size == 0, f"{bad.size} MBs differ, first {bad[:5]}"


def test_predict_single_mb_grid_and_empty_batch(ctx, oracle):
    rng = np.random.default_rng(5)
    ref = random_ref(rng, 1, 1)
    xy = np.zeros((64, 2), np.uint32)
    mvs = random_mvs(rng, 64)
    assert np.array_equal(vp8a.predict_inter_mb(ctx, ref, xy, mvs), oracle.predict_inter_mb(ref, xy, mvs))
    assert vp8a.predict_inter_mb(ctx, ref, xy[:0], mvs[:0]).shape == (0, 384)


def test_predict_device_buffers_and_unaligned_output(ctx, oracle):
    import torch

    rng = np.random.default_rng(9)
    ref = random_ref(rng, 5, 3)
    n = 100
    xy = positions(rng, n, 5, 3)
    mvs = random_mvs(rng, 16 * n)
    want = oracle.predict_split_mv(ref, xy, mvs)
    dref = [torch.from_numpy(p).cuda() for p in ref]
    dxy = torch.from_numpy(np.ascontiguousarray(xy, np.uint32).view(np.int32)).cuda()
    dmv = torch.from_numpy(np.ascontiguousarray(mvs, np.int16)).cuda()
    raw = torch.zeros(n * 384 + 1, dtype=torch.uint8, device="cuda")
    out = raw[1:]  # odd address: the byte-store path
    p = planes(*dref)
    st = ctx._lib.vp8a_predict_split_mv(ctx.handle, C.byref(p), ptr(dxy), ptr(dmv), n, 0, abi.FILTER_SIXTAP, ptr(out))
    assert st == abi.OK
    ctx.synchronize()
    assert np.array_equal(out.cpu().numpy().reshape(n, 384), want)


def frame_case(w, h, seed):
    frames, _ = synth.make_sequence(w, h, 7, seed=seed, pieces=5, occluders=4)
    k = 3
    refs = [vp8a.pad_to_mb(*frames[k - 1]), vp8a.pad_to_mb(*frames[0]), vp8a.pad_to_mb(*frames[k + 1])]
    return frames[k], refs


@pytest.mark.parametrize("w,h,seed", [(320, 240, 31), (1920, 1080, 7)])
def test_predict_inter_frame_from_analysis(ctx, oracle, w, h, seed):
    # The real decisions of the device analysis predicted from their own
    # references (the 320x240 sequence is the one whose decisions exercise
    # NEW, NEAREST/NEAR and SPLITMV in the analysis tests).
    frame, refs = frame_case(w, h, seed)
    ids = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]
    dec = vp8a.analyse_inter_frame(ctx, frame, refs, ids, vp8a.rd_lambda(44))
    if w == 320:
        assert (dec["mode"] == abi.MODE_SPLIT).any() and (dec["mode"] == abi.MODE_NEW).any()
    got = tuple(np.full(p.shape, 3, np.uint8) for p in refs[0])
    want = tuple(np.full(p.shape, 3, np.uint8) for p in refs[0])
    vp8a.predict_inter_frame(ctx, refs, ids, dec, got)
    assert oracle.predict_inter_frame(refs, ids, dec, want) == 0
    for g, wnt in zip(got, want):
        assert np.array_equal(g, wnt)


@pytest.mark.parametrize("filter_set", [abi.FILTER_SIXTAP, abi.FILTER_BILINEAR])
def test_predict_inter_frame_mixed_decisions_device_strided(ctx, oracle, filter_set):
    # Synthetic decisions: intra MBs, a reference id with no planes, SPLIT and
    # whole-MB vectors; a reference and the output planes with a row pitch
    # that is not a multiple of 4 (byte loads and stores), all buffers on
    # the device.
    import torch

    rng = np.random.default_rng(31 + filter_set)
    mb_cols, mb_rows = 9, 6
    refs = [random_ref(rng, mb_cols, mb_rows) for _ in range(2)]
    ids = [abi.REF_GOLDEN, abi.REF_LAST]
    n = mb_cols * mb_rows
    dec = np.zeros(n, abi.MB_DECISION_DTYPE)
    dec["ref_frame"] = rng.choice([abi.REF_INTRA, abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF], n)
    dec["mode"] = rng.choice([abi.MODE_ZERO, abi.MODE_NEW, abi.MODE_SPLIT], n)
    m = random_mvs(rng, n)
    dec["mv"]["row"], dec["mv"]["col"] = m[:, 0], m[:, 1]
    sm = random_mvs(rng, 16 * n).reshape(n, 16, 2)
    dec["split_mvs"]["row"], dec["split_mvs"]["col"] = sm[..., 0], sm[..., 1]

    def padded(p, extra):
        a = np.full((p.shape[0], p.shape[1] + extra), 200, np.uint8)
        return a

    want = [padded(p, 3)[:, : p.shape[1]] for p in refs[0]]
    skipped = oracle.predict_inter_frame(refs, ids, dec, want, filter_set=filter_set)
    assert skipped == int(np.isin(dec["ref_frame"], [abi.REF_INTRA, abi.REF_ALTREF]).sum())
    def strided(p):  # row pitch width + 3: word loads of the source are off
        d = torch.zeros((p.shape[0], p.shape[1] + 3), dtype=torch.uint8, device="cuda")
        d[:, : p.shape[1]] = torch.from_numpy(p).cuda()
        return d[:, : p.shape[1]]

    dref = [[torch.from_numpy(p).cuda() for p in refs[0]], [strided(p) for p in refs[1]]]
    dout = [torch.full((p.shape[0], p.shape[1] + 3), 200, dtype=torch.uint8, device="cuda")[:, : p.shape[1]]
            for p in refs[0]]
    ddec = torch.from_numpy(dec.view(np.uint8).copy()).cuda()
    vp8a.predict_inter_frame(ctx, dref, ids, ddec, dout, filter_set=filter_set)
    ctx.synchronize()
    for g, wnt in zip(dout, want):
        assert np.array_equal(g.cpu().numpy(), wnt)


def test_predict_errors(ctx):
    rng = np.random.default_rng(1)
    ref = random_ref(rng, 2, 2)
    with pytest.raises(vp8a.Vp8aError) as e:
        vp8a.predict_inter_mb(ctx, ref, [(0, 0)], [(1, 1)], filter_set=2)
    assert e.value.status == abi.E_INVALID_ARGUMENT
    other = random_ref(rng, 3, 2)
    dec = np.zeros(4, abi.MB_DECISION_DTYPE)
    out = tuple(np.zeros_like(p) for p in ref)
    with pytest.raises(vp8a.Vp8aError) as e:
        vp8a.predict_inter_frame(ctx, [other], [abi.REF_LAST], dec, out)
    assert e.value.status == abi.E_REFERENCE_DIMENSIONS_MISMATCH
    with pytest.raises(vp8a.Vp8aError) as e:
        vp8a.predict_inter_frame(ctx, [ref], [abi.REF_INTRA], dec, out)
    assert e.value.status == abi.E_INVALID_ARGUMENT
