"""Parity: the batched §17/§18 motion-search kernels (through the C ABI)
reproduce the oracle bit-exactly — MVs and SADs — over every MB of the
320x240 sequence, edge and clamp cases, and odd plane sizes."""
import numpy as np
import pytest
from util import extract_mbs, sr_tuples

import vp8a
from vp8a import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def seq():
    frames, _ = synth.make_sequence(320, 240, 3, seed=11)
    ref = vp8a.pad_to_mb(*frames[0])[0]
    mbs, xy = extract_mbs(frames[1][0], 15, 20)
    return ref, mbs, xy


def centers_for(n, rng, kind):
    if kind == "zero":
        return np.zeros((n, 2), np.int16)
    if kind == "small":
        return rng.integers(-64, 65, (n, 2)).astype(np.int16)
    if kind == "wide":
        return rng.integers(-1023, 1024, (n, 2)).astype(np.int16)
    if kind == "extreme":
        return rng.choice(np.array([-32768, -1024, -1023, -1020, 1020, 1023, 1024, 32767], np.int16), (n, 2))
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["zero", "small", "wide", "extreme"])
@pytest.mark.parametrize("iters", [0, 1, 8, 13])
def test_diamond_parity(ctx, oracle, seq, kind, iters):
    ref, mbs, xy = seq
    c = centers_for(len(mbs), np.random.default_rng(iters * 7 + len(kind)), kind)
    got = vp8a.small_diamond_search_luma(ctx, ref, mbs, xy, c, iters)
    want = oracle.small_diamond_search_luma(ref, mbs, xy, c, iters)
    assert sr_tuples(got) == sr_tuples(want)


@pytest.mark.parametrize("kind", ["zero", "small", "wide"])
def test_half_and_quarter_parity(ctx, oracle, seq, kind):
    ref, mbs, xy = seq
    rng = np.random.default_rng(5)
    whole = (centers_for(len(mbs), rng, kind).astype(np.int32) // 4 * 4).clip(-1020, 1020).astype(np.int16)
    assert sr_tuples(vp8a.half_pixel_refine_luma(ctx, ref, mbs, xy, whole)) == sr_tuples(
        oracle.half_pixel_refine_luma(ref, mbs, xy, whole))
    half = (centers_for(len(mbs), rng, kind).astype(np.int32) // 2 * 2).clip(-1022, 1022).astype(np.int16)
    assert sr_tuples(vp8a.quarter_pixel_refine_luma(ctx, ref, mbs, xy, half)) == sr_tuples(
        oracle.quarter_pixel_refine_luma(ref, mbs, xy, half))


def test_sad_at_mv_parity_all_fractions(ctx, oracle, seq):
    ref, mbs, xy = seq
    rng = np.random.default_rng(9)
    n = len(mbs)
    for trial in range(4):
        mv = rng.integers(-1023, 1024, (n, 2)).astype(np.int16) if trial else rng.integers(-40, 41, (n, 2)).astype(
            np.int16)
        assert np.array_equal(vp8a.mb_luma_sad_at_mv(ctx, ref, mbs, xy, mv),
                              oracle.mb_luma_sad_at_mv(ref, mbs, xy, mv))


def test_descent_parity(ctx, oracle, seq):
    ref, mbs, xy = seq
    c = centers_for(len(mbs), np.random.default_rng(3), "small")
    got = vp8a.motion_descent(ctx, ref, mbs, xy, c, 8)
    want = oracle.motion_descent(ref, mbs, xy, c, 8)
    for g, w in zip(got, want):
        assert sr_tuples(g) == sr_tuples(w)


def test_masked_descent_runs_only_the_active_items(ctx, oracle, seq):
    # vp8a_motion_descent_masked: the active items get the oracle's descent,
    # the others keep what the output buffers held.
    import ctypes as C

    from vp8a import abi
    from vp8a.frames import ptr

    ref, mbs, xy = seq
    rng = np.random.default_rng(8)
    c = centers_for(len(mbs), rng, "small")
    cc = np.ascontiguousarray(np.asarray(c).astype(np.int16).reshape(-1, 2))
    xyc = np.ascontiguousarray(np.asarray(xy, dtype=np.uint32).reshape(-1, 2))
    active = (rng.random(len(mbs)) < 0.3).astype(np.uint8)
    active[0], active[-1] = 1, 0
    want = oracle.motion_descent(ref, mbs, xy, c, 8)
    outs = [np.zeros(len(mbs), abi.SEARCH_RESULT_DTYPE) for _ in range(3)]
    for o in outs:
        o["sad"] = 0xDEADBEEF
    r = vp8a.luma_ref(ref)
    lib = ctx._lib
    assert lib.vp8a_motion_descent_masked(ctx.handle, C.byref(r), ptr(np.ascontiguousarray(mbs)), ptr(xyc), ptr(cc),
                                          8, len(mbs), ptr(active), *[ptr(o) for o in outs]) == abi.OK
    on = active.astype(bool)
    for g, w in zip(outs, want):
        assert sr_tuples(g[on]) == sr_tuples(w[on])
        assert (g["sad"][~on] == 0xDEADBEEF).all()
    assert lib.vp8a_motion_descent_masked(ctx.handle, C.byref(r), ptr(np.ascontiguousarray(mbs)), ptr(xyc), ptr(cc),
                                          8, len(mbs), None, *[ptr(o) for o in outs]) == abi.E_INVALID_ARGUMENT


@pytest.mark.parametrize("w,h", [(16, 16), (33, 17), (48, 80), (200, 24)])
def test_odd_plane_sizes(ctx, oracle, w, h):
    rng = np.random.default_rng(w * h)
    plane = rng.integers(0, 256, (h, w + 7), dtype=np.uint8)  # row stride > width
    mbr, mbc = (h + 15) // 16, (w + 15) // 16
    src = rng.integers(0, 256, (mbr * mbc, 256), dtype=np.uint8)
    xy = np.stack(np.meshgrid(np.arange(mbc), np.arange(mbr)), -1).reshape(-1, 2).astype(np.uint32)
    c = rng.integers(-80, 81, (len(xy), 2)).astype(np.int16)
    got = vp8a.motion_descent(ctx, plane, src, xy, c, 8, width=w, height=h)
    want = oracle.motion_descent(plane, src, xy, c, 8, width=w, height=h)
    for g, ww in zip(got, want):
        assert sr_tuples(g) == sr_tuples(ww)
    mv = rng.integers(-300, 301, (len(xy), 2)).astype(np.int16)
    assert np.array_equal(vp8a.mb_luma_sad_at_mv(ctx, plane, src, xy, mv, width=w, height=h),
                          oracle.mb_luma_sad_at_mv(plane, src, xy, mv, width=w, height=h))


def test_reference_kats_on_gpu(ctx):
    # The reference's exact-translation KATs (src/motion_search.rs:995,
    # :1243, :1446) through the CUDA path.
    from util import feature_plane, mb_block, stepped_plane, two_d_ramp_plane

    ref = feature_plane(64, 32, 128, 240, 6, 4, 4)
    src = mb_block(feature_plane(64, 32, 128, 240, 4, 4, 4), 0, 0)
    r = vp8a.small_diamond_search_luma(ctx, ref, src, [[0, 0]], [[0, 0]], 32)[0]
    assert (int(r["mv"]["row"]), int(r["mv"]["col"]), int(r["sad"])) == (0, 8, 0)
    ref = two_d_ramp_plane(64, 64)
    src = mb_block(synth.translate(ref, 0, 4), 1, 1)
    r = vp8a.half_pixel_refine_luma(ctx, ref, src, [[1, 1]], [[0, 0]])[0]
    assert (int(r["mv"]["row"]), int(r["mv"]["col"]), int(r["sad"])) == (0, 2, 0)
    ref = stepped_plane(64, 64)
    src = mb_block(synth.translate(ref, 0, 2), 1, 1)
    h = vp8a.half_pixel_refine_luma(ctx, ref, src, [[1, 1]], [[0, 0]])[0]["mv"]
    r = vp8a.quarter_pixel_refine_luma(ctx, ref, src, [[1, 1]], [[int(h["row"]), int(h["col"])]])[0]
    assert (int(r["mv"]["row"]), int(r["mv"]["col"]), int(r["sad"])) == (0, 1, 0)


def test_device_resident_inputs(ctx, oracle, seq):
    # The same entry point with torch CUDA buffers (no host staging).
    torch = pytest.importorskip("torch")
    ref, mbs, xy = seq
    c = centers_for(len(mbs), np.random.default_rng(1), "small")
    want = oracle.small_diamond_search_luma(ref, mbs, xy, c, 8)
    d_ref = torch.from_numpy(ref).cuda()
    d_src = torch.from_numpy(mbs).cuda()
    d_xy = torch.from_numpy(xy.astype(np.int32)).cuda()
    d_c = torch.from_numpy(c).cuda()
    d_out = torch.zeros(len(mbs) * 8, dtype=torch.uint8, device="cuda")
    r = vp8a.luma_ref(d_ref)
    import ctypes as C

    lib = vp8a.load()
    st = lib.vp8a_small_diamond_search_luma(ctx.handle, C.byref(r), d_src.data_ptr(), d_xy.data_ptr(),
                                            d_c.data_ptr(), 8, len(mbs), d_out.data_ptr())
    assert st == 0
    ctx.synchronize()
    got = np.frombuffer(d_out.cpu().numpy().tobytes(), vp8a.abi.SEARCH_RESULT_DTYPE)
    assert sr_tuples(got) == sr_tuples(want)
