"""Parity: the §15 filter pass and the §9.4 candidate sweep on the device
reproduce the oracle exactly — filtered planes, every candidate's SSD, and
the (level, sharpness) the reference's searches select."""
import numpy as np
import pytest

import vp8a
from vp8a import abi, synth

pytestmark = pytest.mark.gpu


def lf_case(width, height, seed, frac_bpred=0.2, frac_coeffs=0.6):
    frames, _ = synth.make_sequence(width, height, 1, seed=seed)
    src = frames[0]
    padded = vp8a.pad_to_mb(*src)
    recon, has = synth.quantised_recon(padded)
    rng = np.random.default_rng(seed)
    n = has.size
    m = np.zeros(n, abi.MB_LF_INFO_DTYPE)
    m["has_coeffs"] = (rng.random(n) < frac_coeffs) & has.reshape(-1)
    m["ref_frame"] = rng.integers(0, 4, n)
    m["inter_mode"] = np.where(m["ref_frame"] == 0, abi.MODE_NONE, rng.integers(0, 5, n))
    m["y_mode_is_bpred"] = (rng.random(n) < frac_bpred) | (m["inter_mode"] == abi.MODE_SPLIT)
    m["segment_id"] = rng.integers(-1, 4, n)
    return src, recon, m


CONFIGS = [
    dict(level=20, sharpness=0),
    dict(level=63, sharpness=7),
    dict(level=5, sharpness=3, key_frame=True),
    dict(level=40, sharpness=0, simple=True),
    dict(level=30, sharpness=2, delta_enabled=1, ref_delta_last=3, ref_delta_golden=-9, ref_delta_altref=12,
         ref_delta_current=-2, bpred_mode_delta=4, zero_mv_mode_delta=-5, other_mv_mode_delta=2,
         split_mv_mode_delta=7),
    dict(level=0, sharpness=1, segmentation_enabled=1, segment_abs=1, segment_lf_level=[0, 17, 40, 63]),
    dict(level=25, sharpness=5, segmentation_enabled=1, segment_abs=0, segment_lf_level=[-30, 10, 50, 0]),
]


@pytest.mark.parametrize("cfg", CONFIGS)
@pytest.mark.parametrize("size", [(320, 240), (72, 40), (17, 33)])
def test_filter_frame_parity(ctx, oracle, cfg, size):
    src, recon, m = lf_case(*size, seed=sum(size))
    c = abi.filter_config(**cfg)
    got = vp8a.filter_frame(ctx, recon, m, c)
    want = oracle.filter_frame(recon, m, c)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_filter_frame_hand_derived_on_gpu(ctx):
    y = np.full((16, 32), 100, np.uint8)
    y[:, 16:32] = 110
    u = np.full((8, 16), 100, np.uint8)
    v = u.copy()
    m = np.zeros(2, abi.MB_LF_INFO_DTYPE)
    m["segment_id"] = -1
    fy, fu, fv = vp8a.filter_frame(ctx, (y, u, v), m, abi.filter_config(20, 0, key_frame=True))
    for r in range(16):
        assert list(fy[r, 13:19]) == [101, 103, 104, 106, 107, 109]
    assert np.array_equal(fu, u)


@pytest.mark.parametrize("every_rows", [0, 2, 3, 8])
def test_sweep_table_parity(ctx, oracle, every_rows):
    src, recon, m = lf_case(96, 72, seed=7)
    base = abi.filter_config(0, 2, delta_enabled=1, ref_delta_last=2, zero_mv_mode_delta=-3)
    got = vp8a.filter_sweep(ctx, recon, m, base, src, every_rows)
    want = oracle.filter_sweep(recon, m, base, src, every_rows, threads=8)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("size", [(64, 2048), (48, 2400)])
def test_sweep_tall_pictures(ctx, oracle, size):
    # Tall pictures take the sweep's other shared-memory layouts: 128 MB rows
    # keep compact slot rings (with the next-MB prefetch), 150 rows keep the
    # rings in global memory.
    src, recon, m = lf_case(*size, seed=size[1])
    base = abi.filter_config(0, 1)
    got = vp8a.filter_sweep(ctx, recon, m, base, src, 0)
    want = oracle.filter_sweep(recon, m, base, src, 0, threads=8)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("size,every_rows", [((400, 16), 0), ((4096, 64), 0), ((320, 240), 0), ((320, 240), 3),
                                             ((1920, 96), 0)])
def test_sweep_grid_groups_with_segments_and_deltas(ctx, oracle, size, every_rows):
    # The sweep scores one pass per group of sharpness values whose interior
    # limits agree at every MB level the configuration can produce, and
    # fills the group's table entries from it. Segment and delta levels make
    # the groups uneven; wide and short pictures take few half-warps per
    # step; the oracle scores every (level, sharpness) on its own.
    src, recon, m = lf_case(*size, seed=size[0] + size[1])
    base = abi.filter_config(0, 3, segmentation_enabled=1, segment_abs=0, segment_lf_level=[-20, 4, 9, 0],
                             delta_enabled=1, ref_delta_golden=5, split_mv_mode_delta=-4)
    got = vp8a.filter_sweep(ctx, recon, m, base, src, every_rows)
    want = oracle.filter_sweep(recon, m, base, src, every_rows, threads=8)
    assert np.array_equal(got, want)


def test_sweep_unaligned_strides(ctx, oracle):
    # Row strides that allow neither word nor asynchronous copies.
    src, recon, m = lf_case(96, 72, seed=11)

    def widen(planes, extra):
        out = []
        for p in planes:
            w = np.zeros((p.shape[0], p.shape[1] + extra), np.uint8)
            w[:, : p.shape[1]] = p
            out.append(w[:, : p.shape[1]])
        return out

    rs, ss = widen(recon, 3), widen(src, 5)
    base = abi.filter_config(0, 2)
    got = vp8a.filter_sweep(ctx, rs, m, base, ss, 0)
    want = oracle.filter_sweep(recon, m, base, src, 0, threads=8)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("size,seed", [((320, 240), 3), ((72, 40), 4), ((33, 65), 5)])
def test_selection_parity(ctx, oracle, size, seed):
    src, recon, m = lf_case(*size, seed=seed)
    for bs in (0, 3):
        base = abi.filter_config(0, bs)
        assert vp8a.select_filter_params(ctx, recon, m, base, src) == oracle.select_filter_params(
            recon, m, base, src, threads=8)
        for er, sweep in ((8, False), (16, True), (2, True)):
            assert vp8a.select_filter_params_sampled(ctx, recon, m, base, src, er, sweep) == \
                oracle.select_filter_params_sampled(recon, m, base, src, er, sweep, threads=8)


def test_reconstruction_ssd_parity(ctx, oracle):
    src, recon, _ = lf_case(75, 41, seed=9)
    assert vp8a.reconstruction_ssd(ctx, recon, src) == oracle.reconstruction_ssd(recon, src)


def test_sweep_1080p_full_grid(ctx, oracle):
    src, recon, m = lf_case(1920, 1080, seed=44)
    base = abi.filter_config(0, 0)
    got = vp8a.filter_sweep(ctx, recon, m, base, src, 0)
    # Every level at sharpness 0 and every sharpness at three levels:
    # 85 full-frame candidates of the oracle.
    for lv in range(64):
        assert got[lv, 0] == oracle.score_filter_candidate(recon, m, base, src, lv, 0), lv
    for lv in (1, 31, 63):
        for sh in range(8):
            assert got[lv, sh] == oracle.score_filter_candidate(recon, m, base, src, lv, sh), (lv, sh)
    lvl, sh = oracle.select_from_table(got, 0)
    assert (lvl, sh) == vp8a.select_filter_params(ctx, recon, m, base, src)


def test_lf_errors(ctx):
    src, recon, m = lf_case(32, 32, seed=1)
    with pytest.raises(vp8a.Vp8aError, match="LoopFilterLevelOutOfRange"):
        vp8a.filter_frame(ctx, recon, m, abi.filter_config(64, 0))
    with pytest.raises(vp8a.Vp8aError, match="SharpnessLevelOutOfRange"):
        vp8a.filter_frame(ctx, recon, m, abi.filter_config(10, 8))


def key_frame_case(width, height, seed):
    """An intra picture's §15 side information: every MB intra, some B_PRED."""
    src, recon, m = lf_case(width, height, seed)
    rng = np.random.default_rng(seed + 1)
    m["ref_frame"] = abi.REF_INTRA
    m["inter_mode"] = abi.MODE_NONE
    m["y_mode_is_bpred"] = rng.random(m.size) < 0.4
    m["segment_id"] = -1
    return src, recon, m


@pytest.mark.parametrize("size", [(320, 240), (176, 144), (640, 368)])
def test_key_frame_auto_lf(ctx, oracle, size):
    # encode_keyframe_auto_loop_filter's pick (src/encoder.rs:6638-6655):
    # the sampled search with FilterSampling::for_key_frame, and the full
    # search, on key-frame hev thresholds and intra MBs.
    src, recon, m = key_frame_case(*size, seed=size[0])
    er, sw = oracle.key_frame_sampling(recon[0].shape[0] // 16)
    for bs in (0, 4):
        base = abi.filter_config(0, bs, key_frame=True)
        assert vp8a.select_filter_params_key_frame(ctx, recon, m, base, src) == \
            oracle.select_filter_params_sampled(recon, m, base, src, er, sw, threads=8)
        assert vp8a.select_filter_params_key_frame(ctx, recon, m, base, src, sampled=False) == \
            oracle.select_filter_params(recon, m, base, src, threads=8)


@pytest.mark.parametrize("size", [(640, 368), (1920, 1080)])
def test_sweep_every_launch_shape_gives_the_same_table(oracle, size):
    # The sweep's launch shape (passes per CTA, threads per CTA, prefetch) is
    # picked by measurement or by the cost model; every shape must give the
    # oracle's table.
    src, recon, m = lf_case(*size, seed=size[0] // 8)
    base = abi.filter_config(0, 0)
    want = oracle.filter_sweep(recon, m, base, src, 0, threads=8)
    ran = set()
    with vp8a.Context(0) as c:
        assert np.array_equal(vp8a.filter_sweep(c, recon, m, base, src, 0), want)
        tuned = c.last_sweep_layout()
        assert tuned[0] in (1, 2, 3) and tuned[3] >= 1
        for passes in (1, 2, 3):
            for threads in (1024, 768, 512, 384, 352, 256, 192, 128):
                for pre in (0, 1):
                    c.force_sweep_layout(passes, threads, pre)
                    try:
                        got = vp8a.filter_sweep(c, recon, m, base, src, 0)
                    except vp8a.Vp8aError as e:
                        assert e.status == abi.E_INVALID_ARGUMENT
                        continue
                    assert c.last_sweep_layout()[:3] == (passes, threads, pre)
                    assert np.array_equal(got, want), (passes, threads, pre)
                    ran.add((passes, threads, pre))
        c.force_sweep_layout(0)
        c.set_autotune(False)
        assert np.array_equal(vp8a.filter_sweep(c, recon, m, base, src, 0), want)
    # 1080p's slot rings leave room for one pass per CTA only; smaller
    # pictures fit more shapes.
    assert len(ran) >= (3 if size[0] > 1000 else 6), ran
