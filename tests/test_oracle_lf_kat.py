"""Pins the oracle's §15 loop filter against the reference's hand-derived
known-answer tests (src/loop_filter.rs:2632-3200), ported case by case."""
import numpy as np

from vp8a import abi


def test_derive_kats(oracle):
    d = oracle.lf_derive
    assert d(30, 0, True)[0] == 30 and d(0, 0, True)[0] == 1
    assert d(20, 2, True)[0] == 7 and d(10, 1, True)[0] == 5
    assert d(40, 7, True)[0] == 2 and d(8, 5, True)[0] == 2
    assert [d(l, 0, True)[1] for l in (45, 40, 39, 15, 14)] == [2, 2, 1, 1, 0]
    assert [d(l, 0, False)[1] for l in (45, 40, 39, 20, 19, 15, 14)] == [3, 3, 2, 2, 1, 1, 0]
    assert d(30, 0, True)[2:] == (94, 90)
    assert d(63, 0, True)[2:] == (193, 189)


def test_simple_segment_kats(oracle):
    assert list(oracle.simple_segment(1, [10, 10, 200, 200])) == [10, 10, 200, 200]
    s = oracle.simple_segment(255, [100, 100, 116, 116])
    assert s[1] >= 100 and s[2] <= 116 and s[2] - s[1] < 16 and s[0] == 100 and s[3] == 116


def test_common_adjust_hand_derived(oracle):
    a, s = oracle.common_adjust(False, [100, 100, 108, 108])
    assert a == 3 and list(s) == [100, 103, 105, 108]
    a, s = oracle.common_adjust(True, [90, 100, 108, 120])
    assert a == -1 and s[1] == 99 and s[2] == 109


def test_subblock_and_mb_filter_kats(oracle):
    seg = [10, 200, 100, 100, 108, 108, 108, 108]
    assert list(oracle.subblock_filter(0, 5, 255, seg)) == seg
    before = np.array([100, 100, 100, 100, 110, 110, 110, 110])
    s = oracle.subblock_filter(50, 100, 255, before)
    assert s[3] > before[3] and s[4] < before[4] and s[2] >= before[2] and s[5] <= before[5]
    before = np.array([100, 100, 100, 110, 120, 120, 120, 120])
    s = oracle.subblock_filter(0, 100, 255, before)
    assert s[2] == before[2] and s[5] == before[5] and s[3] > before[3] and s[4] < before[4]
    assert list(oracle.mb_filter(0, 5, 255, seg)) == seg
    s = oracle.mb_filter(0, 100, 255, before)
    assert s[1] == before[1] and s[6] == before[6] and s[3] > before[3] and s[4] < before[4]
    # mb_filter_low_hev_hand_derived (:2951).
    assert list(oracle.mb_filter(50, 100, 255, [100, 100, 100, 100, 116, 116, 116, 116])) == [
        100, 102, 104, 107, 109, 112, 114, 116]


def _mb(y_mode_b=False, seg=-1, ref=abi.REF_INTRA, mode=abi.MODE_NONE, coeffs=False):
    m = np.zeros(1, abi.MB_LF_INFO_DTYPE)
    m["y_mode_is_bpred"] = int(y_mode_b)
    m["segment_id"] = seg
    m["ref_frame"] = ref
    m["inter_mode"] = mode
    m["has_coeffs"] = int(coeffs)
    return m


def test_mb_filter_level_kats(oracle):
    c = abi.filter_config(20, 0, key_frame=True)
    lvl = oracle.mb_filter_level
    assert lvl(c, _mb()) == 20 and lvl(c, _mb(seg=3)) == 20
    c = abi.filter_config(20, 0, key_frame=True, segmentation_enabled=1, segment_lf_level=[5, -8, 0, 0])
    assert lvl(c, _mb(seg=0)) == 25 and lvl(c, _mb(seg=1)) == 12
    c = abi.filter_config(20, 0, key_frame=True, segmentation_enabled=1, segment_abs=1,
                          segment_lf_level=[40, 0, 63, 7])
    assert (lvl(c, _mb(seg=0)), lvl(c, _mb(seg=2)), lvl(c, _mb(seg=1))) == (40, 63, 0)
    c = abi.filter_config(20, 0, key_frame=True, segmentation_enabled=1, segment_lf_level=[60, -40, 0, 0])
    assert lvl(c, _mb(seg=0)) == 63 and lvl(c, _mb(seg=1)) == 0
    c = abi.filter_config(20, 0, key_frame=True, delta_enabled=1, ref_delta_current=4, bpred_mode_delta=-3)
    assert lvl(c, _mb()) == 24 and lvl(c, _mb(y_mode_b=True)) == 21
    c = abi.filter_config(62, 0, key_frame=True, delta_enabled=1, ref_delta_current=10)
    assert lvl(c, _mb()) == 63
    c = abi.filter_config(2, 0, key_frame=True, delta_enabled=1, ref_delta_current=-10)
    assert lvl(c, _mb()) == 0
    c = abi.filter_config(20, 0, key_frame=True, delta_enabled=0, ref_delta_current=30, bpred_mode_delta=30)
    assert lvl(c, _mb(y_mode_b=True)) == 20
    # Inter deltas (calculate_mb_filter_level_inter, :1280): ref + mode.
    c = abi.filter_config(20, 0, delta_enabled=1, ref_delta_last=2, ref_delta_golden=-3, ref_delta_altref=5,
                          zero_mv_mode_delta=1, other_mv_mode_delta=-2, split_mv_mode_delta=4)
    assert lvl(c, _mb(ref=abi.REF_LAST, mode=abi.MODE_ZERO)) == 23
    assert lvl(c, _mb(ref=abi.REF_GOLDEN, mode=abi.MODE_NEW)) == 15
    assert lvl(c, _mb(ref=abi.REF_ALTREF, mode=abi.MODE_SPLIT)) == 29


def _flat(value, mb_cols, mb_rows):
    return (np.full((mb_rows * 16, mb_cols * 16), value, np.uint8),
            np.full((mb_rows * 8, mb_cols * 8), value, np.uint8),
            np.full((mb_rows * 8, mb_cols * 8), value, np.uint8))


def test_filter_frame_level_zero_is_noop(oracle):
    y, u, v = _flat(100, 2, 1)
    y[:, 16:32] = 200
    mbs = np.concatenate([_mb(), _mb()])
    out = oracle.filter_frame((y, u, v), mbs, abi.filter_config(0, 0, key_frame=True))
    assert np.array_equal(out[0], y)


def test_filter_frame_normal_mb_edge_hand_derived(oracle):
    y, u, v = _flat(100, 2, 1)
    y[:, 16:32] = 110
    mbs = np.concatenate([_mb(), _mb()])
    fy, fu, fv = oracle.filter_frame((y, u, v), mbs, abi.filter_config(20, 0, key_frame=True))
    for r in range(16):
        assert list(fy[r, 13:19]) == [101, 103, 104, 106, 107, 109]
        assert fy[r, 12] == y[r, 12] and fy[r, 19] == y[r, 19] and fy[r, 0] == 100 and fy[r, 31] == 110
    assert np.array_equal(fu, u) and np.array_equal(fv, v)


def test_filter_frame_leftmost_mb_filters_top_edge_only(oracle):
    y, u, v = _flat(100, 1, 2)
    y[16:32, :] = 120
    u[8:16, :] = 120
    mbs = np.concatenate([_mb(), _mb()])
    fy, fu, _ = oracle.filter_frame((y, u, v), mbs, abi.filter_config(20, 0, key_frame=True))
    assert not np.array_equal(fy[13:19], y[13:19])  # top MB edge at row 16 filtered
    assert np.array_equal(fy[:, :], fy[:, :1].repeat(16, 1))  # columns identical: no vertical edge
    assert not np.array_equal(fu, u)
