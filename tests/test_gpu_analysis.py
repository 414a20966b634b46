"""Parity: the device wavefront analysis (exhaustive per-MB picker across
LAST/GOLDEN/ALTREF with SPLITMV and the f64 RD decision) reproduces the
oracle's decisions and per-reference search traces exactly."""
import numpy as np
import pytest

import vp8a
from vp8a import abi, synth

pytestmark = pytest.mark.gpu

DEC_FIELDS = ["ref_frame", "mode", "partition", "mv", "j", "total", "split_mvs", "submv_modes"]


def assert_same(got, want):
    for f in DEC_FIELDS:
        g, w = got[f], want[f]
        if not np.array_equal(g, w):
            bad = np.argwhere(g != w) if g.shape == w.shape else None
            raise AssertionError(f"field {f} differs at {bad[:5] if bad is not None else '?'}")


def refs_for(frames, k, arnr=None):
    last = vp8a.pad_to_mb(*frames[k - 1])
    golden = vp8a.pad_to_mb(*frames[max(0, k - 8)])
    altref = vp8a.pad_to_mb(*(arnr if arnr is not None else frames[min(len(frames) - 1, k + 1)]))
    return [last, golden, altref]


@pytest.mark.parametrize("n_refs", [1, 2, 3])
def test_analysis_config1(ctx, oracle, n_refs):
    frames, _ = synth.make_sequence(320, 240, 7, seed=31, pieces=5, occluders=4)
    k = 3
    refs = refs_for(frames, k)[:n_refs]
    ids = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF][:n_refs]
    lam = vp8a.rd_lambda(44)
    got, gtr = vp8a.analyse_inter_frame(ctx, frames[k], refs, ids, lam, trace=True)
    want, wtr = oracle.analyse_inter_frame(frames[k], refs, ids, lam, trace=True)
    assert np.array_equal(gtr, wtr)
    assert_same(got, want)


@pytest.mark.parametrize("w,h,qi", [(72, 40, 10), (17, 33, 90), (160, 16, 44), (16, 160, 127)])
def test_analysis_odd_sizes(ctx, oracle, w, h, qi):
    frames, _ = synth.make_sequence(w, h, 4, seed=w * 3 + h, pieces=3, occluders=2)
    refs = refs_for(frames, 2)
    ids = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]
    lam = vp8a.rd_lambda(qi)
    got, gtr = vp8a.analyse_inter_frame(ctx, frames[2], refs, ids, lam, trace=True)
    want, wtr = oracle.analyse_inter_frame(frames[2], refs, ids, lam, trace=True)
    assert np.array_equal(gtr, wtr)
    assert_same(got, want)


def test_analysis_modes_exercised(ctx):
    # The sequence must exercise NEW, NEAREST/NEAR and SPLITMV decisions
    # for the parity above to mean something.
    frames, _ = synth.make_sequence(320, 240, 7, seed=31, pieces=5, occluders=4)
    got = vp8a.analyse_inter_frame(ctx, frames[3], refs_for(frames, 3), [1, 2, 3], vp8a.rd_lambda(44))
    modes = set(np.unique(got["mode"]).tolist())
    assert abi.MODE_NEW in modes and abi.MODE_SPLIT in modes and len(modes) >= 4


def test_analysis_1080p_three_refs(ctx, oracle):
    frames, _ = synth.make_sequence(1920, 1080, 9, seed=8, pieces=9, occluders=12)
    arnr = oracle.build_arnr_altref(frames[2:9], 3, 3, threads=8)
    refs = refs_for(frames, 8, arnr)
    ids = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]
    lam = vp8a.rd_lambda(44)
    got = vp8a.analyse_inter_frame(ctx, frames[8], refs, ids, lam)
    want = oracle.analyse_inter_frame(frames[8], refs, ids, lam, threads=8)
    assert_same(got, want)


def test_analysis_errors(ctx):
    frames, _ = synth.make_sequence(64, 48, 2, seed=1)
    bad = vp8a.pad_to_mb(*synth.make_sequence(32, 32, 1, seed=2)[0][0])
    with pytest.raises(vp8a.Vp8aError, match="ReferenceDimensionsMismatch"):
        vp8a.analyse_inter_frame(ctx, frames[1], [bad], [1], 72.0)
    with pytest.raises(vp8a.Vp8aError, match="InvalidArgument"):
        vp8a.analyse_inter_frame(ctx, frames[1], [vp8a.pad_to_mb(*frames[0])], [7], 72.0)
