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
    # rd_lambda is finite and non-negative.
    for lam in (-1.0, float("nan"), float("inf")):
        with pytest.raises(vp8a.Vp8aError, match="InvalidArgument"):
            vp8a.analyse_inter_frame(ctx, frames[1], [vp8a.pad_to_mb(*frames[0])], [1], lam)


def test_analysis_and_lf_device_resident(ctx, oracle):
    # Every buffer (planes, ids, outputs) in device memory: the calls are
    # stream-ordered and must match the host-buffer results.
    import ctypes as C

    torch = pytest.importorskip("torch")
    frames, _ = synth.make_sequence(96, 64, 4, seed=77, pieces=2, occluders=1)
    refs = refs_for(frames, 2)
    host = vp8a.analyse_inter_frame(ctx, frames[2], refs, [1, 2, 3], 72.0)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    cur = [d(p) for p in frames[2]]
    drefs = [[d(p) for p in r] for r in refs]
    ids = d(np.array([1, 2, 3], np.uint8))
    out = torch.zeros(host.size * abi.MB_DECISION_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    lib = vp8a.load()
    f = vp8a.i420(*cur)
    pl = (abi.Planes * 3)(*[vp8a.planes(*r) for r in drefs])
    ctxs = abi.default_mv_contexts()
    st = lib.vp8a_analyse_inter_frame(ctx.handle, C.byref(f), C.cast(pl, C.c_void_p), ids.data_ptr(), 3,
                                      C.byref(ctxs), 72.0, out.data_ptr(), None)
    assert st == 0, lib.vp8a_last_error()
    ctx.synchronize()
    got = np.frombuffer(out.cpu().numpy().tobytes(), abi.MB_DECISION_DTYPE).reshape(host.shape)
    assert_same(got, host)
    recon, has = synth.quantised_recon(vp8a.pad_to_mb(*frames[2]))
    mbs = vp8a.lf_info_from_decisions(host, has)
    base = abi.filter_config(0, 0)
    want = vp8a.select_filter_params(ctx, recon, mbs, base, frames[2])
    drec = [d(p) for p in recon]
    dm = d(mbs.view(np.uint8))
    lv = torch.zeros(1, dtype=torch.uint8, device="cuda")
    sh = torch.zeros(1, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    st = lib.vp8a_select_filter_params(ctx.handle, C.byref(vp8a.planes(*drec)), dm.data_ptr(), C.byref(base),
                                       C.byref(vp8a.source(*cur)), lv.data_ptr(), sh.data_ptr())
    assert st == 0, lib.vp8a_last_error()
    ctx.synchronize()
    assert (int(lv.item()), int(sh.item())) == want


@pytest.mark.parametrize("planes", [True, False])
def test_analysis_with_and_without_subpel_planes(oracle, planes):
    # The half- and quarter-pel refinements read precomputed sub-pel planes
    # (default) or synthesise each candidate in the wavefront; both give the
    # oracle's decisions and traces. GOLDEN is four frames back (up to 32
    # px of motion), which puts vectors near the frame edges.
    frames, _ = synth.make_sequence(320, 240, 7, seed=57, pieces=6, occluders=5)
    refs = refs_for(frames, 4)
    ids = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]
    lam = vp8a.rd_lambda(30)
    want, wtr = oracle.analyse_inter_frame(frames[4], refs, ids, lam, trace=True)
    with vp8a.Context(0) as c:
        c.set_subpel_planes(planes)
        got, gtr = vp8a.analyse_inter_frame(c, frames[4], refs, ids, lam, trace=True)
    assert np.array_equal(gtr, wtr)
    assert_same(got, want)


def test_analysis_with_proposals(ctx, oracle):
    # A proposed vector per (MB, reference) is a second NEWMV candidate:
    # random vectors (some zero, some beyond +-1023, some close to the true
    # motion) give exactly the oracle's decisions, and good ones are taken.
    frames, _ = synth.make_sequence(320, 240, 7, seed=31, pieces=5, occluders=4)
    refs = refs_for(frames, 3)
    ids = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]
    lam = vp8a.rd_lambda(44)
    rng = np.random.default_rng(5)
    n = 20 * 15
    prop = np.zeros((n, 3), abi.MV_DTYPE)
    prop["row"] = rng.integers(-40, 41, (n, 3))
    prop["col"] = rng.integers(-40, 41, (n, 3))
    prop[rng.random((n, 3)) < 0.1] = (0, 0)
    far = rng.random((n, 3)) < 0.05
    prop["col"][far] = 1100
    want = oracle.analyse_inter_frame(frames[3], refs, ids, lam, proposals=prop, threads=8)
    got = vp8a.analyse_inter_frame(ctx, frames[3], refs, ids, lam, proposals=prop)
    assert_same(got, want)
    # Proposals the search cannot reach are taken: the frame is the
    # reference moved 30 px right, and every MB proposes that vector.
    frames, _ = synth.make_sequence(128, 96, 1, seed=4)
    ref = vp8a.pad_to_mb(*frames[0])
    y = frames[0][0]
    cur = (np.ascontiguousarray(np.concatenate([y[:, 30:], np.repeat(y[:, -1:], 30, axis=1)], axis=1)),
           frames[0][1], frames[0][2])
    prop = np.zeros((48, 1), abi.MV_DTYPE)
    prop["col"] = 120
    want = oracle.analyse_inter_frame(cur, [ref], [1], lam, proposals=prop)
    got = vp8a.analyse_inter_frame(ctx, cur, [ref], [1], lam, proposals=prop)
    assert_same(got, want)
    assert ((want["mode"] == abi.MODE_NEW) & (want["mv"]["col"] == 120)).any()


def test_batched_analysis_with_proposals(ctx, oracle):
    # vp8a_analyse_inter_frames_proposals: a work list of frames of two sizes,
    # some jobs with proposal vectors and one without, each equal to the
    # oracle's single-frame decision with (or without) its proposals.
    ids = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]
    lam = vp8a.rd_lambda(44)
    rng = np.random.default_rng(9)
    jobs, wants = [], []
    for (w, h), seed, with_props in (((320, 240), 31, True), ((176, 144), 7, False), ((176, 144), 8, True)):
        frames, _ = synth.make_sequence(w, h, 7, seed=seed, pieces=5, occluders=4)
        refs = refs_for(frames, 3)
        n = ((w + 15) // 16) * ((h + 15) // 16)
        job = dict(frame=frames[3], refs=refs, ref_ids=ids, lam=lam)
        prop = None
        if with_props:
            prop = np.zeros((n, 3), abi.MV_DTYPE)
            prop["row"] = rng.integers(-40, 41, (n, 3))
            prop["col"] = rng.integers(-40, 41, (n, 3))
            prop[rng.random((n, 3)) < 0.1] = (0, 0)
            job["proposals"] = prop
        jobs.append(job)
        wants.append(oracle.analyse_inter_frame(frames[3], refs, ids, lam, proposals=prop, threads=8))
    got = vp8a.analyse_inter_frames(ctx, jobs)
    for g, w_ in zip(got, wants):
        assert_same(g, w_)
