"""Parity of the batched work-list entry points: every job of a batch of
uneven-size frames gets exactly what the single-job call (itself pinned to
the oracle by the other parity tests) gives, and the batches are checked
against the oracle directly on a few jobs.

* vp8a_analyse_inter_frames — the MB rows of many frames in one persistent
  launch (mixed reference counts: one launch per count);
* vp8a_build_arnr_altrefs — one search and one blend launch for every job,
  including pass-through jobs (strength 0, a single frame);
* vp8a_reconstruct_inter_frames — one prediction and one reconstruction
  launch, with segments, both filter sets and intra MBs;
* vp8a_filter_sweeps — the candidate grids of many pictures in one launch,
  whole frames and sampled bands, normal and simple filters.
"""
import numpy as np
import pytest

import vp8a
from vp8a import abi, synth

pytestmark = pytest.mark.gpu

SIZES = [(176, 144), (64, 48), (320, 240), (72, 40), (17, 33), (160, 16), (16, 160), (96, 72)]
IDS = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF]


def stream(w, h, seed, n=4):
    frames, _ = synth.make_sequence(w, h, n, seed=seed, pieces=3, occluders=2)
    return frames


def analysis_jobs(n_refs_cycle=(3, 2, 1)):
    jobs = []
    for i, (w, h) in enumerate(SIZES):
        fr = stream(w, h, 100 + i)
        nr = n_refs_cycle[i % len(n_refs_cycle)]
        refs = [vp8a.pad_to_mb(*fr[2]), vp8a.pad_to_mb(*fr[0]), vp8a.pad_to_mb(*fr[3])][:nr]
        jobs.append(dict(frame=fr[1], refs=refs, ref_ids=IDS[:nr], lam=vp8a.rd_lambda(20 + 10 * i)))
    return jobs


def test_analyse_inter_frames_matches_single_calls(ctx, oracle):
    jobs = analysis_jobs()
    got = vp8a.analyse_inter_frames(ctx, jobs)
    for j, g in zip(jobs, got):
        want = vp8a.analyse_inter_frame(ctx, j["frame"], j["refs"], j["ref_ids"], j["lam"])
        assert np.array_equal(g.view(np.uint8), want.view(np.uint8)), j["frame"][0].shape
    # Two jobs against the oracle directly.
    for k in (0, 4):
        j = jobs[k]
        want = oracle.analyse_inter_frame(j["frame"], j["refs"], j["ref_ids"], j["lam"])
        assert np.array_equal(got[k].reshape(-1).view(np.uint8), np.asarray(want).reshape(-1).view(np.uint8))


def test_analyse_inter_frames_many_small_jobs(ctx):
    # More jobs than resident clusters hold rows: items wrap around the
    # clusters several times, job boundaries fall inside a cluster's turn.
    jobs = []
    for i in range(40):
        w, h = 16 * (1 + i % 5) + i % 3, 16 * (1 + (i * 7) % 4)
        fr = stream(w, h, 500 + i, n=3)
        jobs.append(dict(frame=fr[1], refs=[vp8a.pad_to_mb(*fr[0]), vp8a.pad_to_mb(*fr[2])], ref_ids=IDS[:2],
                         lam=vp8a.rd_lambda(44)))
    got = vp8a.analyse_inter_frames(ctx, jobs)
    for j, g in zip(jobs, got):
        want = vp8a.analyse_inter_frame(ctx, j["frame"], j["refs"], j["ref_ids"], j["lam"])
        assert np.array_equal(g.view(np.uint8), want.view(np.uint8))


def test_build_arnr_altrefs_matches_single_calls(ctx, oracle):
    jobs = []
    for i, (w, h) in enumerate(SIZES):
        fr = stream(w, h, 200 + i, n=5)
        jobs.append((fr, 2, [3, 0, 6, 1][i % 4]))
    jobs.append((stream(48, 32, 9, n=1), 0, 3))  # a single frame: pass-through
    got = vp8a.build_arnr_altrefs(ctx, jobs)
    for (frames, center, strength), g in zip(jobs, got):
        want = vp8a.build_arnr_altref(ctx, frames, center, strength)
        for a, b in zip(g, want):
            assert np.array_equal(a, b)
    frames, center, strength = jobs[2]
    want = oracle.build_arnr_altref(frames, center, strength)
    for a, b in zip(got[2], want):
        assert np.array_equal(a, b)


def test_reconstruct_inter_frames_matches_single_calls(ctx, oracle):
    rng = np.random.default_rng(3)
    ajobs = analysis_jobs(n_refs_cycle=(3,))
    decs = vp8a.analyse_inter_frames(ctx, ajobs)
    jobs = []
    for i, (a, d) in enumerate(zip(ajobs, decs)):
        n = d.size
        d = d.reshape(-1).copy()
        d["ref_frame"][rng.random(n) < 0.1] = abi.REF_INTRA
        seg = rng.integers(-1, 4, n).astype(np.int8) if i % 2 else None
        jobs.append(dict(frame=a["frame"], refs=a["refs"], ref_ids=a["ref_ids"], decisions=d,
                         quant=abi.quant_indices(20 + 13 * i, uv_ac=i - 3), mb_segment=seg,
                         segment_quant=[-10, 5, 30, 0] if i % 2 else None, segment_abs=False,
                         filter_set=abi.FILTER_BILINEAR if i == 3 else abi.FILTER_SIXTAP, full_pixel=i == 3,
                         recon=tuple(np.full(p.shape, 7, np.uint8) for p in a["refs"][0]),
                         lf_info=np.zeros(n, abi.MB_LF_INFO_DTYPE)))
    got = vp8a.reconstruct_inter_frames(ctx, jobs)
    for j, (cf, fl) in zip(jobs, got):
        rec = tuple(np.full(p.shape, 7, np.uint8) for p in j["refs"][0])
        lf = np.zeros(j["decisions"].size, abi.MB_LF_INFO_DTYPE)
        wcf, wfl = vp8a.reconstruct_inter_frame(ctx, j["frame"], j["refs"], j["ref_ids"], j["decisions"],
                                                j["quant"], rec, mb_segment=j["mb_segment"],
                                                segment_quant=j["segment_quant"], full_pixel=j["full_pixel"],
                                                filter_set=j["filter_set"], lf_info=lf)
        for a, b in zip(j["recon"], rec):
            assert np.array_equal(a, b)
        assert np.array_equal(cf, wcf) and np.array_equal(fl, wfl)
        assert np.array_equal(j["lf_info"].view(np.uint8), lf.view(np.uint8))
    j = jobs[1]
    want = tuple(np.full(p.shape, 7, np.uint8) for p in j["refs"][0])
    wcf, wfl, _ = oracle.reconstruct_inter_frame(j["frame"], j["refs"], j["ref_ids"], j["decisions"], j["quant"],
                                                 want, mb_segment=j["mb_segment"], segment_quant=j["segment_quant"])
    for a, b in zip(j["recon"], want):
        assert np.array_equal(a, b)
    assert np.array_equal(got[1][0], wcf)


def lf_job(w, h, seed, every_rows=0, **cfg):
    frames, _ = synth.make_sequence(w, h, 1, seed=seed)
    src = frames[0]
    recon, has = synth.quantised_recon(vp8a.pad_to_mb(*src))
    rng = np.random.default_rng(seed)
    n = has.size
    m = np.zeros(n, abi.MB_LF_INFO_DTYPE)
    m["has_coeffs"] = (rng.random(n) < 0.6) & has.reshape(-1)
    m["ref_frame"] = rng.integers(0, 4, n)
    m["inter_mode"] = np.where(m["ref_frame"] == 0, abi.MODE_NONE, rng.integers(0, 5, n))
    m["y_mode_is_bpred"] = rng.random(n) < 0.2
    m["segment_id"] = rng.integers(-1, 4, n)
    return (recon, m, abi.filter_config(**cfg), src, every_rows)


def test_filter_sweeps_matches_single_calls(ctx, oracle):
    jobs = [lf_job(176, 144, 1, level=0, sharpness=2, delta_enabled=1, ref_delta_last=2),
            lf_job(320, 240, 2, every_rows=3, level=0, sharpness=0),
            lf_job(72, 40, 3, level=0, sharpness=5, simple=True),
            lf_job(17, 33, 4, level=0, sharpness=1, segmentation_enabled=1, segment_lf_level=[0, 5, -9, 30]),
            lf_job(64, 2048, 5, level=0, sharpness=3),  # tall: its own layout
            lf_job(160, 16, 6, level=0, sharpness=7)]
    got = vp8a.filter_sweeps(ctx, jobs)
    for j, g in zip(jobs, got):
        want = vp8a.filter_sweep(ctx, *j)
        assert np.array_equal(g, want)
    recon, m, base, src, er = jobs[2]
    assert np.array_equal(got[2], oracle.filter_sweep(recon, m, base, src, er, threads=8))


def test_batch_empty_and_errors(ctx):
    assert vp8a.analyse_inter_frames(ctx, []) == []
    assert vp8a.filter_sweeps(ctx, []) == []
    fr = stream(32, 32, 1, n=2)
    bad = dict(frame=fr[1], refs=[vp8a.pad_to_mb(*stream(48, 32, 2, n=1)[0])], ref_ids=IDS[:1], lam=1.0)
    good = dict(frame=fr[1], refs=[vp8a.pad_to_mb(*fr[0])], ref_ids=IDS[:1], lam=1.0)
    with pytest.raises(vp8a.Vp8aError) as e:
        vp8a.analyse_inter_frames(ctx, [good, bad])
    assert e.value.status == abi.E_REFERENCE_DIMENSIONS_MISMATCH
    with pytest.raises(vp8a.Vp8aError) as e:
        vp8a.build_arnr_altrefs(ctx, [(fr, 5, 3)])
    assert e.value.status == abi.E_INVALID_ARGUMENT
    # The context stays usable after a rejected batch.
    got = vp8a.analyse_inter_frames(ctx, [good])
    want = vp8a.analyse_inter_frame(ctx, good["frame"], good["refs"], good["ref_ids"], good["lam"])
    assert np.array_equal(got[0].view(np.uint8), want.view(np.uint8))


def test_select_filter_params_batch_matches_single_walks(ctx, oracle):
    # The reference's walk (grid, refine, sharpness) for several pictures of
    # different sizes and configurations, every stage of all of them in one
    # batched launch: each job's pair equals the oracle's own walk.
    from test_gpu_lf import lf_case

    jobs = []
    for i, (size, cfg) in enumerate([((320, 240), dict(sharpness=0)), ((176, 144), dict(sharpness=3)),
                                     ((72, 40), dict(sharpness=0, key_frame=True)),
                                     ((640, 368), dict(sharpness=5, delta_enabled=1, ref_delta_last=4))]):
        src, recon, m = lf_case(*size, seed=300 + i)
        jobs.append((recon, m, abi.filter_config(0, **cfg), src))
    got = vp8a.select_filter_params_batch(ctx, jobs)
    want = [oracle.select_filter_params(r, m, b, s, threads=8) for r, m, b, s in jobs]
    assert got == want
    assert any(lv != 0 for lv, _ in want)
