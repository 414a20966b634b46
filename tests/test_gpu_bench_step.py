"""Parity of the benchmarked step itself: bench.py's device step (GpuStep) on
the bench's own workload — 1920x1080, seed 20261203, P frame 8 against
LAST = frame 7, GOLDEN = frame 0 and the ARNR anchor of frames 9-15 (centre
12), qi 44 — must give the oracle's outputs exactly: the MB-padded ALTREF
anchor, every MB decision, the reconstruction, the loop-filter records, all
512 entries of the 64 x 8 candidate table (505 distinct candidates; level 0
is one entry for every sharpness) and the walk's (level, sharpness). This is
the same comparison bench.py prints as `parity` in its JSON line."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def test_bench_step_matches_oracle(ctx, oracle):
    import torch

    import bench
    import vp8a

    frames, digest = bench.make_inputs(bench.SEED)
    gs = bench.GpuStep(ctx, frames, vp8a.load(), torch, 0)
    choice = None
    for _ in range(2):  # two steps in a row: buffers are reused, results must not drift
        choice = gs.step()
    got = bench.gpu_step_outputs(gs, choice)
    want = bench.cpu_step(oracle, frames, os.cpu_count() or 1)
    ok, detail = bench.step_parity(got, want)
    assert ok, detail
    # The comparison must be about real work: more than one mode, coded
    # residual, and a full table of distinct finite SSDs.
    dec = got["decisions"]
    assert len(np.unique(dec["mode"])) >= 2
    assert got["lf_info"]["has_coeffs"].any() and not got["lf_info"]["has_coeffs"].all()
    t = got["lf_table"].reshape(64, 8)
    assert (t < np.uint64(1) << np.uint64(63)).all()
    assert len(np.unique(t[1:])) > 100
