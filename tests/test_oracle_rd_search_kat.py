"""Known answers of the RD-effort inter search on the oracle (the CPU
restatement), derived by hand from src/encoder/inter_search.rs (see
rd_kat_cases): descent shape per effort, the good_enough gate, the
reference-loop stop, the +-255 px range cap and the half/quarter-pel
vector gates. tests/test_gpu_rd_search.py runs the same cases on the
device."""
import math

import numpy as np
import pytest

import vp8a
from vp8a import abi

import rd_kat_cases as K

LAM = 0.5  # rd_lambda(0): the SAD term dominates every rate term here


def run(oracle, src, refs, ids, y1_ac, effort, nb):
    return oracle.rd_inter_search(src, refs, ids, LAM, y1_ac, effort, nb)


@pytest.mark.parametrize("effort", [0, 1, 2, 3])
def test_ramp_descent_per_effort(oracle, effort):
    src, ref = K.ramp_case()
    nb = K.intra_neighbours(K.RAMP_W // 16, K.RAMP_H // 16)
    o = K.mb_of(run(oracle, src, [ref], [abi.REF_LAST], 8, effort, nb), K.RAMP_MB)
    col, sad = K.RAMP_WHOLE[effort]
    assert (int(o["found"][0]["mv"]["row"]), int(o["found"][0]["mv"]["col"]), int(o["found"][0]["sad"])) == \
        (0, col, sad)
    assert o["n_searched"] == 1 and o["leader"] == 0


def test_ramp_fastest_half_pel_result(oracle):
    # Fastest refines at half-pel only. On the ramp the half-pel sample
    # right of x is (128 x + 64 + 64) >> 7 = x + 1, so the candidate half a
    # pixel right of 4 px predicts like 5 px: SAD 256 * 35; the diagonal
    # ones have the same SAD and a dearer row differential.
    src, ref = K.ramp_case()
    nb = K.intra_neighbours(K.RAMP_W // 16, K.RAMP_H // 16)
    o = K.mb_of(run(oracle, src, [ref], [abi.REF_LAST], 8, abi.EFFORT_FASTEST, nb), K.RAMP_MB)
    assert (int(o["mv"]["row"]), int(o["mv"]["col"]), int(o["sad"])) == (0, 18, 256 * 35)
    assert o["mode"] == abi.MODE_NEW


@pytest.mark.parametrize("y1_ac,want", [(284, (0, 0, 256 * 10)), (8, (0, 40, 0))])
def test_good_enough_gate(oracle, y1_ac, want):
    # good_enough = 128 * max(1, y1_ac / 8): 4480 for y1_ac 284, 128 for 8.
    # The zero seed's SAD on a ramp moved 10 px is 2560: no descent under
    # the first, the exact 10 px under the second.
    src, ref = K.ramp_case(10)
    nb = K.intra_neighbours(K.RAMP_W // 16, K.RAMP_H // 16)
    o = K.mb_of(run(oracle, src, [ref], [abi.REF_LAST], y1_ac, abi.EFFORT_BALANCED, nb), K.RAMP_MB)
    f = o["found"][0]
    assert (int(f["mv"]["row"]), int(f["mv"]["col"]), int(f["sad"])) == want


@pytest.mark.parametrize("effort,n_searched,second", [(abi.EFFORT_BALANCED, 1, None),
                                                      (abi.EFFORT_FASTEST, 2, (0, 0, 256 * 40))])
def test_reference_loop_stop_and_other_refs(oracle, effort, n_searched, second):
    # Two references holding the same ramp. Balanced finds SAD 0 on the
    # first and stops the reference loop; Fastest's first result (SAD 9216)
    # is not good enough, and the second reference is searched without
    # descent (search_other_refs off): its zero seed.
    src, ref = K.ramp_case()
    nb = K.intra_neighbours(K.RAMP_W // 16, K.RAMP_H // 16)
    o = K.mb_of(run(oracle, src, [ref, ref], [abi.REF_LAST, abi.REF_GOLDEN], 8, effort, nb), K.RAMP_MB)
    assert o["n_searched"] == n_searched
    if second is None:
        assert int(o["found"][1]["sad"]) == 0xFFFFFFFF
    else:
        f = o["found"][1]
        assert (int(f["mv"]["row"]), int(f["mv"]["col"]), int(f["sad"])) == second


def test_range_cap_255_px(oracle):
    # The census seeds point 300 px right; the whole-pel range is capped at
    # 255 px, where the source's MB is an exact copy: SAD 0 at 1020
    # quarter-pels (not 1200).
    src, ref, nb = K.far_case(3)
    o = K.mb_of(run(oracle, src, [ref], [abi.REF_LAST], 8, abi.EFFORT_BALANCED, nb), K.FAR_MB)
    f = o["found"][0]
    assert (int(f["mv"]["row"]), int(f["mv"]["col"]), int(f["sad"])) == (0, 1020, 0)


def cost_of(oracle, ref, src, mb, row, col, census_best):
    """sad + sqrt(lambda) * bits of a NEW vector against the census best
    (the f32 MvCostTable sum)."""
    from util import extract_mbs

    mbs, xy = extract_mbs(src[0], K.FAR_H // 16, K.FAR_W // 16)
    i = mb[1] * (K.FAR_W // 16) + mb[0]
    sad = int(oracle.mb_luma_sad_at_mv(ref[0], mbs[i:i + 1], xy[i:i + 1], [[row, col]])[0])
    c = abi.default_mv_contexts()
    b = np.float32(oracle.mv_component_bits(list(c.p[0]), row - census_best[0])) + \
        np.float32(oracle.mv_component_bits(list(c.p[1]), col - census_best[1]))
    return sad + math.sqrt(LAM) * float(b), sad


@pytest.mark.parametrize("effort", [abi.EFFORT_FASTEST, abi.EFFORT_FAST])
def test_half_and_quarter_gates(oracle, effort):
    # The source MB is the reference's half-pel sample 255.5 px right: an
    # exact match at 1022 quarter-pels. The whole-pel search stops at the
    # 255 px cap (1020); the half-pel candidates at 1022 exceed 1020 and are
    # skipped, so Fastest (no quarter-pel) stays at 1020; Fast's quarter-pel
    # step may go to 1021 (<= 1022) and takes the cheapest of 1019..1021.
    src, ref, nb = K.far_case(5, half_pel_source=True)
    o = K.mb_of(run(oracle, src, [ref], [abi.REF_LAST], 8, effort, nb), K.FAR_MB)
    assert int(o["found"][0]["mv"]["col"]) == 1020
    exact, exact_sad = cost_of(oracle, ref, src, K.FAR_MB, 0, 1022, (0, 1200))
    assert exact_sad == 0  # what the gates keep out of reach
    if effort == abi.EFFORT_FASTEST:
        assert (int(o["mv"]["row"]), int(o["mv"]["col"])) == (0, 1020)
    else:
        costs = {c: cost_of(oracle, ref, src, K.FAR_MB, 0, c, (0, 1200)) for c in (1019, 1020, 1021)}
        best = min(costs, key=lambda c: costs[c][0])
        assert best == 1021
        assert (int(o["mv"]["row"]), int(o["mv"]["col"]), int(o["sad"])) == (0, best, costs[best][1])
