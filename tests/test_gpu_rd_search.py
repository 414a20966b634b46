"""Parity: the RD-effort inter search kernel (decide_mb_rd's search part,
through the C ABI) reproduces the oracle exactly for every effort level."""
import numpy as np
import pytest

import vp8a
from vp8a import abi, synth

pytestmark = pytest.mark.gpu

FIELDS = ["ref_frame", "mode", "n_searched", "leader", "mv", "sad", "cost", "bits", "found"]


def check(got, want):
    for f in FIELDS:
        if not np.array_equal(got[f], want[f]):
            bad = np.argwhere(got[f] != want[f])
            raise AssertionError(f"{f} differs at {bad[:5].tolist()}")


def case(w, h, seed, n=5):
    frames, _ = synth.make_sequence(w, h, n, seed=seed, pieces=3, occluders=2)
    refs = [vp8a.pad_to_mb(*frames[2]), vp8a.pad_to_mb(*frames[0]), vp8a.pad_to_mb(*frames[min(4, n - 1)])]
    return frames, refs


@pytest.mark.parametrize("effort", [0, 1, 2, 3])
@pytest.mark.parametrize("qi", [10, 44, 100])
def test_rd_search_parity(ctx, oracle, effort, qi):
    frames, refs = case(320, 240, 41)
    lam = vp8a.rd_lambda(qi)
    y1_ac = [4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31,
             32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48][min(qi, 44)] if qi <= 44 else 135
    dec = oracle.analyse_inter_frame(frames[3], refs, [1, 2, 3], lam)
    nb = oracle.neighbours_from_decisions(dec)
    got = vp8a.rd_inter_search(ctx, frames[3], refs, [1, 2, 3], lam, y1_ac, effort, nb)
    want = oracle.rd_inter_search(frames[3], refs, [1, 2, 3], lam, y1_ac, effort, nb)
    check(got, want)


@pytest.mark.parametrize("w,h,nrefs", [(17, 33, 1), (72, 40, 2), (160, 16, 3)])
def test_rd_search_odd_sizes(ctx, oracle, w, h, nrefs):
    frames, refs = case(w, h, w + h)
    lam = vp8a.rd_lambda(60)
    dec = oracle.analyse_inter_frame(frames[3], refs[:nrefs], [1, 2, 3][:nrefs], lam)
    nb = oracle.neighbours_from_decisions(dec)
    for effort in range(4):
        got = vp8a.rd_inter_search(ctx, frames[3], refs[:nrefs], [1, 2, 3][:nrefs], lam, 70, effort, nb)
        want = oracle.rd_inter_search(frames[3], refs[:nrefs], [1, 2, 3][:nrefs], lam, 70, effort, nb)
        check(got, want)


def test_rd_search_1080p_balanced(ctx, oracle):
    frames, refs = case(1920, 1080, 9, n=5)
    lam = vp8a.rd_lambda(44)
    dec = vp8a.analyse_inter_frame(ctx, frames[3], refs, [1, 2, 3], lam)
    nb = vp8a.neighbours_from_decisions(dec)
    got = vp8a.rd_inter_search(ctx, frames[3], refs, [1, 2, 3], lam, 48, abi.EFFORT_BALANCED, nb)
    want = oracle.rd_inter_search(frames[3], refs, [1, 2, 3], lam, 48, abi.EFFORT_BALANCED, nb, threads=8)
    check(got, want)


# The hand-derived known-answer cases (rd_kat_cases; their values are
# asserted on the oracle in test_oracle_rd_search_kat.py) on the device:
# every output field equal to the oracle's, and the key answers directly.
@pytest.mark.parametrize("effort", [0, 1, 2, 3])
def test_rd_search_known_answers_on_device(ctx, oracle, effort):
    import rd_kat_cases as K

    src, ref = K.ramp_case()
    nb = K.intra_neighbours(K.RAMP_W // 16, K.RAMP_H // 16)
    got = vp8a.rd_inter_search(ctx, src, [ref, ref], [1, 2], 0.5, 8, effort, nb)
    check(got, oracle.rd_inter_search(src, [ref, ref], [1, 2], 0.5, 8, effort, nb))
    f = K.mb_of(got, K.RAMP_MB)["found"][0]
    assert (int(f["mv"]["col"]), int(f["sad"])) == K.RAMP_WHOLE[effort]
    for half in (False, True):
        fsrc, fref, fnb = K.far_case(5 if half else 3, half_pel_source=half)
        got = vp8a.rd_inter_search(ctx, fsrc, [fref], [1], 0.5, 8, effort, fnb)
        check(got, oracle.rd_inter_search(fsrc, [fref], [1], 0.5, 8, effort, fnb))
        o = K.mb_of(got, K.FAR_MB)
        assert int(o["found"][0]["mv"]["col"]) == 1020 and int(o["mv"]["col"]) != 1022
