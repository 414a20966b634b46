"""Self-consistency pins of the oracle's RD-effort inter search
(src/encoder/inter_search.rs:198-552, :846-1060). The reference has no unit
tests for this module; its integration tests check decoded pictures. These
check the properties the search's listing implies: the shared half-pel
planes give the same prediction as the six-tap synthesis, every result's
cost is SAD + sqrt(lambda) * bits, and exact translations are recovered."""
import math

import numpy as np
import pytest

import vp8a
from vp8a import abi, synth


@pytest.fixture(scope="module")
def case(oracle):
    frames, _ = synth.make_sequence(160, 96, 5, seed=12, pieces=3, occluders=2)
    refs = [vp8a.pad_to_mb(*frames[2]), vp8a.pad_to_mb(*frames[0]), vp8a.pad_to_mb(*frames[4])]
    dec = oracle.analyse_inter_frame(frames[3], refs, [1, 2, 3], oracle.rd_lambda(44))
    return frames, refs, oracle.neighbours_from_decisions(dec)


@pytest.mark.parametrize("effort", [0, 1, 2, 3])
def test_rd_costs_and_sads_consistent(oracle, case, effort):
    frames, refs, nb = case
    lam = oracle.rd_lambda(44)
    out = oracle.rd_inter_search(frames[3], refs, [1, 2, 3], lam, 48, effort, nb)
    ls = math.sqrt(lam)
    from util import extract_mbs

    mbs, xy = extract_mbs(frames[3][0], out.shape[0], out.shape[1])
    for i, o in enumerate(out.reshape(-1)):
        assert o["cost"] == float(o["sad"]) + ls * o["bits"]
        k = [1, 2, 3].index(int(o["ref_frame"]))
        want = oracle.mb_luma_sad_at_mv(refs[k][0], mbs[i:i + 1], xy[i:i + 1],
                                        [[int(o["mv"]["row"]), int(o["mv"]["col"])]])[0]
        assert int(o["sad"]) == int(want)


def test_rd_recovers_translation(oracle):
    # Frame 1 is frame 0 moved by an exact quarter-pel vector: interior MBs
    # must find it (zero residual).
    frames, offs = synth.make_sequence(96, 96, 2, seed=4)
    ref = vp8a.pad_to_mb(*frames[0])
    dr, dc = offs[1]
    moved = synth.translate(frames[0][0], 2 * dr, 2 * dc)
    cur = (moved, frames[1][1], frames[1][2])
    n = 36
    nb = np.zeros(n * 3, abi.MB_INFO_DTYPE)
    out = oracle.rd_inter_search(cur, [ref], [1], oracle.rd_lambda(44), 48, 3, nb)
    inner = out[1:-1, 1:-1].reshape(-1)
    hits = sum(1 for o in inner if (int(o["mv"]["row"]), int(o["mv"]["col"])) == (-dr, -dc) or o["sad"] == 0)
    assert hits >= len(inner) // 2
