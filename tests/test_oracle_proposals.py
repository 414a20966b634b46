"""The proposal option of the oracle's exhaustive analysis (a second NEWMV
candidate per MB and reference): zero vectors are no candidates, so all-zero
proposals leave every decision as it is; a proposal is taken only when its
cost beats the searched vector's."""
import numpy as np

import vp8a
from vp8a import abi, synth


def test_zero_proposals_change_nothing(oracle):
    frames, _ = synth.make_sequence(96, 64, 4, seed=13, pieces=3, occluders=2)
    refs = [vp8a.pad_to_mb(*frames[2]), vp8a.pad_to_mb(*frames[0])]
    lam = oracle.rd_lambda(44)
    plain = oracle.analyse_inter_frame(frames[3], refs, [1, 2], lam)
    zero = np.zeros((plain.size, 2), abi.MV_DTYPE)
    got = oracle.analyse_inter_frame(frames[3], refs, [1, 2], lam, proposals=zero)
    assert got.tobytes() == plain.tobytes()


def test_proposal_of_an_out_of_reach_translation_is_taken(oracle):
    # The frame is the reference moved 30 px right: beyond the diamond's
    # reach from the zero predictor, so the plain search misses it. With the
    # true vector proposed for every MB the first MBs take it as NEWMV and
    # the rest follow (NEWMV or the census vectors), every MB's total cost
    # is at most the plain one, and most interior MBs code it.
    frames, _ = synth.make_sequence(128, 96, 1, seed=4)
    ref = vp8a.pad_to_mb(*frames[0])
    y = frames[0][0]
    moved = np.concatenate([y[:, 30:], np.repeat(y[:, -1:], 30, axis=1)], axis=1)
    cur = (np.ascontiguousarray(moved), frames[0][1], frames[0][2])
    lam = oracle.rd_lambda(44)
    n = 8 * 6
    prop = np.zeros((n, 1), abi.MV_DTYPE)
    prop["row"], prop["col"] = 0, 120
    plain = oracle.analyse_inter_frame(cur, [ref], [1], lam)
    got = oracle.analyse_inter_frame(cur, [ref], [1], lam, proposals=prop)
    inner = got[1:-1, :-3].reshape(-1)
    hits = sum(1 for o in inner if (int(o["mv"]["row"]), int(o["mv"]["col"])) == (0, 120))
    plain_hits = sum(1 for o in plain[1:-1, :-3].reshape(-1) if (int(o["mv"]["row"]), int(o["mv"]["col"])) == (0, 120))
    assert hits >= len(inner) // 2 and plain_hits == 0
    assert got["total"].sum() < 0.5 * plain["total"].sum()
    assert (got["mode"] == abi.MODE_NEW).any()
