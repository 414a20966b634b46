"""The oracle's §13 trellis quantiser (oracle/trellis.c, restating
trellis_scan_direct, src/encoder.rs:3468-3582) against the reference's own
tests of it, ported:

* trellis_basis_norm_distortion_tracks_pixel_ssd (src/encoder.rs:15856): the
  IDCT basis norms lie in 0.24..0.26;
* level_rate_matches_coeff_token_bits / the token tree: coeff_token_bits
  equals a walk of the RFC 6386 §13.2 coefficient tree written here from
  the RFC's tree array;
* trellis_lut_and_early_exit_match_reference (src/encoder.rs:14834): the
  production scan equals the test module's listing
  (trellis_quantize_block_reference, src/encoder.rs:14269-14500), restated
  here in Python over the same magnitude regimes, block types, entry
  contexts, quantisers and lambdas (default probabilities);
* trellis_round_trips_and_never_raises_rd_cost (src/encoder.rs:15910): the
  trellis never raises J = D + lambda * R over plain rounding.
"""
import math

import numpy as np
import pytest

ZIGZAG = [0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15]
BANDS = [0, 1, 2, 3, 6, 4, 5, 6, 6, 6, 6, 6, 6, 6, 6, 7]
# RFC 6386 §13.2 coeff_tree: a node's two children; leaves are -token
# (tokens DCT_0..DCT_4 = 0..4, cat1..cat6 = 5..10, EOB = 11).
TREE = [-11, 2, -0, 4, -1, 6, 8, 12, -2, 10, -3, -4, 14, 16, -5, -6, 18, 20, -7, -8, -9, -10]
PCAT = [[159], [165, 145], [173, 148, 140], [176, 155, 140, 135], [180, 157, 141, 134, 130],
        [254, 254, 243, 230, 196, 177, 153, 140, 133, 130, 129]]
CAT_BASE = [5, 7, 11, 19, 35, 67]
# BlockType (plane index, first coefficient): YAfterY2, Y2, UV, YNoY2.
FIRST = {0: 1, 1: 0, 2: 0, 3: 0}


def token_of(a):
    if a <= 4:
        return a
    return 5 + sum(a > b for b in (6, 10, 18, 34, 66))


def tree_path(token, start):
    """The (node, bit) steps from tree index `start` to the leaf `token` (a
    child > 0 is a node index, else the leaf -child; 0 is DCT_0's leaf, the
    root is never a child)."""
    for bit in (0, 1):
        c = TREE[start + bit]
        if c <= 0 and -c == token:
            return [(start, bit)]
        if c > 0:
            sub = tree_path(token, c)
            if sub is not None:
                return [(start, bit)] + sub
    return None


def token_bits_by_tree(oracle, probs, pwz, level):
    token = token_of(level)
    bits = 0.0
    for node, bit in tree_path(token, 2 if pwz else 0):
        bits += oracle.bool_bits(probs[node >> 1], bit)
    if token >= 5:
        cat = token - 5
        extra = level - CAT_BASE[cat]
        n = len(PCAT[cat])
        for j, p in enumerate(PCAT[cat]):
            bits += oracle.bool_bits(p, (extra >> (n - 1 - j)) & 1)
    if level != 0:
        bits += oracle.bool_bits(128, 0)
    return bits


def default_probs():
    import os
    import re

    text = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                             "vp8_tables.h")).read()
    body = text[text.index("VO_DEFAULT_COEF_PROBS"):]
    body = body[body.index("{"):body.index(";")]
    nums = [int(x) for x in re.findall(r"\d+", body)]
    return np.array(nums, np.uint8).reshape(4, 8, 3, 11)


def test_basis_norms(oracle):
    norms = oracle.idct_basis_norm_sq()
    assert ((norms > 0.24) & (norms < 0.26)).all()
    assert norms[0] == 0.25


def test_coeff_token_bits_walk_the_rfc_tree(oracle):
    probs = default_probs()
    levels = list(range(0, 80)) + [100, 500, 2047, 2048]
    for plane in range(4):
        for i in range(16):
            for ctx in range(3):
                p = probs[plane][BANDS[i]][ctx]
                for pwz in (0, 1):
                    for lv in levels:
                        assert oracle.coeff_token_bits(plane, i, ctx, pwz, lv) == token_bits_by_tree(oracle, p, pwz,
                                                                                                       lv), \
                            (plane, i, ctx, pwz, lv)
                assert oracle.eob_token_bits(plane, i, ctx) == oracle.bool_bits(p[0], 0)


def reference_listing(oracle, block, dc, ac, first_coeff, entry_ctx3, plane, lam, norms):
    """trellis_quantize_block_reference (src/encoder.rs:14269-14500)."""
    if lam <= 0.0:
        raise AssertionError("only the trellis path is compared")
    INF = math.inf
    scan_x = [int(block[ZIGZAG[k]]) for k in range(16)]
    step = [dc if k == 0 else ac for k in range(16)]

    def dist(k, m):
        err = abs(scan_x[k]) - m * step[k]
        return norms[k] * float(err * err)

    suffix = [0.0] * 17
    for k in range(15, first_coeff - 1, -1):
        suffix[k] = suffix[k + 1] + dist(k, 0)
    surv = [(INF, False)] * 3
    surv[entry_ctx3] = (0.0, False)
    choice = [[(INF, 0, 0)] * 3 for _ in range(16)]
    best_term = surv[entry_ctx3][0] + lam * oracle.eob_token_bits(plane, first_coeff, entry_ctx3) + suffix[first_coeff]
    best_pos, best_ctx = -1, entry_ctx3
    for k in range(first_coeff, 16):
        q = step[k]
        m_round = (abs(scan_x[k]) + q // 2) // q
        cands = []
        for c in (m_round, m_round - 1, 0):
            if c >= 0 and c not in cands:
                cands.append(c)
        nxt = [(INF, False)] * 3
        nchoice = [(INF, 0, 0)] * 3
        for in_ctx, (scost, spwz) in enumerate(surv):
            if scost >= INF:
                continue
            for m in cands:
                d = dist(k, m)
                r = oracle.coeff_token_bits(plane, k, in_ctx, spwz, m)
                cost = scost + d + lam * r
                out = 0 if m == 0 else (1 if m == 1 else 2)
                if cost < nxt[out][0]:
                    nxt[out] = (cost, m == 0)
                    nchoice[out] = (cost, m, in_ctx)
        choice[k] = nchoice
        for out, (ccost, lvl, _) in enumerate(nchoice):
            if ccost >= INF or lvl == 0:
                continue
            term = ccost + lam * oracle.eob_token_bits(plane, k + 1, out) + suffix[k + 1] if k + 1 < 16 else ccost
            if term < best_term:
                best_term, best_pos, best_ctx = term, k, out
        surv = nxt
    levels = [0] * 16
    if best_pos >= 0:
        k, ctx = best_pos, best_ctx
        while True:
            _, lvl, prev = choice[k][ctx]
            levels[k] = -lvl if scan_x[k] < 0 else lvl
            if k == first_coeff:
                break
            ctx = prev
            k -= 1
    out = np.zeros(16, np.int16)
    for k in range(16):
        out[ZIGZAG[k]] = levels[k]
    return out


def factors(qi):
    from vp8a import abi
    import vp8a

    return vp8a.dequant_factors(abi.quant_indices(qi))


@pytest.mark.parametrize("qi", [8, 40, 100])
def test_scan_matches_the_test_module_listing(oracle, qi):
    norms = oracle.idct_basis_norm_sq()
    f = factors(qi)  # (y1_dc, y1_ac, y2_dc, y2_ac, uv_dc, uv_ac)
    base_lambda = (f[1] * f[1] / 32.0) * 0.04
    specs = [(1, 0, f[2], f[3]), (0, 0, f[0], f[1]), (3, 1, f[0], f[1]), (2, 2, f[4], f[5])]
    cases = 0
    for plane, entry, dc, ac in specs:
        for scale, offset in ((1, 0), (ac, 0), (ac * 3, 8), (ac * 24, 64)):
            for seed in range(12):
                lcg = ((0xC0FFEE00 + seed) * 2891336453) & 0xFFFFFFFF

                def nxt():
                    nonlocal lcg
                    lcg = (lcg * 1103515245 + 12345) & 0xFFFFFFFF
                    return lcg >> 16

                base = np.zeros(16, np.int16)
                for k in range(16):
                    mag = (nxt() % (scale + offset + 1)) // (1 + k // 4)
                    sign = 1 if nxt() % 2 == 0 else -1
                    base[k] = max(-2048, min(2047, sign * mag))
                for lam in (base_lambda * 0.25, base_lambda, base_lambda * 6.0):
                    want = reference_listing(oracle, base, dc, ac, FIRST[plane], entry, plane, lam, norms)
                    got = oracle.trellis_quantize_block(base, dc, ac, FIRST[plane], plane, lam, entry_ctx3=entry)
                    assert np.array_equal(got, want), (plane, entry, scale, seed, lam)
                    cases += 1
    assert cases == 4 * 4 * 12 * 3


def block_bits(oracle, plane, first_coeff, scan_q):
    """The §13.3 token bits of a block in scan order (entry context 0):
    each coded level with the context of the one before, then the EOB after
    the last non-zero one (none at position 16)."""
    nz = [k for k in range(first_coeff, 16) if scan_q[k] != 0]
    if not nz:
        return oracle.eob_token_bits(plane, first_coeff, 0)
    last = nz[-1]
    bits, ctx, pwz = 0.0, 0, False
    for k in range(first_coeff, last + 1):
        a = abs(int(scan_q[k]))
        bits += oracle.coeff_token_bits(plane, k, ctx, pwz, a)
        ctx, pwz = (0 if a == 0 else (1 if a == 1 else 2)), a == 0
    if last + 1 < 16:
        bits += oracle.eob_token_bits(plane, last + 1, ctx)
    return bits


def test_trellis_never_raises_rd_cost(oracle):
    import vp8a  # noqa: F401

    norms = oracle.idct_basis_norm_sq()
    f = factors(40)
    lam = (f[1] * f[1] / 32.0) * 0.04
    dc, ac = f[4], f[5]
    fewer = 0
    for seed in range(32):
        st = (0xBEEF + seed * 0x9E3D) & 0xFFFFFFFF
        src = np.zeros(16, np.int32)
        for i in range(16):
            st = (st * 1103515245 + 12345) & 0xFFFFFFFF
            src[i] = min(255, max(0, 128 + (st >> 15) % 90 - 45))
        base = oracle.forward_dct_4x4((src - 128).astype(np.int16))
        plain = oracle.enc_quantize_block(base, dc, ac)
        trel = oracle.trellis_quantize_block(base, dc, ac, 0, 2, lam)

        def cost(qb):
            sx = [int(base.reshape(16)[ZIGZAG[k]]) for k in range(16)]
            sq = [int(qb.reshape(16)[ZIGZAG[k]]) for k in range(16)]
            d = sum(norms[k] * float((abs(sx[k]) - abs(sq[k]) * (dc if k == 0 else ac)) ** 2) for k in range(16))
            return d + lam * block_bits(oracle, 2, 0, sq)

        assert cost(trel) <= cost(plain) + 1e-6, seed
        fewer += int(np.count_nonzero(trel) < np.count_nonzero(plain))
    assert fewer > 0
