"""Pins the oracle's §16.3 census and RD bit costs against the reference's
unit tests (src/near_mv.rs tests, src/motion_vector.rs, src/encoder.rs)."""
import math

import pytest

from vp8a import abi

LAST = abi.REF_LAST


def test_census_kats(oracle):
    b = oracle.mb_info()
    assert oracle.find_near_mvs(b, b, b) == ([(0, 0)] * 3, [0, 0, 0, 0])
    a = oracle.mb_info(LAST, (8, -4))
    mvs, cnt = oracle.find_near_mvs(a, b, b)
    assert cnt[1] == 2 and mvs[1] == (8, -4) and mvs[0] == (8, -4)
    mvs, cnt = oracle.find_near_mvs(b, oracle.mb_info(LAST, (12, 0)), b)
    assert cnt[1] == 2 and mvs[1] == (12, 0)
    mvs, cnt = oracle.find_near_mvs(oracle.mb_info(LAST, (0, 0)), b, b)
    assert cnt[0] == 2 and cnt[1] == 0
    mvs, cnt = oracle.find_near_mvs(b, oracle.mb_info(LAST, (0, 0)), b)
    assert cnt[0] == 2
    v = (16, 8)
    mvs, cnt = oracle.find_near_mvs(oracle.mb_info(LAST, v), oracle.mb_info(LAST, v), b)
    assert cnt[1] == 4 and mvs[1] == v
    va, vl = (16, 0), (0, 16)
    mvs, cnt = oracle.find_near_mvs(oracle.mb_info(LAST, va), oracle.mb_info(LAST, vl), b)
    assert cnt[1] == 2 and cnt[2] == 2 and mvs[1] == va and mvs[2] == vl
    mvs, cnt = oracle.find_near_mvs(oracle.mb_info(LAST, va), oracle.mb_info(LAST, vl), oracle.mb_info(LAST, vl))
    assert cnt[1] == 3 and cnt[2] == 2 and mvs[1] == vl and mvs[2] == va
    s = [(4, 4)] * 16
    mvs, cnt = oracle.find_near_mvs(oracle.mb_info(LAST, (4, 4), True, s), oracle.mb_info(LAST, (8, 8), True, s),
                                    oracle.mb_info(LAST, (12, 12), True, s))
    assert cnt[3] == 5


def test_bool_bits_table(oracle):
    # bool_bits (src/encoder.rs:2229): -log2(p/256) with slot 0 = 8.0; a
    # `true` read at prob 0 indexes min(256, 255) = 255 (the code, not the
    # comment beside it, which calls that slot 8.0).
    assert oracle.bool_bits(128, False) == 1.0 and oracle.bool_bits(128, True) == 1.0
    assert oracle.bool_bits(0, False) == 8.0 and oracle.bool_bits(0, True) == -math.log2(255 / 256.0)
    for p in (1, 7, 100, 255):
        assert oracle.bool_bits(p, False) == -math.log2(p / 256.0)
        assert oracle.bool_bits(p, True) == -math.log2((256 - p) / 256.0)


@pytest.mark.parametrize("value", [0, 1, -1, 7, -7, 8, -8, 15, 16, 100, -517, 1023, -1023])
def test_mv_component_bits_matches_listing(oracle, value):
    # mv_component_bits (src/motion_vector.rs:345), restated in Python.
    p = abi.default_mv_contexts().p[0]
    bb = oracle.bool_bits
    a = abs(value)
    bits = 0.0
    if a > 7:
        bits += bb(p[0], True)
        for i in range(3):
            bits += bb(p[9 + i], (a >> i) & 1)
        for i in range(9, 3, -1):
            bits += bb(p[9 + i], (a >> i) & 1)
        if a & 0xFFF0:
            bits += bb(p[9 + 3], (a >> 3) & 1)
    else:
        bits += bb(p[0], False)
        tree = [2, 8, 4, 6, -0, -1, -2, -3, 10, 12, -4, -5, -6, -7]
        s, i = 0.0, 0
        for k in (2, 1, 0):
            bit = (a >> k) & 1
            s += bb(p[2 + (i >> 1)], bit)
            nxt = tree[i + bit]
            if nxt <= 0:
                break
            i = nxt
        bits += s
    if a:
        bits += bb(p[1], value < 0)
    assert oracle.mv_component_bits(list(p), value) == bits


def test_rd_lambda(oracle):
    # rd_lambda (src/encoder.rs:3742): q^2/32 with q = AC_QLOOKUP[qi].
    assert oracle.rd_lambda(44) == 48.0 * 48.0 / 32.0
    assert oracle.rd_lambda(0) == 16.0 / 32.0
    assert oracle.rd_lambda(127) == 284.0 * 284.0 / 32.0
