"""Pins the oracle's §14 inter reconstruction (oracle/recon.c, trellis off)
to the reference's own tests: the transform known answers of
src/forward_transform.rs (tests, :800-1000) and src/inverse_transform.rs
(tests, :900-1400), the dequantisation-factor tests of src/dequant.rs
(tests, :411-700), and, for the per-MB chain of pick_mb_for_ref
(src/encoder.rs:8704-8800), an independent plain-Python transliteration of
the listed steps run on seeded MBs. Each test names the reference test or
function it restates.
"""
import numpy as np
import oracle
import pytest

from vp8a import abi


@pytest.fixture(autouse=True, scope="module")
def _oracle_built(request):
    request.getfixturevalue("oracle")  # builds liboracle.so from current sources


DC_Q = [4, 5, 6, 7, 8, 9, 10, 10, 11, 12, 13, 14, 15, 16, 17, 17, 18, 19, 20, 20, 21, 21, 22, 22, 23, 23, 24, 25, 25,
        26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 46, 47, 48, 49, 50,
        51, 52, 53, 54, 55, 56, 57, 58, 59, 60, 61, 62, 63, 64, 65, 66, 67, 68, 69, 70, 71, 72, 73, 74, 75, 76, 76,
        77, 78, 79, 80, 81, 82, 83, 84, 85, 86, 87, 88, 89, 91, 93, 95, 96, 98, 100, 101, 102, 104, 106, 108, 110,
        112, 114, 116, 118, 122, 124, 126, 128, 130, 132, 134, 136, 138, 140, 143, 145, 148, 151, 154, 157]
AC_Q = [4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32,
        33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51, 52, 53, 54, 55, 56, 57, 58, 60,
        62, 64, 66, 68, 70, 72, 74, 76, 78, 80, 82, 84, 86, 88, 90, 92, 94, 96, 98, 100, 102, 104, 106, 108, 110,
        112, 114, 116, 119, 122, 125, 128, 131, 134, 137, 140, 143, 146, 149, 152, 155, 158, 161, 164, 167, 170,
        173, 177, 181, 185, 189, 193, 197, 201, 205, 209, 213, 217, 221, 225, 229, 234, 239, 245, 249, 254, 259,
        264, 269, 274, 279, 284]
C8, S8 = 20091, 35468


# ---- independent transliterations (plain Python ints) ---------------------

def wrap32(v):
    return ((v + (1 << 31)) & 0xFFFFFFFF) - (1 << 31)


def idct(inp):
    """§14.4 inverse DCT with the reference's wrapping i32 arithmetic."""
    tmp = [0] * 16
    for col in range(4):
        i0, i4, i8, i12 = inp[col], inp[4 + col], inp[8 + col], inp[12 + col]
        a1, b1 = wrap32(i0 + i8), wrap32(i0 - i8)
        c1 = wrap32((wrap32(i4 * S8) >> 16) - wrap32(i12 + (wrap32(i12 * C8) >> 16)))
        d1 = wrap32(wrap32(i4 + (wrap32(i4 * C8) >> 16)) + (wrap32(i12 * S8) >> 16))
        tmp[col], tmp[12 + col] = wrap32(a1 + d1), wrap32(a1 - d1)
        tmp[4 + col], tmp[8 + col] = wrap32(b1 + c1), wrap32(b1 - c1)
    out = [0] * 16
    for row in range(4):
        r0, r1, r2, r3 = tmp[4 * row:4 * row + 4]
        a1, b1 = wrap32(r0 + r2), wrap32(r0 - r2)
        c1 = wrap32((wrap32(r1 * S8) >> 16) - wrap32(r3 + (wrap32(r3 * C8) >> 16)))
        d1 = wrap32(wrap32(r1 + (wrap32(r1 * C8) >> 16)) + (wrap32(r3 * S8) >> 16))
        for k, v in ((0, a1 + d1), (3, a1 - d1), (1, b1 + c1), (2, b1 - c1)):
            out[4 * row + k] = ((wrap32(wrap32(v) + 4) >> 3) + 32768) % 65536 - 32768
    return out


def iwht(inp):
    tmp = [0] * 16
    for col in range(4):
        i0, i4, i8, i12 = inp[col], inp[4 + col], inp[8 + col], inp[12 + col]
        a1, b1, c1, d1 = i0 + i12, i4 + i8, i4 - i8, i0 - i12
        tmp[col], tmp[4 + col], tmp[8 + col], tmp[12 + col] = a1 + b1, c1 + d1, a1 - b1, d1 - c1
    out = [0] * 16
    for row in range(4):
        r0, r1, r2, r3 = tmp[4 * row:4 * row + 4]
        a1, b1, c1, d1 = r0 + r3, r1 + r2, r1 - r2, r0 - r3
        for k, v in enumerate((a1 + b1, c1 + d1, a1 - b1, d1 - c1)):
            out[4 * row + k] = (v + 3) >> 3
    return out


def rdiv2(v):
    r = (v + 1) >> 1 if v >= 0 else -((-v + 1) >> 1)
    return max(-32768, min(32767, r))


def cm(i):
    return i + ((i * C8) >> 16)


def sm(i):
    return (i * S8) >> 16


def fdct(inp):
    tmp = [0] * 16
    for col in range(4):
        i0, i4, i8, i12 = inp[col], inp[4 + col], inp[8 + col], inp[12 + col]
        tmp[col] = (i0 + i12) + (i4 + i8)
        tmp[4 + col] = (cm(i0) - cm(i12)) + (sm(i4) - sm(i8))
        tmp[8 + col] = (i0 + i12) - (i4 + i8)
        tmp[12 + col] = (sm(i0) - sm(i12)) - (cm(i4) - cm(i8))
    out = [0] * 16
    for row in range(4):
        r0, r1, r2, r3 = tmp[4 * row:4 * row + 4]
        out[4 * row] = rdiv2((r0 + r3) + (r1 + r2))
        out[4 * row + 1] = rdiv2((cm(r0) - cm(r3)) + (sm(r1) - sm(r2)))
        out[4 * row + 2] = rdiv2((r0 + r3) - (r1 + r2))
        out[4 * row + 3] = rdiv2((sm(r0) - sm(r3)) - (cm(r1) - cm(r2)))
    return out


def fwht(inp):
    tmp = [0] * 16
    for col in range(4):
        i0, i4, i8, i12 = inp[col], inp[4 + col], inp[8 + col], inp[12 + col]
        a1, b1, c1, d1 = i0 + i12, i4 + i8, i4 - i8, i0 - i12
        tmp[col], tmp[4 + col], tmp[8 + col], tmp[12 + col] = a1 + b1, c1 + d1, a1 - b1, d1 - c1
    out = [0] * 16
    for row in range(4):
        r0, r1, r2, r3 = tmp[4 * row:4 * row + 4]
        a1, b1, c1, d1 = r0 + r3, r1 + r2, r1 - r2, r0 - r3
        for k, v in enumerate((a1 + b1, c1 + d1, a1 - b1, d1 - c1)):
            out[4 * row + k] = rdiv2(v)
    return out


def rdiv(num, den):
    r = (num + den // 2) // den if num >= 0 else -(((-num) + den // 2) // den)
    return (r + 32768) % 65536 - 32768


def to16(v):
    return (v + 32768) % 65536 - 32768


def spec_mb(src, pred, f, split):
    """pick_mb_for_ref's transform -> skip -> dequantise -> reconstruct."""
    y1dc, y1ac, y2dc, y2ac, uvdc, uvac = f
    src, pred = [int(x) for x in src], [int(x) for x in pred]

    def res(n, base, bi, bj):
        return [src[base + (bi * 4 + r) * n + bj * 4 + c] - pred[base + (bi * 4 + r) * n + bj * 4 + c]
                for r in range(4) for c in range(4)]

    y = [fdct(res(16, 0, i, j)) for i in range(4) for j in range(4)]
    y2 = [0] * 16
    if not split:
        y2 = fwht([b[0] for b in y])
        for b in y:
            b[0] = 0
        y2 = [rdiv(y2[0], y2dc)] + [rdiv(c, y2ac) for c in y2[1:]]
    y = [[rdiv(b[0], y1dc)] + [rdiv(c, y1ac) for c in b[1:]] for b in y]
    uv = [[fdct(res(8, 256 + 64 * p, i, j)) for i in range(2) for j in range(2)] for p in range(2)]
    uv = [[[rdiv(b[0], uvdc)] + [rdiv(c, uvac) for c in b[1:]] for b in pl] for pl in uv]
    nz = (0 if split else sum(c != 0 for c in y2)) + sum(c != 0 for b in y for c in b[(0 if split else 1):])
    nz += sum(c != 0 for pl in uv for b in pl for c in b)
    skip = nz == 0
    dy2 = [to16(y2[0] * y2dc)] + [to16(c * y2ac) for c in y2[1:]]
    dy = [[to16(b[0] * y1dc)] + [to16(c * y1ac) for c in b[1:]] for b in y]
    duv = [[[to16(b[0] * uvdc)] + [to16(c * uvac) for c in b[1:]] for b in pl] for pl in uv]
    has = any(c for c in dy2) or any(c for b in dy for c in b) or any(c for pl in duv for b in pl for c in b)
    rec = list(pred)
    if not skip:
        if not split:
            dcs = iwht(dy2)
            for k in range(16):
                dy[k][0] = dcs[k]

        def add(blk, n, base, bi, bj):
            r16 = idct(blk)
            for r in range(4):
                for c in range(4):
                    o = base + (bi * 4 + r) * n + bj * 4 + c
                    rec[o] = max(0, min(255, rec[o] + r16[r * 4 + c]))

        for i in range(4):
            for j in range(4):
                add(dy[i * 4 + j], 16, 0, i, j)
        for p in range(2):
            for i in range(2):
                for j in range(2):
                    add(duv[p][i * 2 + j], 8, 256 + 64 * p, i, j)
    coeffs = y2 + [c for b in y for c in b] + [c for pl in uv for b in pl for c in b]
    return np.array(rec, np.uint8), np.array(coeffs, np.int16), int(skip) | (int(has) << 1)


# ---- the reference's known answers ------------------------------------------

def test_uniform_blocks_concentrate_to_dc_and_roundtrip():
    # fwht/fdct_uniform_block_concentrates_to_dc, fwht_iwht / fdct_idct
    # roundtrip_uniform_block, forward_transforms_of_zero_are_zero.
    for v in [1, 2, 5, 8, 16, 64, 100]:
        for fn in (oracle.forward_wht_4x4, oracle.forward_dct_4x4):
            out = fn([v] * 16)
            assert out[0] == 8 * v and not out[1:].any()
    for v in [0, 1, 2, 3, 5, 8, 16, 32, 64, 100]:
        assert (oracle.inverse_wht_4x4(oracle.forward_wht_4x4([v] * 16)) == v).all()
        assert (oracle.inverse_dct_4x4(oracle.forward_dct_4x4([v] * 16)) == v).all()
    assert not oracle.forward_dct_4x4([0] * 16).any() and not oracle.forward_wht_4x4([0] * 16).any()


def test_fdct_gradient_and_random_roundtrip_error_bounds():
    # fdct_idct_roundtrip_gradient_block, fdct_idct_random_small_inputs_have_bounded_error.
    grad = [r * 8 for r in range(4) for _ in range(4)]
    c = oracle.forward_dct_4x4(grad)
    assert c[4] != 0 and c[1] == 0
    assert (np.abs(oracle.inverse_dct_4x4(c) - np.array(grad)) <= 1).all()
    state = 0xDEADBEEF
    for _ in range(32):
        block = []
        for _ in range(16):
            state = (state * 1103515245 + 12345) & 0xFFFFFFFF
            r = state >> 16
            block.append(r % 129 - 64)
        back = oracle.inverse_dct_4x4(oracle.forward_dct_4x4(block))
        assert (np.abs(back - np.array(block)) <= 2).all()


def test_inverse_transform_known_answers():
    # dct_dc_only_is_uniform_block, dct_dc_rounding_with_larger_value,
    # wht_hand_derived_two_value_input, dct_first_ac_coefficient_uses_cosine_constants.
    b = [0] * 16
    b[0] = 8
    assert (oracle.inverse_dct_4x4(b) == 1).all()
    b[0] = 64
    assert (oracle.inverse_dct_4x4(b) == 8).all()
    w = [0] * 16
    w[0], w[4] = 8, 8
    assert oracle.inverse_wht_4x4(w).tolist() == [2] * 8 + [0] * 8
    a = [0] * 16
    a[1] = 100
    got = oracle.inverse_dct_4x4(a)
    assert got.tolist() == idct(a) and len(set(got.tolist())) > 1


def test_idct_extreme_coefficients_wrap():
    # dct_extreme_coefficients_wrap_without_panic: the i32 intermediates wrap.
    rng = np.random.default_rng(2)
    cases = [[32767] * 16, [-32768] * 16, [32767 if k % 2 else -32768 for k in range(16)]]
    cases += [rng.integers(-32768, 32768, 16).tolist() for _ in range(50)]
    for blk in cases:
        assert oracle.inverse_dct_4x4(blk).tolist() == idct(blk)


def test_transforms_match_transliteration_on_random_blocks():
    rng = np.random.default_rng(3)
    for _ in range(300):
        res = rng.integers(-255, 256, 16).tolist()
        assert oracle.forward_dct_4x4(res).tolist() == fdct(res)
        assert oracle.forward_wht_4x4(res).tolist() == fwht(res)
        big = rng.integers(-4000, 4000, 16).tolist()
        assert oracle.inverse_wht_4x4(big).tolist() == iwht(big)


def test_enc_quantize_rounds_half_away_from_zero():
    # enc_round_div / enc_quantize_block (src/encoder.rs:2112-2132).
    got = oracle.enc_quantize_block([10, -10, 7, -7, 2, 3, -3, 0, 5, -5, 12, -12, 1, -1, 250, -250], 4, 5)
    assert got.tolist() == [3, -2, 1, -1, 0, 1, -1, 0, 1, -1, 2, -2, 0, 0, 50, -50]


def test_dequant_factor_known_answers():
    # src/dequant.rs tests: y1 lookups, y2 dc doubled, y2 ac 155/100 floored
    # at 8 and truncating, uv dc capped at 132, uv ac delta, clamps.
    f = oracle.dequant_factors(40, 3)
    assert f[0] == DC_Q[43] and f[1] == AC_Q[40]
    assert oracle.dequant_factors(30)[2] == DC_Q[30] * 2
    assert oracle.dequant_factors(30, 0, 5)[2] == DC_Q[35] * 2
    assert oracle.dequant_factors(60)[3] == 108
    assert oracle.dequant_factors(0)[3] == 8
    assert oracle.dequant_factors(5)[3] == 13
    assert oracle.dequant_factors(117)[4] == 132 and oracle.dequant_factors(120)[4] == 132
    assert oracle.dequant_factors(50)[4] == DC_Q[50]
    assert oracle.dequant_factors(50, 0, 0, 0, 0, -4)[5] == AC_Q[46]
    assert oracle.dequant_factors(10, -20)[0] == DC_Q[0]
    assert oracle.dequant_factors(200)[1] == AC_Q[127]
    hi = oracle.dequant_factors(2**31 - 1, 1, 1, 1, 1, 1)
    lo = oracle.dequant_factors(-2**31, -1, -1, -1, -1, -1)
    assert hi[:2] == (DC_Q[127], AC_Q[127]) and lo[:2] == (DC_Q[0], AC_Q[0])


def test_segment_factors():
    # segment_delta_mode_adds_to_baseline, segment_absolute_mode_replaces_baseline,
    # segment_keeps_perplane_deltas, extreme segment saturation.
    qi = abi.quant_indices(40)
    assert oracle.segment_factors(qi, 10)[1] == AC_Q[50]
    assert oracle.segment_factors(qi, -15)[1] == AC_Q[25]
    assert oracle.segment_factors(qi, 70, absolute=True)[1] == AC_Q[70]
    qd = abi.quant_indices(40, uv_ac=-4)
    assert oracle.segment_factors(qd, 10)[5] == AC_Q[46]
    assert oracle.segment_factors(abi.quant_indices(200), 2**31 - 1)[1] == AC_Q[127]
    assert oracle.segment_factors(qi) == oracle.dequant_factors(40)


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("qi", [0, 10, 44, 90, 127])
def test_reconstruct_mb_matches_transliteration(split, qi):
    rng = np.random.default_rng(qi * 2 + split)
    f = oracle.dequant_factors(qi)
    for k in range(6):
        pred = rng.integers(0, 256, 384).astype(np.uint8)
        spread = [2, 8, 40, 255, 0, 4][k]
        src = np.clip(pred.astype(int) + rng.integers(-spread, spread + 1, 384), 0, 255).astype(np.uint8)
        rec, cf, fl = oracle.reconstruct_inter_mb(src, pred, f, split)
        want_rec, want_cf, want_fl = spec_mb(src, pred, f, split)
        assert np.array_equal(cf, want_cf)
        assert fl == want_fl
        assert np.array_equal(rec, want_rec)
        if spread == 0:
            assert fl == abi.MB_SKIP and np.array_equal(rec, pred)


def test_reconstruct_adds_dc_residue():
    # reconstruct_adds_dc_residue (src/motion_comp.rs tests): a uniform luma
    # offset quantises to a pure Y2 DC; the reconstruction is the prediction
    # plus one constant on luma and the prediction on chroma.
    pred = np.full(384, 100, np.uint8)
    src = pred.copy()
    src[:256] = 140
    f = oracle.dequant_factors(20)
    rec, cf, fl = oracle.reconstruct_inter_mb(src, pred, f, False)
    assert cf[0] != 0 and not cf[1:].any()
    assert len(set(rec[:256].tolist())) == 1 and rec[0] != 100
    assert (rec[256:] == 100).all()
    assert fl == abi.MB_HAS_COEFFS
