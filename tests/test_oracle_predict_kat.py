"""Pins the oracle's §18 inter prediction (oracle/predict.c) to the
reference's own known-answer and cross-check tests of src/motion_comp.rs
(tests module, :2387-4560). Each test names the reference test it restates;
the expected values are the ones those tests assert, or an independent
literal transcription of the spec arithmetic (§18.3 interp, Hinterp then
Vinterp over an edge-clamped halo) written here in plain Python, as the
reference's ref_sixtap_2d does.
"""
import numpy as np
import oracle
import pytest

from vp8a import abi


@pytest.fixture(autouse=True, scope="module")
def _oracle_built(request):
    request.getfixturevalue("oracle")  # builds liboracle.so from current sources


SIXTAP = [
    [0, 0, 128, 0, 0, 0],
    [0, -6, 123, 12, -1, 0],
    [2, -11, 108, 36, -8, 1],
    [0, -9, 93, 50, -6, 0],
    [3, -16, 77, 77, -16, 3],
    [0, -6, 50, 93, -9, 0],
    [1, -8, 36, 108, -11, 2],
    [0, -1, 12, 123, -6, 0],
]
BILINEAR = [[0, 0, 128 - 16 * f, 16 * f, 0, 0] for f in range(8)]
SETS = {abi.FILTER_SIXTAP: SIXTAP, abi.FILTER_BILINEAR: BILINEAR}


def spec_interp(fil, p, origin, s):
    """§18.3 interp over a flat buffer: move back two positions, six taps."""
    a = 0
    idx = origin - 2 * s
    for tap in fil:
        a += int(p[idx]) * tap
        idx += s
    return min(max((a + 64) >> 7, 0), 255)


def spec_sixtap_2d(halo, mx, my, taps):
    """Hinterp over the 9 halo rows, Vinterp from the intermediate's row 2."""
    temp = [spec_interp(taps[mx], halo, r * 9 + 2 + c, 1) for r in range(9) for c in range(4)]
    return np.array([[spec_interp(taps[my], temp, (2 + r) * 4 + c, 4) for c in range(4)] for r in range(4)],
                    np.uint8)


def rand_halo(seed, n=81):
    """The reference tests' LCG halo (Knuth's MMIX constants, byte = s >> 33)."""
    s = seed
    out = np.zeros(n, np.uint8)
    for i in range(n):
        s = (s * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        out[i] = (s >> 33) & 0xFF
    return out


def build_reference(mb_cols, mb_rows):
    """build_reference (src/motion_comp.rs tests): y[i] = i % 251,
    u[i] = (3i + 1) % 251, v[i] = (7i + 2) % 251 over MB-padded planes."""
    lw, lh, cw, ch = mb_cols * 16, mb_rows * 16, mb_cols * 8, mb_rows * 8
    y = (np.arange(lw * lh) % 251).astype(np.uint8).reshape(lh, lw)
    u = ((np.arange(cw * ch) * 3 + 1) % 251).astype(np.uint8).reshape(ch, cw)
    v = ((np.arange(cw * ch) * 7 + 2) % 251).astype(np.uint8).reshape(ch, cw)
    return y, u, v


def spec_block(plane, bx, by, mv_eighth, taps):
    """filter_block_4x4 from first principles: the edge-clamped 9x9 halo at
    (bx, by) + (mv >> 3) - 2, then Hinterp/Vinterp (whole fraction: copy)."""
    h, w = plane.shape
    row, col = mv_eighth
    ys = np.clip(by + (row >> 3) - 2 + np.arange(9), 0, h - 1)
    xs = np.clip(bx + (col >> 3) - 2 + np.arange(9), 0, w - 1)
    halo = plane[np.ix_(ys, xs)].reshape(81)
    return spec_sixtap_2d(halo, col & 7, row & 7, taps)


def wrap16(v):
    return ((v + 0x8000) & 0xFFFF) - 0x8000


def spec_split(ref, mb_col, mb_row, mvs16, full_pixel, taps):
    y, u, v = ref
    out_y = np.zeros((16, 16), np.uint8)
    for b, (r, c) in enumerate(mvs16):
        e = (wrap16(2 * r), wrap16(2 * c))
        if full_pixel:
            e = (e[0] & ~7, e[1] & ~7)
        sb, sc = divmod(b, 4)
        out_y[4 * sb:4 * sb + 4, 4 * sc:4 * sc + 4] = spec_block(y, mb_col * 16 + 4 * sc, mb_row * 16 + 4 * sb, e, taps)
    sums = np.zeros((4, 2), np.int64)
    for b, (r, c) in enumerate(mvs16):
        k = ((b >> 1) & 1) + ((b >> 2) & 2)
        sums[k] += (2 * r, 2 * c)
    avg = lambda s: (s + 4) >> 3 if s >= 0 else -((-s + 4) >> 3)  # noqa: E731
    outs = []
    for plane in (u, v):
        o = np.zeros((8, 8), np.uint8)
        for k in range(4):
            e = (wrap16(avg(int(sums[k][0]))), wrap16(avg(int(sums[k][1]))))
            if full_pixel:
                e = (e[0] & ~7, e[1] & ~7)
            sb, sc = divmod(k, 2)
            o[4 * sb:4 * sb + 4, 4 * sc:4 * sc + 4] = spec_block(plane, mb_col * 8 + 4 * sc, mb_row * 8 + 4 * sb, e,
                                                                 taps)
        outs.append(o)
    return np.concatenate([out_y.reshape(-1), outs[0].reshape(-1), outs[1].reshape(-1)])


def test_chroma_mv_of_repeated_vector_is_quarter():
    # chroma_mv_of_repeated_vector_is_quarter (:2572): stored (3,-5) = (6,-10) -> (3,-5).
    assert oracle.chroma_mv(6, -10) == (3, -5)


def test_chroma_mv_matches_reference_closed_form():
    # chroma_mv_matches_reference_closed_form (:2583): (c + 1 + (c >> 31) * 2) / 2, truncating.
    def ref_form(c):
        n = c + 1 + (-1 if c < 0 else 0) * 2
        return -((-n) // 2) if n < 0 else n // 2

    for c in [0, 2, 6, 10, 14, 100, -2, -6, -10, -14, -100, 2046, -2046]:
        assert oracle.chroma_mv(c, c) == (ref_form(c), ref_form(c)), c


def test_interp_matches_spec_formula():
    # interp_matches_spec_formula (:3077), through sixtap_2d with a vertical
    # identity: block sample (0, 0) is interp over halo row 2, columns 0..5.
    def first(support, mx):
        halo = np.zeros((9, 9), np.uint8)
        halo[2, :6] = support
        return int(oracle.sixtap_2d(halo, mx, 0)[0, 0])

    support = [10, 20, 30, 40, 50, 60]
    assert first(support, 0) == 30
    assert first(support, 4) == 35
    for mx in range(8):
        assert first([200] * 6, mx) == 200
    assert first([0, 255, 0, 0, 255, 0], 2) == 0


@pytest.mark.parametrize("fs", [abi.FILTER_SIXTAP, abi.FILTER_BILINEAR])
def test_sixtap_2d_matches_independent_spec_reference(fs):
    # sixtap_2d_matches_independent_spec_reference (:3170).
    for seed in range(3):
        halo = rand_halo(seed * 977 + 13)
        for mx in range(8):
            for my in range(8):
                got = oracle.sixtap_2d(halo, mx, my, fs)
                assert np.array_equal(got, spec_sixtap_2d(halo, mx, my, SETS[fs])), (seed, mx, my)


def test_sixtap_2d_flat_halo_passes_dc_and_whole_fraction_copies():
    # sixtap_2d_flat_halo_passes_dc (:3189), sixtap_2d_whole_fraction_copies_block (:3204).
    flat = np.full(81, 137, np.uint8)
    for fs in SETS:
        for mx in range(8):
            for my in range(8):
                assert (oracle.sixtap_2d(flat, mx, my, fs) == 137).all()
    halo = rand_halo(42)
    assert np.array_equal(oracle.sixtap_2d(halo, 0, 0), halo.reshape(9, 9)[2:6, 2:6])


def test_sixtap_2d_horizontal_only_known_values():
    # sixtap_2d_horizontal_only_known_values (:3218): ramp halo, mx = 2, my = 0.
    halo = np.tile((np.arange(9) * 20).astype(np.uint8), 9)
    out = oracle.sixtap_2d(halo, 2, 0)
    for r in range(4):
        for c in range(4):
            assert out[r, c] == spec_interp(SIXTAP[2], halo, r * 9 + 2 + c, 1)


def test_predict_zero_mv_copies_corresponding_mb():
    # predict_zero_mv_copies_corresponding_mb (:2728).
    y, u, v = build_reference(2, 2)
    out = oracle.predict_inter_mb((y, u, v), [(1, 1)], [(0, 0)])[0]
    assert np.array_equal(out[:256].reshape(16, 16), y[16:32, 16:32])
    assert np.array_equal(out[256:320].reshape(8, 8), u[8:16, 8:16])
    assert np.array_equal(out[320:].reshape(8, 8), v[8:16, 8:16])


def test_predict_whole_pixel_offset_shifts_source():
    # predict_whole_pixel_offset_shifts_source (:2763): luma (8, 16) ->
    # offsets (2, 4) luma and (1, 2) chroma, pure copies.
    y, u, v = build_reference(3, 3)
    out = oracle.predict_inter_mb((y, u, v), [(1, 1)], [(8, 16)])[0]
    assert np.array_equal(out[:256].reshape(16, 16), y[18:34, 20:36])
    assert np.array_equal(out[256:320].reshape(8, 8), u[9:17, 10:18])
    assert np.array_equal(out[320:].reshape(8, 8), v[9:17, 10:18])


def test_predict_full_pixel_version_truncates_to_whole():
    # predict_full_pixel_version_truncates_to_whole (:2851): luma (4, 0) ->
    # (8, 0) eighth-pel, chroma 4 -> 0 under full_pixel.
    y, u, v = build_reference(2, 2)
    out = oracle.predict_inter_mb((y, u, v), [(0, 0)], [(4, 0)], full_pixel=True)[0]
    assert np.array_equal(out[:256].reshape(16, 16), y[1:17, 0:16])
    assert np.array_equal(out[256:320].reshape(8, 8), u[0:8, 0:8])


@pytest.mark.parametrize("mb", [(1, 1), (0, 0)])
def test_predict_inter_mb_sub_pixel_matches_per_block(mb):
    # predict_inter_mb_sub_pixel_matches_per_block (:3950) in-bounds and
    # predict_inter_mb_sub_pixel_at_border_uses_mb_halo_clamp (:3585) at the
    # corner: the MB-scale listing equals independent per-4x4 blocks.
    ref = build_reference(3, 3)
    got = oracle.predict_inter_mb(ref, [mb], [(3, 5)])[0]
    want = spec_split(ref, mb[0], mb[1], [(3, 5)] * 16, False, SIXTAP)
    assert np.array_equal(got, want)


def test_predict_inter_mb_uses_selected_filter_set():
    # predict_inter_mb_uses_selected_filter_set (:4042).
    ref = build_reference(3, 3)
    six = oracle.predict_inter_mb(ref, [(1, 1)], [(3, 5)], filter_set=abi.FILTER_SIXTAP)[0]
    bil = oracle.predict_inter_mb(ref, [(1, 1)], [(3, 5)], filter_set=abi.FILTER_BILINEAR)[0]
    assert not np.array_equal(six[:256], bil[:256])
    assert np.array_equal(bil, spec_split(ref, 1, 1, [(3, 5)] * 16, False, BILINEAR))


@pytest.mark.parametrize("full_pixel", [False, True])
@pytest.mark.parametrize("mb", [(1, 1), (0, 0)])
def test_predict_split_mv_matches_per_block_spec(full_pixel, mb):
    # strided_into_assembly_matches_predict_split_mv (:4470): sixteen distinct
    # vectors mixing whole- and sub-pel fractions, mid-grid and corner MB,
    # both full_pixel polarities.
    mvs = []
    for i in range(16):
        fr = 0 if i % 2 == 0 else (i % 7) + 1
        fc = 0 if i % 3 == 0 else (i % 5) + 1
        mvs.append(((i % 3 - 1) * 8 + fr, (i % 4 - 2) * 8 + fc))
    ref = build_reference(3, 3)
    got = oracle.predict_split_mv(ref, [mb], mvs, full_pixel=full_pixel)[0]
    assert np.array_equal(got, spec_split(ref, mb[0], mb[1], mvs, full_pixel, SIXTAP))


def test_split_chroma_mvs_average_doubled_quadrants():
    # split_chroma_mvs (:2175): chroma block k averages luma blocks with
    # chroma_idx_for_luma_subblock(b) = ((b >> 1) & 1) + ((b >> 2) & 2) == k.
    rng = np.random.default_rng(3)
    mvs = rng.integers(-1023, 1024, (16, 2))
    got = oracle.split_chroma_mvs(mvs)
    for k in range(4):
        blocks = [b for b in range(16) if ((b >> 1) & 1) + ((b >> 2) & 2) == k]
        for comp in range(2):
            s = int(sum(2 * mvs[b][comp] for b in blocks))
            want = (s + 4) >> 3 if s >= 0 else -((-s + 4) >> 3)
            assert got[k][comp] == want
    # Equal vectors: the split average equals chroma_mv of the doubled one.
    same = np.tile([[3, -5]], (16, 1))
    assert [tuple(r) for r in oracle.split_chroma_mvs(same)] == [oracle.chroma_mv(6, -10)] * 4


def test_predict_inter_frame_routes_split_whole_and_intra():
    # The encoder's per-MB prediction (src/encoder.rs:8704-8735): SPLIT
    # decisions take predict_split_mv, the rest predict_inter_mb from their
    # own reference; intra MBs keep the output's pixels.
    refs = [build_reference(2, 2), tuple(255 - p for p in build_reference(2, 2))]
    dec = np.zeros(4, abi.MB_DECISION_DTYPE)
    dec["ref_frame"] = [abi.REF_LAST, abi.REF_GOLDEN, abi.REF_INTRA, abi.REF_LAST]
    dec["mode"] = [abi.MODE_NEW, abi.MODE_SPLIT, abi.MODE_NONE, abi.MODE_ZERO]
    dec["mv"][0] = (3, -5)
    rng = np.random.default_rng(7)
    sm = rng.integers(-40, 40, (16, 2))
    dec["split_mvs"][1]["row"], dec["split_mvs"][1]["col"] = sm[:, 0], sm[:, 1]
    out = tuple(np.full(p.shape, 77, np.uint8) for p in refs[0])
    assert oracle.predict_inter_frame(refs, [abi.REF_LAST, abi.REF_GOLDEN], dec, out) == 1

    def mb_of(planes, col, row):
        y, u, v = planes
        return np.concatenate([y[16 * row:16 * row + 16, 16 * col:16 * col + 16].reshape(-1),
                               u[8 * row:8 * row + 8, 8 * col:8 * col + 8].reshape(-1),
                               v[8 * row:8 * row + 8, 8 * col:8 * col + 8].reshape(-1)])

    assert np.array_equal(mb_of(out, 0, 0), oracle.predict_inter_mb(refs[0], [(0, 0)], [(3, -5)])[0])
    assert np.array_equal(mb_of(out, 1, 0), oracle.predict_split_mv(refs[1], [(1, 0)], dec["split_mvs"][1])[0])
    assert (mb_of(out, 0, 1) == 77).all()
    assert np.array_equal(mb_of(out, 1, 1), mb_of(refs[0], 1, 1))
