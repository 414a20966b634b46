"""Pins the oracle's motion-search restatement against the reference's own
known-answer unit tests (src/motion_search.rs:918-1600), ported case by
case. The six-tap ground truth is built with an independent whole-plane
numpy implementation (vp8a.synth.translate), not with the oracle."""
import numpy as np
import pytest
from util import feature_plane, mb_block, ramp_plane, stepped_plane, two_d_ramp_plane

from vp8a import synth

MV_MIN, MV_MAX = -1023, 1023


def one(o_fn, plane, mb_col, mb_row, src, mv, *extra):
    r = o_fn(plane, np.asarray(src, np.uint8).reshape(1, 256), [[mb_col, mb_row]], [mv], *extra)
    x = r[0]
    return (int(x["mv"]["row"]), int(x["mv"]["col"])), int(x["sad"])


def test_block_sad_kats(oracle):
    a = (np.arange(256) % 251).astype(np.uint8)
    assert oracle.block_sad_16x16(a, a) == 0  # :918
    a = np.full(256, 10, np.uint8)
    b = a.copy()
    b[42] = 11
    assert oracle.block_sad_16x16(a, b) == 1  # :927
    assert oracle.block_sad_16x16(np.zeros(256, np.uint8), np.full(256, 255, np.uint8)) == 256 * 255  # :935
    a = np.zeros(256, np.uint8)
    b = np.zeros(256, np.uint8)
    a[:3] = [10, 20, 30]
    b[:3] = [3, 5, 2]
    assert oracle.block_sad_16x16(a, b) == 50  # block_sad_known_manual_sum :942


def test_sad_at_zero_mv_equals_direct_block_sad(oracle):
    ref = ramp_plane(32, 32)
    src_plane = ref.copy()
    src_plane[0:16, 0:16:4] = (src_plane[0:16, 0:16:4].astype(np.int32) + 5).astype(np.uint8)
    src = mb_block(src_plane, 0, 0)
    expect = oracle.block_sad_16x16(src, mb_block(ref, 0, 0))
    assert oracle.mb_luma_sad_at_mv(ref, src.reshape(1, 256), [[0, 0]], [[0, 0]])[0] == expect


def test_diamond_exact_translation_horizontal(oracle):
    ref = feature_plane(64, 32, 128, 240, 6, 4, 4)
    src = mb_block(feature_plane(64, 32, 128, 240, 4, 4, 4), 0, 0)
    mv, sad = one(oracle.small_diamond_search_luma, ref, 0, 0, src, (0, 0), 32)
    assert mv == (0, 8) and sad == 0  # :995


def test_diamond_exact_translation_diagonal(oracle):
    ref = feature_plane(64, 64, 100, 220, 8, 8, 5)
    src = mb_block(feature_plane(64, 64, 100, 220, 5, 6, 5), 0, 0)
    mv, sad = one(oracle.small_diamond_search_luma, ref, 0, 0, src, (0, 0), 64)
    assert mv == (8, 12) and sad == 0


def test_diamond_zero_iters_and_identity(oracle):
    ref = ramp_plane(32, 32)
    src = mb_block(ref, 0, 0)
    assert one(oracle.small_diamond_search_luma, ref, 0, 0, src, (0, 0), 0) == ((0, 0), 0)
    assert one(oracle.small_diamond_search_luma, ref, 0, 0, src, (0, 0), 8) == ((0, 0), 0)


def test_diamond_snaps_and_clamps_center(oracle):
    flat = np.full((32, 32), 200, np.uint8)
    assert one(oracle.small_diamond_search_luma, flat, 0, 0, np.full(256, 200), (1, 5), 0) == ((0, 4), 0)
    flat = np.full((32, 32), 128, np.uint8)
    (r, c), sad = one(oracle.small_diamond_search_luma, flat, 0, 0, np.full(256, 128), (32767, -32768), 4)
    assert MV_MIN <= r <= MV_MAX and MV_MIN <= c <= MV_MAX and r % 4 == 0 and c % 4 == 0 and sad == 0
    assert (r, c) == (1020, -1020)


def test_diamond_off_picture_edge(oracle):
    ref = ramp_plane(32, 32)
    (r, c), _ = one(oracle.small_diamond_search_luma, ref, 0, 0, mb_block(ref, 0, 0), (-64, -64), 8)
    assert r % 4 == 0 and c % 4 == 0 and MV_MIN <= r <= MV_MAX and MV_MIN <= c <= MV_MAX


def test_diamond_never_increases_sad(oracle):
    ref = feature_plane(48, 48, 90, 230, 6, 6, 5)
    src = mb_block(feature_plane(48, 48, 90, 230, 4, 6, 5), 0, 0)
    center = oracle.mb_luma_sad_at_mv(ref, src.reshape(1, 256), [[0, 0]], [[0, 0]])[0]
    mv, sad = one(oracle.small_diamond_search_luma, ref, 0, 0, src, (0, 0), 8)
    assert sad <= center and mv == (0, 8) and sad == 0


def test_half_pixel_kats(oracle):
    flat = np.full((32, 32), 200, np.uint8)
    assert one(oracle.half_pixel_refine_luma, flat, 0, 0, np.full(256, 200), (0, 0)) == ((0, 0), 0)
    # half_pixel_refine_finds_half_pixel_horizontal_shift (:1243): the
    # source MB(1,1) is the six-tap synthesis at (0, +1/2 px).
    ref = two_d_ramp_plane(64, 64)
    pred = synth.translate(ref, 0, 4)
    src = mb_block(pred, 1, 1)
    assert one(oracle.half_pixel_refine_luma, ref, 1, 1, src, (0, 0)) == ((0, 2), 0)
    # Boundary clamp (:1327).
    flat = np.full((32, 32), 100, np.uint8)
    assert one(oracle.half_pixel_refine_luma, flat, 0, 0, np.full(256, 100), (1020, 1020)) == ((1020, 1020), 0)


def test_half_pixel_never_worsens(oracle):
    ref = ramp_plane(48, 48)
    src_plane = ref.copy().astype(np.int32)
    src_plane[:, 1:-1] = (ref[:, :-2].astype(np.int32) + ref[:, 1:-1]) // 2
    src = mb_block(src_plane.astype(np.uint8), 1, 1)
    center = oracle.mb_luma_sad_at_mv(ref, src.reshape(1, 256), [[1, 1]], [[0, 0]])[0]
    (r, c), sad = one(oracle.half_pixel_refine_luma, ref, 1, 1, src, (0, 0))
    assert sad <= center and abs(r) <= 2 and abs(c) <= 2 and r % 2 == 0 and c % 2 == 0


def test_quarter_pixel_kats(oracle):
    flat = np.full((32, 32), 200, np.uint8)
    assert one(oracle.quarter_pixel_refine_luma, flat, 0, 0, np.full(256, 200), (0, 2)) == ((0, 2), 0)
    # quarter_pixel_refine_finds_quarter_pixel_horizontal_shift (:1446).
    ref = stepped_plane(64, 64)
    src = mb_block(synth.translate(ref, 0, 2), 1, 1)
    half, _ = one(oracle.half_pixel_refine_luma, ref, 1, 1, src, (0, 0))
    assert one(oracle.quarter_pixel_refine_luma, ref, 1, 1, src, half) == ((0, 1), 0)
    flat = np.full((32, 32), 100, np.uint8)
    assert one(oracle.quarter_pixel_refine_luma, flat, 0, 0, np.full(256, 100), (1022, 1022)) == ((1022, 1022), 0)


def test_quarter_at_whole_center_equals_half(oracle):
    # :1582 — on an identical source the quarter refinement at a whole
    # centre keeps the centre with SAD 0.
    ref = ramp_plane(48, 48)
    src = mb_block(ref, 1, 1)
    assert one(oracle.quarter_pixel_refine_luma, ref, 1, 1, src, (0, 0)) == ((0, 0), 0)


@pytest.mark.parametrize("mx,my", [(mx, my) for mx in range(8) for my in range(8)])
def test_sixtap_matches_independent_listing(oracle, mx, my):
    # sixtap_mb_luma_matches_per_subblock_path / sixtap_2d_matches_
    # independent_spec_reference (src/motion_comp.rs:3170, :3330): the
    # MB two-pass equals an independent whole-plane two-pass.
    rng = np.random.default_rng(mx * 8 + my)
    plane = rng.integers(0, 256, (40, 40), dtype=np.uint8)
    halo = plane[8 - 2 : 8 + 19, 8 - 2 : 8 + 19]
    got = oracle.sixtap_mb_luma(halo, mx, my)
    want = synth.translate(plane, my, mx)[8:24, 8:24]
    assert np.array_equal(got, want)
