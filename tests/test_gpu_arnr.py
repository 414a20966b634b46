"""Parity: the ARNR kernels (build_arnr_altref through the C ABI) produce
the oracle's anchor picture byte for byte."""
import numpy as np
import pytest

import vp8a
from vp8a import synth

pytestmark = pytest.mark.gpu


def same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.fixture(scope="module")
def seq7():
    frames, _ = synth.make_sequence(320, 240, 7, seed=21)
    return frames


@pytest.mark.parametrize("center", [3, 6, 0])
@pytest.mark.parametrize("strength", [0, 1, 3, 6])
def test_arnr_config1(ctx, oracle, seq7, center, strength):
    assert same(vp8a.build_arnr_altref(ctx, seq7, center, strength),
                oracle.build_arnr_altref(seq7, center, strength))


@pytest.mark.parametrize("w,h", [(17, 9), (47, 33), (64, 48), (100, 18)])
def test_arnr_odd_sizes_and_strides(ctx, oracle, w, h):
    frames, _ = synth.make_sequence(w, h, 5, seed=w + h)
    # Give the planes a row pitch wider than the width.
    padded = []
    for y, u, v in frames:
        Y = np.zeros((h, w + 5), np.uint8)
        Y[:, :w] = y
        U = np.zeros(u.shape[:1] + (u.shape[1] + 3,), np.uint8)
        U[:, : u.shape[1]] = u
        V = np.zeros_like(U)
        V[:, : v.shape[1]] = v
        padded.append((Y[:, :w], U[:, : u.shape[1]], V[:, : v.shape[1]]))
    for center in (0, 2, 4):
        assert same(vp8a.build_arnr_altref(ctx, padded, center, 3), oracle.build_arnr_altref(padded, center, 3))


def test_arnr_scene_change_and_identity(ctx):
    r, c = np.mgrid[0:48, 0:48]
    y = (64 + ((r * 3 + c * 2) & 0x7F)).astype(np.uint8)
    u = np.full((24, 24), 120, np.uint8)
    v = np.full((24, 24), 136, np.uint8)
    out = vp8a.build_arnr_altref(ctx, [(y, u, v), (255 - y, u, v)], 0, 6)
    assert np.array_equal(out[0], y)
    out = vp8a.build_arnr_altref(ctx, [(y, u, v)], 0, 3)
    assert same(out, (y, u, v))


def test_arnr_errors(ctx):
    y = np.zeros((32, 32), np.uint8)
    c = np.zeros((16, 16), np.uint8)
    small = (np.zeros((16, 16), np.uint8), np.zeros((8, 8), np.uint8), np.zeros((8, 8), np.uint8))
    with pytest.raises(vp8a.Vp8aError, match="ReferenceDimensionsMismatch"):
        vp8a.build_arnr_altref(ctx, [(y, c, c), small], 0, 3)
    with pytest.raises(vp8a.Vp8aError, match="InvalidArgument"):
        vp8a.build_arnr_altref(ctx, [(y, c, c)], 1, 3)


def test_arnr_1080p_lookahead7(ctx, oracle):
    frames, _ = synth.make_sequence(1920, 1080, 7, seed=5)
    assert same(vp8a.build_arnr_altref(ctx, frames, 3, 3), oracle.build_arnr_altref(frames, 3, 3, threads=8))


@pytest.mark.parametrize("w,h", [(320, 240), (17, 9), (47, 33), (100, 18), (1920, 1080)])
def test_arnr_into_mb_padded_planes(ctx, oracle, w, h):
    # vp8a_build_arnr_altref_planes: the oracle's anchor, edge-replicated
    # into the MB-padded layout of a reference (pad_to_mb), written by the
    # blend kernel itself; planes with a row pitch wider than the padded
    # width keep their extra bytes.
    frames, _ = synth.make_sequence(w, h, 5, seed=w * 7 + h)
    want = vp8a.pad_to_mb(*oracle.build_arnr_altref(frames, 2, 3, threads=8))
    got = vp8a.build_arnr_altref_planes(ctx, frames, 2, 3)
    assert same(got, want)
    wide = [np.full((p.shape[0], p.shape[1] + 12), 7, np.uint8) for p in want]
    vp8a.build_arnr_altref_planes(ctx, frames, 2, 3, out=[x[:, : p.shape[1]] for x, p in zip(wide, want)])
    assert same([x[:, : p.shape[1]] for x, p in zip(wide, want)], want)
    assert all((x[:, p.shape[1]:] == 7).all() for x, p in zip(wide, want))


def test_arnr_batched_into_mb_padded_planes(ctx, oracle):
    jobs = []
    for i, (w, h) in enumerate([(176, 144), (64, 48), (47, 33)]):
        frames, _ = synth.make_sequence(w, h, 5, seed=90 + i)
        jobs.append((frames, 2 if i != 1 else 4, 3))
    got = vp8a.build_arnr_altrefs_planes(ctx, jobs)
    for (frames, center, strength), g in zip(jobs, got):
        assert same(g, vp8a.pad_to_mb(*oracle.build_arnr_altref(frames, center, strength)))


def test_arnr_planes_grid_mismatch(ctx):
    frames, _ = synth.make_sequence(64, 48, 3, seed=4)
    bad = (np.zeros((64, 64), np.uint8), np.zeros((32, 32), np.uint8), np.zeros((32, 32), np.uint8))
    with pytest.raises(vp8a.Vp8aError, match="ReferenceDimensionsMismatch"):
        vp8a.build_arnr_altref_planes(ctx, frames, 1, 3, out=bad)
