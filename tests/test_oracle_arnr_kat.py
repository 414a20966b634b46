"""Pins the oracle's ARNR restatement against the reference's unit tests
(src/arnr.rs:677-1136): identity cases, denoising, motion tracking,
scene-change exclusion, dimension errors and the weight table."""
import numpy as np
import pytest

W = H = 48


class Lcg:
    """The reference test LCG (src/arnr.rs tests)."""

    def __init__(self, seed):
        self.s = seed & (2**64 - 1)

    def next(self):
        self.s = (self.s * 6364136223846793005 + 1) & (2**64 - 1)
        return self.s >> 33

    def noise(self, amp):
        return int(self.next() % (2 * amp + 1)) - amp


def clean_scene():
    r, c = np.mgrid[0:H, 0:W]
    y = (64 + ((r * 3 + c * 2) & 0x7F)).astype(np.uint8)
    return y, np.full((H // 2, W // 2), 120, np.uint8), np.full((H // 2, W // 2), 136, np.uint8)


def noisy(plane, seed, amp):
    rng = Lcg(seed)
    flat = plane.reshape(-1)
    out = np.array([min(max(int(p) + rng.noise(amp), 0), 255) for p in flat], np.uint8)
    return out.reshape(plane.shape)


def mse(a, b):
    return float(((a.astype(np.int64) - b.astype(np.int64)) ** 2).mean())


def test_strength_zero_and_single_frame_identity(oracle):
    y, u, v = clean_scene()
    out = oracle.build_arnr_altref([(y, u, v)], 0, 3)
    assert all(np.array_equal(a, b) for a, b in zip(out, (y, u, v)))
    ny = noisy(y, 7, 6)
    out = oracle.build_arnr_altref([(ny, u, v), (y, u, v)], 0, 0)
    assert np.array_equal(out[0], ny)


def test_static_noisy_window_denoises(oracle):
    cy, cu, cv = clean_scene()
    planes = [noisy(cy, 1000 + i, 6) for i in range(5)]
    out = oracle.build_arnr_altref([(p, cu, cv) for p in planes], 2, 3)
    assert mse(out[0], cy) < mse(planes[2], cy) / 2.0


def test_motion_compensation_tracks_translation(oracle):
    cy, cu, cv = clean_scene()
    planes = []
    for i in range(3):
        dx = (i - 1) * 4
        sc = np.clip(np.arange(W) - dx, 0, W - 1)
        planes.append(noisy(cy[:, sc], 2000 + i, 6))
    out = oracle.build_arnr_altref([(p, cu, cv) for p in planes], 1, 3)
    assert mse(out[0], cy) < mse(planes[1], cy)


def test_scene_change_neighbour_excluded(oracle):
    cy, cu, cv = clean_scene()
    out = oracle.build_arnr_altref([(cy, cu, cv), (255 - cy, cu, cv)], 0, 6)
    assert np.array_equal(out[0], cy)


def test_dimension_mismatch_rejected(oracle):
    cy, cu, cv = clean_scene()
    small = (np.zeros((32, 32), np.uint8), np.full((16, 16), 128, np.uint8), np.full((16, 16), 128, np.uint8))
    with pytest.raises(RuntimeError, match="ReferenceDimensionsMismatch"):
        oracle.build_arnr_altref([(cy, cu, cv), small], 0, 3)


def test_weight_table_formula(oracle):
    # weight_table_matches_pixel_weight (:838): w = 16 S / (S + d^2),
    # checked through a two-frame blend of flat planes at every |d|.
    for strength in (1, 3, 6):
        s = 8 << strength
        for d in (0, 1, 4, 17, 255):
            base = np.full((16, 16), 0, np.uint8)
            other = np.full((16, 16), d, np.uint8)
            c = np.full((8, 8), 128, np.uint8)
            # SAD per pixel must stay <= 12 for the block to blend.
            if d > 12:
                continue
            out = oracle.build_arnr_altref([(base, c, c), (other, c, c)], 0, strength)
            w = (16 * s) // (s + d * d)
            acc, ws = 0 + w * d, 16 + w
            assert int(out[0][0, 0]) == (acc + ws // 2) // ws
