"""The cost-volume definition the GPU parity test holds vp8a_lp_windows to
(`util.windows_ref`), checked against a scalar restatement of the same
formula at sampled cells, including MBs whose windows cross every plane
edge."""
import numpy as np
import pytest
from util import windows_ref


def avg2_scalar(p, y, x):
    h, w = p.shape
    s = 0
    for a in (0, 1):
        for b in (0, 1):
            s += int(p[min(max(y + a, 0), h - 1), min(max(x + b, 0), w - 1)])
    return (s + 2) >> 2


@pytest.mark.parametrize("w,h", [(72, 40), (48, 48)])
def test_windows_definition_matches_the_scalar_formula(w, h):
    rng = np.random.default_rng(w + h)
    src = rng.integers(0, 256, (h, w), dtype=np.uint8)
    ref = rng.integers(0, 256, (h, w), dtype=np.uint8)
    mbc, mbr = (w + 15) // 16, (h + 15) // 16
    xy = np.array([[c, r] for r in range(mbr) for c in range(mbc)], np.uint32)
    got = windows_ref(src, ref, xy)
    for i, (c, r) in enumerate(xy):
        mx, my = int(c) * 16, int(r) * 16
        for oy, ox in ((0, 0), (0, 31), (31, 0), (31, 31), (7, 19), (16, 16)):
            sad = sum(abs(avg2_scalar(ref, my - 32 + 2 * (oy + ky), mx - 32 + 2 * (ox + kx)) -
                          avg2_scalar(src, my + 2 * ky, mx + 2 * kx)) for ky in range(8) for kx in range(8))
            c0 = (np.float32(32) - np.float32(sad) * np.float32(1 / 64)) * np.float32(1 / 32)
            c1 = (np.float32(avg2_scalar(ref, my - 32 + 2 * (oy + 4), mx - 32 + 2 * (ox + 4))) - np.float32(128)) \
                * np.float32(1 / 64)
            assert got[i, oy, ox, 0] == c0 and got[i, oy, ox, 1] == c1, (i, oy, ox)
