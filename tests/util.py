"""Plane builders shared by the tests (restating the reference test helpers)."""
import numpy as np


def ramp_plane(width, height):
    """ramp_plane (src/motion_search.rs tests): (x + 3y) % 251."""
    y, x = np.mgrid[0:height, 0:width]
    return ((x + y * 3) % 251).astype(np.uint8)


def feature_plane(width, height, bg, fg, fx, fy, feat):
    """feature_plane (src/motion_search.rs tests): a feat x feat square."""
    p = np.full((height, width), bg, np.uint8)
    p[fy : fy + feat, fx : fx + feat] = fg
    return p


def two_d_ramp_plane(width, height):
    y, x = np.mgrid[0:height, 0:width]
    return np.clip(x + 3 * y, 0, 240).astype(np.uint8)


def stepped_plane(width, height):
    """stepped_plane (src/motion_search.rs tests)."""
    y, x = np.mgrid[0:height, 0:width]
    base = np.clip(x + 2 * y, 0, 180)
    step = np.where(x % 3 == 0, 40, 0)
    stripe = np.where(y % 5 == 0, -20, 0)
    return np.clip(base + step + stripe, 0, 240).astype(np.uint8)


def mb_block(plane, mb_col, mb_row):
    return np.ascontiguousarray(plane[mb_row * 16 : mb_row * 16 + 16, mb_col * 16 : mb_col * 16 + 16]).reshape(256)


def lcg_bytes(n, seed):
    """Deterministic byte stream (LCG) for stress inputs."""
    out = np.zeros(n, np.uint8)
    s = seed & 0xFFFFFFFF
    for i in range(n):
        s = (s * 1664525 + 1013904223) & 0xFFFFFFFF
        out[i] = (s >> 24) & 0xFF
    return out


def extract_mbs(y, mb_rows, mb_cols):
    """Edge-replicated 16x16 source MBs in raster order (extract_mb,
    src/encoder.rs:5549) and their (mb_col, mb_row) positions."""
    h, w = y.shape
    ys = np.minimum(np.arange(mb_rows * 16), h - 1)
    xs = np.minimum(np.arange(mb_cols * 16), w - 1)
    p = y[np.ix_(ys, xs)]
    mbs = p.reshape(mb_rows, 16, mb_cols, 16).transpose(0, 2, 1, 3).reshape(-1, 256)
    xy = np.stack(np.meshgrid(np.arange(mb_cols), np.arange(mb_rows)), -1).reshape(-1, 2)
    return np.ascontiguousarray(mbs), np.ascontiguousarray(xy.astype(np.uint32))


def sr_tuples(a):
    """Structured search results -> list of (row, col, sad)."""
    return [(int(r["mv"]["row"]), int(r["mv"]["col"]), int(r["sad"])) for r in a]


def windows_ref(src, ref, xy):
    """The learned proposal's cost volume by its definition (FP32, before
    the BF16 rounding vp8a_lp_windows applies): both planes averaged 2x2
    (rounded, each coordinate clamped to the plane), the 8 x 8
    half-resolution MB of each listed (col, row) against the 40 x 40
    half-resolution window from (-32, -32) px; at cell (oy, ox) channel 0 is
    (32 - SAD / 64) / 32 and channel 1 (window[oy + 4][ox + 4] - 128) / 64.
    Returns [n, 32, 32, 2] float32."""
    h, w = src.shape

    def avg2(p, ys, xs):
        s = sum(p[np.clip(ys + a, 0, h - 1)][:, np.clip(xs + b, 0, w - 1)].astype(np.int32)
                for a in (0, 1) for b in (0, 1))
        return ((s + 2) >> 2).astype(np.int32)

    out = np.zeros((len(xy), 32, 32, 2), np.float32)
    for i, (c, r) in enumerate(np.asarray(xy).reshape(-1, 2)):
        mx, my = int(c) * 16, int(r) * 16
        win = avg2(ref, my - 32 + 2 * np.arange(40), mx - 32 + 2 * np.arange(40))
        mb = avg2(src, my + 2 * np.arange(8), mx + 2 * np.arange(8))
        sad = np.abs(np.lib.stride_tricks.sliding_window_view(win, (8, 8))[:32, :32] - mb).sum(axis=(2, 3))
        out[i, :, :, 0] = (np.float32(32.0) - sad.astype(np.float32) * np.float32(1 / 64)) * np.float32(1 / 32)
        out[i, :, :, 1] = (win[4:36, 4:36].astype(np.float32) - np.float32(128)) * np.float32(1 / 64)
    return out
