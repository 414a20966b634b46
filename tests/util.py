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
