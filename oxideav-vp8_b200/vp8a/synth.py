"""Seeded synthetic I420 sequences (the stand-in for a video corpus).

The reference publishes no dataset for this path; its benchmark inputs are
generated. This module produces them deterministically from a seed:

* frame 0 = 128 + the sum of 6 sinusoid gratings (random orientation,
  period 8-64 px, amplitude 20-50) + Gaussian noise sigma 4, clipped;
* frame k = frame k-1 translated by a random quarter-pel offset in
  [-8, 8]^2 px through the §18.3 two-pass six-tap filter (8-bit
  intermediate, edge-clamped fetch) + fresh noise sigma 3, clipped;
* chroma planes follow the same recipe at half resolution (2 gratings,
  amplitude 8-16, noise sigma 2) and half the displacement.

`quantised_recon` builds the stand-in for an unfiltered qi-44
reconstruction: every 4x4 block of the MB-padded source is transformed by
an orthonormal 4x4 DCT, quantised with half the qi-44 VP8 steps (VP8's DCT
domain is twice the orthonormal one: DC 40 -> 20, AC 48 -> 24), dequantised
and inverse-transformed. It has the 4x4 blocking the §15 filter targets;
`has_coeffs` marks MBs with any non-zero quantised coefficient.
"""
import hashlib

import numpy as np

SIXTAP = np.array(
    [
        [0, 0, 128, 0, 0, 0],
        [0, -6, 123, 12, -1, 0],
        [2, -11, 108, 36, -8, 1],
        [0, -9, 93, 50, -6, 0],
        [3, -16, 77, 77, -16, 3],
        [0, -6, 50, 93, -9, 0],
        [1, -8, 36, 108, -11, 2],
        [0, -1, 12, 123, -6, 0],
    ],
    np.int32,
)


def translate(plane, e_row, e_col):
    """Resample `plane` at (y + e_row/8, x + e_col/8) with the §18.3 two-pass
    six-tap filter (horizontal first, 8-bit intermediate), clamping fetches
    to the plane edge."""
    h, w = plane.shape
    iy, fy = e_row >> 3, e_row & 7
    ix, fx = e_col >> 3, e_col & 7
    ys = np.clip(np.arange(-2, h + 3) + iy, 0, h - 1)
    xs = np.clip(np.arange(-2, w + 3) + ix, 0, w - 1)
    p = plane[np.ix_(ys, xs)].astype(np.int32)
    t = np.zeros((h + 5, w), np.int32)
    for k in range(6):
        t += p[:, k : k + w] * SIXTAP[fx][k]
    t = np.clip((t + 64) >> 7, 0, 255)
    o = np.zeros((h, w), np.int32)
    for k in range(6):
        o += t[k : k + h, :] * SIXTAP[fy][k]
    return np.clip((o + 64) >> 7, 0, 255).astype(np.uint8)


def _gratings(rng, h, w, n, amp_lo, amp_hi):
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    acc = np.zeros((h, w), np.float64)
    for _ in range(n):
        theta = rng.uniform(0.0, np.pi)
        period = rng.uniform(8.0, 64.0)
        amp = rng.uniform(amp_lo, amp_hi)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        acc += amp * np.sin(2.0 * np.pi * (x * np.cos(theta) + y * np.sin(theta)) / period + phase)
    return acc


def _noisy(rng, base, sigma):
    return np.clip(np.rint(base + rng.normal(0.0, sigma, base.shape)), 0, 255).astype(np.uint8)


def make_sequence(width, height, n_frames, seed, pieces=0, occluders=0):
    """Returns (frames, offsets): frames = list of (y, u, v) uint8 arrays of
    the visible size; offsets[k] = (row, col) quarter-pel translation that
    produced frame k from frame k-1 (offsets[0] = (0, 0)).

    With `pieces` > 0 the picture is cut into that many horizontal bands,
    each translated by its own random quarter-pel offset per frame
    (offsets[k] then lists the band offsets), and `occluders` flat
    rectangles move across the picture with their own velocities — the
    piecewise-motion content that exercises NEW/NEAR/SPLITMV decisions."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cw, ch = (width + 1) // 2, (height + 1) // 2
    y0 = _noisy(rng, 128.0 + _gratings(rng, height, width, 6, 20.0, 50.0), 4.0)
    u0 = _noisy(rng, 128.0 + _gratings(rng, ch, cw, 2, 8.0, 16.0), 2.0)
    v0 = _noisy(rng, 128.0 + _gratings(rng, ch, cw, 2, 8.0, 16.0), 2.0)
    frames = [(y0, u0, v0)]
    offsets = [(0, 0)]
    occ = []
    for _ in range(occluders):
        ow, oh = int(rng.integers(8, max(9, width // 3))), int(rng.integers(8, max(9, height // 3)))
        occ.append([float(rng.uniform(0, width)), float(rng.uniform(0, height)), ow, oh,
                    int(rng.integers(0, 256)), float(rng.uniform(-6, 6)), float(rng.uniform(-6, 6))])
    for _ in range(1, n_frames):
        py, pu, pv = frames[-1]
        if pieces <= 0:
            dr, dc = (int(v) for v in rng.integers(-32, 33, size=2))
            y = translate(py, 2 * dr, 2 * dc)
            u = translate(pu, dr, dc)
            v = translate(pv, dr, dc)
            offsets.append((dr, dc))
        else:
            y, u, v = py.copy(), pu.copy(), pv.copy()
            bands = []
            for b in range(pieces):
                dr, dc = (int(x) for x in rng.integers(-32, 33, size=2))
                r0, r1 = b * height // pieces, (b + 1) * height // pieces
                y[r0:r1] = translate(py, 2 * dr, 2 * dc)[r0:r1]
                c0, c1 = r0 // 2, (r1 + 1) // 2
                u[c0:c1] = translate(pu, dr, dc)[c0:c1]
                v[c0:c1] = translate(pv, dr, dc)[c0:c1]
                bands.append((dr, dc))
            offsets.append(tuple(bands))
        for o in occ:
            o[0] += o[5]
            o[1] += o[6]
            x0, y0_ = int(round(o[0])) % width, int(round(o[1])) % height
            y[y0_ : y0_ + o[3], x0 : x0 + o[2]] = o[4]
            u[y0_ // 2 : (y0_ + o[3]) // 2, x0 // 2 : (x0 + o[2]) // 2] = 255 - o[4]
        y = _noisy(rng, y.astype(np.float64), 3.0)
        u = _noisy(rng, u.astype(np.float64), 2.0)
        v = _noisy(rng, v.astype(np.float64), 2.0)
        frames.append((y, u, v))
    return frames, offsets


def digest(frames):
    """sha256 over every plane of every frame (recorded with results)."""
    h = hashlib.sha256()
    for f in frames:
        for p in f:
            h.update(np.ascontiguousarray(p).tobytes())
    return h.hexdigest()


def _dct4():
    d = np.zeros((4, 4))
    for k in range(4):
        for n in range(4):
            d[k, n] = (0.5 if k == 0 else np.sqrt(0.5)) * np.cos(np.pi * (2 * n + 1) * k / 8.0)
    return d


def _quantise_plane(p, q_dc, q_ac):
    h, w = p.shape
    d = _dct4()
    b = p.astype(np.float64).reshape(h // 4, 4, w // 4, 4).transpose(0, 2, 1, 3)
    coef = np.einsum("ij,abjk,lk->abil", d, b - 128.0, d)
    step = np.full((4, 4), float(q_ac))
    step[0, 0] = float(q_dc)
    q = np.rint(coef / step)
    rec = np.einsum("ji,abjk,kl->abil", d, q * step, d) + 128.0
    rec = np.clip(np.rint(rec), 0, 255).astype(np.uint8)
    nz = (q != 0).any(axis=(2, 3))  # per 4x4 block
    return rec.transpose(0, 2, 1, 3).reshape(h, w), nz


def quantised_recon(padded, q_dc=20, q_ac=24):
    """MB-padded (y, u, v) -> (recon (y, u, v), has_coeffs[mb_rows, mb_cols])."""
    y, u, v = padded
    ry, ny = _quantise_plane(y, q_dc, q_ac)
    ru, nu = _quantise_plane(u, q_dc, q_ac)
    rv, nv = _quantise_plane(v, q_dc, q_ac)
    mbr, mbc = y.shape[0] // 16, y.shape[1] // 16
    has = ny.reshape(mbr, 4, mbc, 4).any(axis=(1, 3))
    has |= nu.reshape(mbr, 2, mbc, 2).any(axis=(1, 3))
    has |= nv.reshape(mbr, 2, mbc, 2).any(axis=(1, 3))
    return (ry, ru, rv), has
