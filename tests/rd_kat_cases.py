"""Known-answer cases for the RD-effort inter search (decide_mb_rd's search,
src/encoder/inter_search.rs:224-552 and :846-1060), derived by hand from
the reference's listing. The reference has no unit tests for this module,
so these pin the restatement (and, through the parity tests, the kernel)
to the listing's behaviour:

* the whole-pel descent's shape per effort (`descent_rounds` 4/8/16/32,
  `wide_pattern`, `search_other_refs`, :95-161): on a horizontal ramp whose
  best match lies 40 px to the right, a NARROW round moves one pixel and a
  WIDE round two, so the whole-pel result is 4 px (Fastest: 4 NARROW
  rounds), 24 px (Fast: 8 WIDE + 8 NARROW), and the exact 40 px for
  Balanced and Thorough (the search stops once the SAD is 0);
* the `good_enough = 128 * max(1, y1_ac / 8)` gate (:868-869): a seed
  whose SAD is at most good_enough is not descended from, and a reference
  whose result is good enough ends the reference loop;
* the +-255 px cap on the whole-pel range (:871-879): a seed far outside
  it is clamped to 255 px;
* the half-pel gate |mv| <= 1020 and the quarter-pel gate |mv| <= 1022
  (:513, :529): around a whole-pel result at 255 px no half-pel candidate
  beyond 1020 quarter-pels is scored, while a quarter-pel one at 1021 is.

Every case is one reference plane and one source frame built here, the
census neighbours given explicitly.
"""
import numpy as np

from vp8a import abi

RAMP_W, RAMP_H = 256, 48          # 16 x 3 MBs
RAMP_MB = (4, 1)                  # (col, row) of the MB under test
RAMP_D = 40                       # its best match, pixels to the right


def ramp_case(d=RAMP_D):
    """Reference luma Y(x, y) = x; the source is the reference moved `d` px
    left, so at the MB under test (x = 64..79) the source is x + d and the
    whole-pel SAD at displacement v pixels is 256 * |v - d| exactly (the
    ramp stays inside 0..255). Chroma is flat."""
    y = np.tile(np.arange(RAMP_W, dtype=np.int32), (RAMP_H, 1))
    ref_y = y.astype(np.uint8)
    src_y = np.clip(y + d, 0, 255).astype(np.uint8)
    cu = np.full((RAMP_H // 2, RAMP_W // 2), 128, np.uint8)
    ref = (ref_y, cu, cu.copy())
    src = (src_y, cu.copy(), cu.copy())
    return src, ref


def intra_neighbours(mb_cols, mb_rows):
    """Census neighbours that are all intra (or outside the frame): every
    census vector is zero, so the only seed is the zero vector."""
    return np.zeros(mb_cols * mb_rows * 3, abi.MB_INFO_DTYPE)


# Whole-pel result (quarter-pel column, SAD) of the ramp MB per effort.
RAMP_WHOLE = {
    abi.EFFORT_FASTEST: (4 * 4, 256 * (RAMP_D - 4)),
    abi.EFFORT_FAST: (4 * 24, 256 * (RAMP_D - 24)),
    abi.EFFORT_BALANCED: (4 * RAMP_D, 0),
    abi.EFFORT_THOROUGH: (4 * RAMP_D, 0),
}

FAR_W, FAR_H = 640, 48            # 40 x 3 MBs
FAR_MB = (5, 1)


def far_case(seed, half_pel_source=False):
    """A textured reference and a source whose MB under test matches the
    reference 255 px to the right (or, with `half_pel_source`, half a pixel
    further: the six-tap half-pel sample between 255 and 256 px), with
    census neighbours on LAST all pointing 300 px to the right (1200
    quarter-pels). The whole-pel range is capped at 255 px, so the seed
    clamps to 255 px instead of 300."""
    rng = np.random.default_rng(seed)
    ref_y = rng.integers(0, 256, (FAR_H, FAR_W), dtype=np.int32)
    mc, mr = FAR_MB
    src_y = rng.integers(0, 256, (FAR_H, FAR_W), dtype=np.int32)
    x0, y0 = mc * 16, mr * 16
    if half_pel_source:
        taps = np.array([3, -16, 77, 77, -16, 3])
        for r in range(16):
            for c in range(16):
                x = x0 + 255 + c
                v = int(np.dot(taps, ref_y[y0 + r, x - 2:x + 4]))
                src_y[y0 + r, x0 + c] = min(max((v + 64) >> 7, 0), 255)
    else:
        src_y[y0:y0 + 16, x0:x0 + 16] = ref_y[y0:y0 + 16, x0 + 255:x0 + 255 + 16]
    cu = np.full((FAR_H // 2, FAR_W // 2), 128, np.uint8)
    ref = (ref_y.astype(np.uint8), cu, cu.copy())
    src = (src_y.astype(np.uint8), cu.copy(), cu.copy())
    nb = intra_neighbours(FAR_W // 16, FAR_H // 16).reshape(FAR_H // 16, FAR_W // 16, 3)
    for k in range(3):  # above, left, above-left of every MB: LAST, (0, 1200)
        nb[:, :, k]["ref_frame"] = abi.REF_LAST
        nb[:, :, k]["mv"]["row"] = 0
        nb[:, :, k]["mv"]["col"] = 1200
    return src, ref, np.ascontiguousarray(nb.reshape(-1))


def mb_of(out, mb):
    return out[mb[1], mb[0]]
