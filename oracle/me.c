/*
 * me.c — oracle restatement of the §17/§18 motion-search primitives.
 *
 * TEST INFRASTRUCTURE ONLY (see vp8a_oracle.h). Follows:
 *   src/motion_search.rs:79-728 (SAD, diamond, half/quarter refinement)
 *   src/motion_comp.rs:187-303 (stored_luma_mv, SIXTAP_FILTERS),
 *   :396-402 (interp), :837-1057 (halo fetch, two-pass MB six-tap),
 *   :1513-1560 (whole-pixel MB fetch).
 * The six-tap is the scalar two-pass listing sixtap_mb_luma_scalar
 * (src/motion_comp.rs:1018-1057): the reference's identity elision and
 * TapPlan run forms are asserted byte-exact with it by its own tests.
 */
#include <stdlib.h>
#include <string.h>

#include "vp8a_oracle.h"

#define MV_MIN (-1023)
#define MV_MAX 1023
#define WHOLE_PIXEL_STEP 4
#define HALF_PIXEL_STEP 2
#define QUARTER_PIXEL_STEP 1

/* SIXTAP_FILTERS (src/motion_comp.rs:294-303) = RFC 6386 §18.3 filters[8][6]. */
static const int SIXTAP[8][6] = {
    {0, 0, 128, 0, 0, 0},     {0, -6, 123, 12, -1, 0}, {2, -11, 108, 36, -8, 1},
    {0, -9, 93, 50, -6, 0},   {3, -16, 77, 77, -16, 3}, {0, -6, 50, 93, -9, 0},
    {1, -8, 36, 108, -11, 2}, {0, -1, 12, 123, -6, 0},
};

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int64_t clampl(int64_t v, int64_t lo, int64_t hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

/* stored_luma_mv (src/motion_comp.rs:187): wrapping doubling to eighth-pel. */
static inline vp8a_mv stored_luma_mv(vp8a_mv mv) {
  vp8a_mv o;
  o.row = (int16_t)(uint16_t)((uint16_t)mv.row * 2u);
  o.col = (int16_t)(uint16_t)((uint16_t)mv.col * 2u);
  return o;
}

/* block_sad_16x16 (src/motion_search.rs:138-161). */
uint32_t vo_block_sad_16x16(const uint8_t* src, const uint8_t* pred) {
  uint32_t acc = 0;
  for (int i = 0; i < 256; i++) {
    int d = (int)src[i] - (int)pred[i];
    acc += (uint32_t)(d < 0 ? -d : d);
  }
  return acc;
}

/* fetch_luma_mb_whole_pixel (src/motion_comp.rs:1513-1560): per-pixel
 * edge-clamped 16x16 fetch at (mb_x, mb_y) + (mv_eighth >> 3). */
void vo_fetch_luma_mb_whole_pixel(const uint8_t* plane, size_t stride, size_t w, size_t h,
                                  size_t mb_x, size_t mb_y, vp8a_mv mv, uint8_t* out) {
  int64_t sx0 = (int64_t)mb_x + (mv.col >> 3);
  int64_t sy0 = (int64_t)mb_y + (mv.row >> 3);
  for (int r = 0; r < 16; r++) {
    int64_t sy = clampl(sy0 + r, 0, (int64_t)h - 1);
    for (int c = 0; c < 16; c++) {
      int64_t sx = clampl(sx0 + c, 0, (int64_t)w - 1);
      out[r * 16 + c] = plane[(size_t)sy * stride + (size_t)sx];
    }
  }
}

/* fetch_luma_mb_halo (src/motion_comp.rs:837-880): 21x21 region with the
 * block origin at (2, 2), edge-clamped. */
void vo_fetch_luma_mb_halo(const uint8_t* plane, size_t stride, size_t w, size_t h,
                           size_t mb_x, size_t mb_y, vp8a_mv mv, uint8_t* out) {
  int64_t sx0 = (int64_t)mb_x + (mv.col >> 3) - 2;
  int64_t sy0 = (int64_t)mb_y + (mv.row >> 3) - 2;
  for (int r = 0; r < 21; r++) {
    int64_t sy = clampl(sy0 + r, 0, (int64_t)h - 1);
    for (int c = 0; c < 21; c++) {
      int64_t sx = clampl(sx0 + c, 0, (int64_t)w - 1);
      out[r * 21 + c] = plane[(size_t)sy * stride + (size_t)sx];
    }
  }
}

/* interp (src/motion_comp.rs:396-402): six-tap dot product, (a+64)>>7,
 * clamp255. */
static inline uint8_t interp(const int* f, const uint8_t* s, size_t step) {
  int a = 0;
  for (int i = 0; i < 6; i++) a += (int)s[i * step] * f[i];
  return (uint8_t)clampi((a + 64) >> 7, 0, 255);
}

/* sixtap_mb_luma_scalar (src/motion_comp.rs:1018-1057): horizontal pass
 * over 21 rows into an 8-bit intermediate, then the vertical pass. */
void vo_sixtap_mb_luma(const uint8_t* halo, int mx, int my, uint8_t* out) {
  const int* fh = SIXTAP[mx & 7];
  const int* fv = SIXTAP[my & 7];
  uint8_t temp[21 * 16];
  for (int r = 0; r < 21; r++)
    for (int c = 0; c < 16; c++) temp[r * 16 + c] = interp(fh, halo + r * 21 + c, 1);
  for (int r = 0; r < 16; r++)
    for (int c = 0; c < 16; c++) out[r * 16 + c] = interp(fv, temp + r * 16 + c, 16);
}

/* mb_luma_sad_at_whole_mv (src/motion_search.rs:291-349). The fused
 * in-bounds branch is a pure row copy of the fetch, so one clamped fetch
 * covers both branches. */
uint32_t vo_mb_luma_sad_at_whole_mv(const vp8a_luma_ref* r, size_t mb_col, size_t mb_row,
                                    const uint8_t* src_y, vp8a_mv mv) {
  uint8_t pred[256];
  vo_fetch_luma_mb_whole_pixel(r->plane, r->stride, r->width, r->height, mb_col * 16,
                               mb_row * 16, stored_luma_mv(mv), pred);
  return vo_block_sad_16x16(src_y, pred);
}

/* mb_luma_sad_at_mv (src/motion_search.rs:470-529). */
uint32_t vo_mb_luma_sad_at_mv(const vp8a_luma_ref* r, size_t mb_col, size_t mb_row,
                              const uint8_t* src_y, vp8a_mv mv) {
  vp8a_mv e = stored_luma_mv(mv);
  int mx = e.col & 7, my = e.row & 7;
  uint8_t pred[256];
  if (mx == 0 && my == 0) {
    vo_fetch_luma_mb_whole_pixel(r->plane, r->stride, r->width, r->height, mb_col * 16,
                                 mb_row * 16, e, pred);
  } else {
    uint8_t halo[441];
    vo_fetch_luma_mb_halo(r->plane, r->stride, r->width, r->height, mb_col * 16, mb_row * 16, e,
                          halo);
    vo_sixtap_mb_luma(halo, mx, my, pred);
  }
  return vo_block_sad_16x16(src_y, pred);
}

/* clamp_component / snap_to_whole_pixel (src/motion_search.rs:354-370). */
static inline int16_t clamp_component(int32_t v) { return (int16_t)clampi(v, MV_MIN, MV_MAX); }
static inline int16_t snap_whole(int16_t v) {
  return (int16_t)((v / WHOLE_PIXEL_STEP) * WHOLE_PIXEL_STEP);
}

/* small_diamond_search_luma (src/motion_search.rs:381-442): clamp then
 * snap; N,S,W,E relative to the moving best; strict '<'; collapsed
 * candidates skipped. */
vp8a_search_result vo_small_diamond_search_luma(const vp8a_luma_ref* r, size_t mb_col,
                                                size_t mb_row, const uint8_t* src_y,
                                                vp8a_mv center, uint32_t max_iters) {
  vp8a_mv best;
  best.row = snap_whole(clamp_component(center.row));
  best.col = snap_whole(clamp_component(center.col));
  uint32_t best_sad = vo_mb_luma_sad_at_whole_mv(r, mb_col, mb_row, src_y, best);
  static const int nb[4][2] = {{-4, 0}, {4, 0}, {0, -4}, {0, 4}};
  for (uint32_t it = 0; it < max_iters; it++) {
    int improved = 0;
    for (int k = 0; k < 4; k++) {
      vp8a_mv cand;
      cand.row = snap_whole(clamp_component((int32_t)best.row + nb[k][0]));
      cand.col = snap_whole(clamp_component((int32_t)best.col + nb[k][1]));
      if (cand.row == best.row && cand.col == best.col) continue;
      uint32_t s = vo_mb_luma_sad_at_whole_mv(r, mb_col, mb_row, src_y, cand);
      if (s < best_sad) {
        best_sad = s;
        best = cand;
        improved = 1;
      }
    }
    if (!improved) break;
  }
  vp8a_search_result res = {best, best_sad};
  return res;
}

/* The eight offsets of half/quarter refinement in their fixed order
 * (src/motion_search.rs:589-598 and :690-699). */
static const int REFINE_OFFS[8][2] = {{-1, -1}, {-1, 0}, {-1, 1}, {0, -1},
                                      {0, 1},   {1, -1}, {1, 0},  {1, 1}};

static vp8a_search_result refine(const vp8a_luma_ref* r, size_t mb_col, size_t mb_row,
                                 const uint8_t* src_y, vp8a_mv center, int step) {
  vp8a_mv best = center;
  uint32_t best_sad = vo_mb_luma_sad_at_mv(r, mb_col, mb_row, src_y, best);
  for (int k = 0; k < 8; k++) {
    vp8a_mv cand;
    cand.row = clamp_component((int32_t)center.row + REFINE_OFFS[k][0] * step);
    cand.col = clamp_component((int32_t)center.col + REFINE_OFFS[k][1] * step);
    if (cand.row == best.row && cand.col == best.col) continue;
    uint32_t s = vo_mb_luma_sad_at_mv(r, mb_col, mb_row, src_y, cand);
    if (s < best_sad) {
      best_sad = s;
      best = cand;
    }
  }
  vp8a_search_result res = {best, best_sad};
  return res;
}

/* half_pixel_refine_luma (src/motion_search.rs:564-627). */
vp8a_search_result vo_half_pixel_refine_luma(const vp8a_luma_ref* r, size_t mb_col,
                                             size_t mb_row, const uint8_t* src_y,
                                             vp8a_mv center) {
  return refine(r, mb_col, mb_row, src_y, center, HALF_PIXEL_STEP);
}

/* quarter_pixel_refine_luma (src/motion_search.rs:666-728). */
vp8a_search_result vo_quarter_pixel_refine_luma(const vp8a_luma_ref* r, size_t mb_col,
                                                size_t mb_row, const uint8_t* src_y,
                                                vp8a_mv center) {
  return refine(r, mb_col, mb_row, src_y, center, QUARTER_PIXEL_STEP);
}

/* ------------------------------------------------------------ batched forms */

void vo_mb_luma_sad_at_mv_batch(const vp8a_luma_ref* r, const uint8_t* src_mbs,
                                const uint32_t* mb_xy, const vp8a_mv* mvs, uint32_t n,
                                uint32_t* out) {
  for (uint32_t i = 0; i < n; i++)
    out[i] = vo_mb_luma_sad_at_mv(r, mb_xy[2 * i], mb_xy[2 * i + 1], src_mbs + 256 * (size_t)i,
                                  mvs[i]);
}

void vo_small_diamond_batch(const vp8a_luma_ref* r, const uint8_t* src_mbs,
                            const uint32_t* mb_xy, const vp8a_mv* centers, uint32_t max_iters,
                            uint32_t n, vp8a_search_result* out) {
  for (uint32_t i = 0; i < n; i++)
    out[i] = vo_small_diamond_search_luma(r, mb_xy[2 * i], mb_xy[2 * i + 1],
                                          src_mbs + 256 * (size_t)i, centers[i], max_iters);
}

void vo_half_refine_batch(const vp8a_luma_ref* r, const uint8_t* src_mbs, const uint32_t* mb_xy,
                          const vp8a_mv* centers, uint32_t n, vp8a_search_result* out) {
  for (uint32_t i = 0; i < n; i++)
    out[i] = vo_half_pixel_refine_luma(r, mb_xy[2 * i], mb_xy[2 * i + 1],
                                       src_mbs + 256 * (size_t)i, centers[i]);
}

void vo_quarter_refine_batch(const vp8a_luma_ref* r, const uint8_t* src_mbs,
                             const uint32_t* mb_xy, const vp8a_mv* centers, uint32_t n,
                             vp8a_search_result* out) {
  for (uint32_t i = 0; i < n; i++)
    out[i] = vo_quarter_pixel_refine_luma(r, mb_xy[2 * i], mb_xy[2 * i + 1],
                                          src_mbs + 256 * (size_t)i, centers[i]);
}

typedef struct {
  const vp8a_luma_ref* r;
  const uint8_t* src;
  const uint32_t* xy;
  const vp8a_mv* centers;
  uint32_t max_iters;
  vp8a_search_result *whole, *half, *quarter;
} descent_job;

static void descent_task(void* arg, uint32_t i) {
  descent_job* j = (descent_job*)arg;
  size_t c = j->xy[2 * i], rr = j->xy[2 * i + 1];
  const uint8_t* s = j->src + 256 * (size_t)i;
  vp8a_search_result w = vo_small_diamond_search_luma(j->r, c, rr, s, j->centers[i], j->max_iters);
  vp8a_search_result h = vo_half_pixel_refine_luma(j->r, c, rr, s, w.mv);
  vp8a_search_result q = vo_quarter_pixel_refine_luma(j->r, c, rr, s, h.mv);
  if (j->whole) j->whole[i] = w;
  if (j->half) j->half[i] = h;
  if (j->quarter) j->quarter[i] = q;
}

/* The per-(MB, ref) descent of pick_mb_for_ref (src/encoder.rs:8576-8596). */
void vo_motion_descent_batch(const vp8a_luma_ref* r, const uint8_t* src_mbs,
                             const uint32_t* mb_xy, const vp8a_mv* centers, uint32_t max_iters,
                             uint32_t n, vp8a_search_result* whole, vp8a_search_result* half,
                             vp8a_search_result* quarter, uint32_t threads) {
  descent_job j = {r, src_mbs, mb_xy, centers, max_iters, whole, half, quarter};
  vo_parallel_for(n, threads, descent_task, &j);
}
