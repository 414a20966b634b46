/*
 * lf.c — oracle restatement of the §15 loop filter and the §9.4 search.
 *
 * TEST INFRASTRUCTURE ONLY (see vp8a_oracle.h). Follows src/loop_filter.rs:
 *   LoopFilterParams::derive                 :99-148
 *   clamp_s8 / u2s / s2u / common_adjust     :157-233
 *   simple_segment / filter_yes / hev        :235-290
 *   subblock_filter / mb_filter              :292-371 (scalar listings; the
 *     branch-free run form :407-476 is asserted equal by the reference)
 *   calculate_mb_filter_level(_inter)        :1222-1331
 *   filter_inter_frame_flags / filter_frame_flags (MB raster order, four
 *     steps per MB)                          :1364-1489, :2506-2630
 *   edge walkers                             :1515-1870
 *   plane_visible_ssd / reconstruction_ssd   :1941-1977
 *   score_filter_candidate                   :2062-2092
 *   select_filter_params_threaded            :2133-2199
 *   select_filter_params_sampled             :2288-2412
 */
#include <stdlib.h>
#include <string.h>

#include "vp8a_oracle.h"

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int absi(int v) { return v < 0 ? -v : v; }

void vo_lf_derive(uint8_t level, uint8_t sharpness, int key_frame, uint8_t out[4]) {
  int interior = level;
  if (sharpness != 0) {
    interior >>= (sharpness > 4) ? 2 : 1;
    int cap = 9 - (int)sharpness;
    if (cap < 0) cap = 0;
    if (interior > cap) interior = cap;
  }
  if (interior == 0) interior = 1;
  int hev;
  if (key_frame) hev = level >= 40 ? 2 : (level >= 15 ? 1 : 0);
  else hev = level >= 40 ? 3 : (level >= 20 ? 2 : (level >= 15 ? 1 : 0));
  int mbedge = ((level + 2) * 2) + interior;
  int subedge = (level * 2) + interior;
  out[0] = (uint8_t)interior;
  out[1] = (uint8_t)hev;
  out[2] = (uint8_t)(mbedge > 255 ? 255 : mbedge);
  out[3] = (uint8_t)(subedge > 255 ? 255 : subedge);
}

static inline int c8(int v) { return v < -128 ? -128 : (v < 128 ? v : 127); }
static inline int u2s(uint8_t v) { return (int)v - 128; }
static inline uint8_t s2u(int v) { return (uint8_t)(c8(v) + 128); }

int32_t vo_common_adjust(int use_outer_taps, uint8_t* seg) {
  int p1 = u2s(seg[0]), p0 = u2s(seg[1]), q0 = u2s(seg[2]), q1 = u2s(seg[3]);
  int outer = use_outer_taps ? c8(p1 - q1) : 0;
  int a = c8(outer + 3 * (q0 - p0));
  int b = c8(a + 3) >> 3;
  a = c8(a + 4) >> 3;
  seg[2] = s2u(q0 - a);
  seg[1] = s2u(p0 + b);
  return a;
}

void vo_simple_segment(uint8_t edge_limit, uint8_t* seg) {
  int p1 = seg[0], p0 = seg[1], q0 = seg[2], q1 = seg[3];
  if (absi(p0 - q0) * 2 + absi(p1 - q1) / 2 <= (int)edge_limit) vo_common_adjust(1, seg);
}

static int filter_yes(int i, int e, int p3, int p2, int p1, int p0, int q0, int q1, int q2,
                      int q3) {
  return (absi(p0 - q0) * 2 + absi(p1 - q1) / 2) <= e && absi(p3 - p2) <= i &&
         absi(p2 - p1) <= i && absi(p1 - p0) <= i && absi(q3 - q2) <= i &&
         absi(q2 - q1) <= i && absi(q1 - q0) <= i;
}
static int hev(int t, int p1, int p0, int q0, int q1) {
  return absi(p1 - p0) > t || absi(q1 - q0) > t;
}

void vo_subblock_filter(uint8_t hev_t, uint8_t interior, uint8_t edge, uint8_t* s) {
  int p3 = u2s(s[0]), p2 = u2s(s[1]), p1 = u2s(s[2]), p0 = u2s(s[3]);
  int q0 = u2s(s[4]), q1 = u2s(s[5]), q2 = u2s(s[6]), q3 = u2s(s[7]);
  if (filter_yes(interior, edge, p3, p2, p1, p0, q0, q1, q2, q3)) {
    int hv = hev(hev_t, p1, p0, q0, q1);
    int a = (vo_common_adjust(hv, s + 2) + 1) >> 1;
    if (!hv) {
      s[5] = s2u(q1 - a);
      s[2] = s2u(p1 + a);
    }
  }
}

void vo_mb_filter(uint8_t hev_t, uint8_t interior, uint8_t edge, uint8_t* s) {
  int p3 = u2s(s[0]), p2 = u2s(s[1]), p1 = u2s(s[2]), p0 = u2s(s[3]);
  int q0 = u2s(s[4]), q1 = u2s(s[5]), q2 = u2s(s[6]), q3 = u2s(s[7]);
  if (filter_yes(interior, edge, p3, p2, p1, p0, q0, q1, q2, q3)) {
    if (!hev(hev_t, p1, p0, q0, q1)) {
      int w = c8(c8(p1 - q1) + 3 * (q0 - p0));
      int a = c8((27 * w + 63) >> 7);
      s[4] = s2u(q0 - a);
      s[3] = s2u(p0 + a);
      a = c8((18 * w + 63) >> 7);
      s[5] = s2u(q1 - a);
      s[2] = s2u(p1 + a);
      a = c8((9 * w + 63) >> 7);
      s[6] = s2u(q2 - a);
      s[1] = s2u(p2 + a);
    } else {
      vo_common_adjust(1, s + 2);
    }
  }
}

/* calculate_mb_filter_level_inter (src/loop_filter.rs:1280-1331); with
 * ref_frame = INTRA it is calculate_mb_filter_level (:1222). */
uint8_t vo_mb_filter_level(const vp8a_filter_config* c, const vp8a_mb_lf_info* mb) {
  int level = c->loop_filter_level;
  if (c->segmentation_enabled) {
    int seg = mb->segment_id < 0 ? 0 : mb->segment_id;
    if (seg > 3) seg = 3;
    if (c->segment_abs) level = c->segment_lf_level[seg];
    else level += c->segment_lf_level[seg];
  }
  level = clampi(level, 0, 63);
  if (c->delta_enabled) {
    int rd;
    switch (mb->ref_frame) {
      case VP8A_REF_LAST: rd = c->ref_delta_last; break;
      case VP8A_REF_GOLDEN: rd = c->ref_delta_golden; break;
      case VP8A_REF_ALTREF: rd = c->ref_delta_altref; break;
      default: rd = c->ref_delta_current; break;
    }
    level += rd;
    if (mb->ref_frame == VP8A_REF_INTRA) {
      if (mb->y_mode_is_bpred) level += c->bpred_mode_delta;
    } else if (mb->inter_mode == VP8A_MODE_ZERO) {
      level += c->zero_mv_mode_delta;
    } else if (mb->inter_mode == VP8A_MODE_SPLIT) {
      level += c->split_mv_mode_delta;
    } else {
      level += c->other_mv_mode_delta;
    }
  }
  return (uint8_t)clampi(level, 0, 63);
}

/* Edge walkers (src/loop_filter.rs:1515-1870). */
static void v_edge_normal(uint8_t* p, size_t stride, size_t x, size_t y0, int len,
                          const uint8_t* prm, int mb_edge) {
  uint8_t edge = mb_edge ? prm[2] : prm[3];
  for (int r = 0; r < len; r++) {
    uint8_t* s = p + (y0 + r) * stride + x - 4;
    uint8_t seg[8];
    memcpy(seg, s, 8);
    if (mb_edge) vo_mb_filter(prm[1], prm[0], edge, seg);
    else vo_subblock_filter(prm[1], prm[0], edge, seg);
    memcpy(s, seg, 8);
  }
}
static void h_edge_normal(uint8_t* p, size_t stride, size_t y, size_t x0, int len,
                          const uint8_t* prm, int mb_edge) {
  uint8_t edge = mb_edge ? prm[2] : prm[3];
  for (int c = 0; c < len; c++) {
    uint8_t seg[8];
    for (int k = 0; k < 8; k++) seg[k] = p[(y - 4 + k) * stride + x0 + c];
    if (mb_edge) vo_mb_filter(prm[1], prm[0], edge, seg);
    else vo_subblock_filter(prm[1], prm[0], edge, seg);
    for (int k = 0; k < 8; k++) p[(y - 4 + k) * stride + x0 + c] = seg[k];
  }
}
static void v_edge_simple(uint8_t* p, size_t stride, size_t x, size_t y0, uint8_t edge) {
  for (int r = 0; r < 16; r++) {
    uint8_t* s = p + (y0 + r) * stride + x - 2;
    uint8_t seg[4];
    memcpy(seg, s, 4);
    vo_simple_segment(edge, seg);
    memcpy(s, seg, 4);
  }
}
static void h_edge_simple(uint8_t* p, size_t stride, size_t y, size_t x0, uint8_t edge) {
  for (int c = 0; c < 16; c++) {
    uint8_t seg[4];
    for (int k = 0; k < 4; k++) seg[k] = p[(y - 2 + k) * stride + x0 + c];
    vo_simple_segment(edge, seg);
    for (int k = 0; k < 4; k++) p[(y - 2 + k) * stride + x0 + c] = seg[k];
  }
}

/* filter_inter_frame_flags (src/loop_filter.rs:1364-1489). `first_row`
 * rows of the MB grid are treated as row 0 (no top edge) — used by the
 * sampled search's bands, which are separate KeyframePlanes. */
static void filter_frame_rows(vp8a_planes* pl, const vp8a_mb_lf_info* mbs,
                              const vp8a_filter_config* cfg, int row_begin, int row_end) {
  size_t ys = pl->y_stride, cs = pl->uv_stride;
  int mb_cols = (int)pl->mb_cols;
  for (int mb_row = row_begin; mb_row < row_end; mb_row++) {
    for (int mb_col = 0; mb_col < mb_cols; mb_col++) {
      const vp8a_mb_lf_info* mb = &mbs[(size_t)mb_row * mb_cols + mb_col];
      uint8_t level = vo_mb_filter_level(cfg, mb);
      if (level == 0) continue;
      uint8_t prm[4];
      vo_lf_derive(level, cfg->sharpness_level, cfg->key_frame, prm);
      int sub = mb->y_mode_is_bpred || mb->has_coeffs;
      size_t yx = (size_t)mb_col * 16, yy = (size_t)mb_row * 16;
      size_t cx = (size_t)mb_col * 8, cy = (size_t)mb_row * 8;
      int has_top = mb_row > row_begin;
      if (cfg->simple) {
        if (mb_col > 0) v_edge_simple(pl->y, ys, yx, yy, prm[2]);
        if (sub)
          for (int q = 1; q < 4; q++) v_edge_simple(pl->y, ys, yx + 4 * q, yy, prm[3]);
        if (has_top) h_edge_simple(pl->y, ys, yy, yx, prm[2]);
        if (sub)
          for (int q = 1; q < 4; q++) h_edge_simple(pl->y, ys, yy + 4 * q, yx, prm[3]);
      } else {
        if (mb_col > 0) {
          v_edge_normal(pl->y, ys, yx, yy, 16, prm, 1);
          v_edge_normal(pl->u, cs, cx, cy, 8, prm, 1);
          v_edge_normal(pl->v, cs, cx, cy, 8, prm, 1);
        }
        if (sub) {
          for (int q = 1; q < 4; q++) v_edge_normal(pl->y, ys, yx + 4 * q, yy, 16, prm, 0);
          v_edge_normal(pl->u, cs, cx + 4, cy, 8, prm, 0);
          v_edge_normal(pl->v, cs, cx + 4, cy, 8, prm, 0);
        }
        if (has_top) {
          h_edge_normal(pl->y, ys, yy, yx, 16, prm, 1);
          h_edge_normal(pl->u, cs, cy, cx, 8, prm, 1);
          h_edge_normal(pl->v, cs, cy, cx, 8, prm, 1);
        }
        if (sub) {
          for (int q = 1; q < 4; q++) h_edge_normal(pl->y, ys, yy + 4 * q, yx, 16, prm, 0);
          h_edge_normal(pl->u, cs, cy + 4, cx, 8, prm, 0);
          h_edge_normal(pl->v, cs, cy + 4, cx, 8, prm, 0);
        }
      }
    }
  }
}

int vo_filter_frame(vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                    const vp8a_filter_config* config) {
  if (!planes || !mbs || !config) return VP8A_E_INVALID_ARGUMENT;
  if (planes->mb_cols == 0 || planes->mb_rows == 0) return VP8A_OK;
  filter_frame_rows(planes, mbs, config, 0, (int)planes->mb_rows);
  return VP8A_OK;
}

/* plane_visible_ssd (src/loop_filter.rs:1941-1960). */
static uint64_t plane_ssd(const uint8_t* rec, size_t rs, const uint8_t* src, size_t ss, size_t w,
                          size_t h) {
  uint64_t ssd = 0;
  for (size_t r = 0; r < h; r++)
    for (size_t c = 0; c < w; c++) {
      int d = (int)rec[r * rs + c] - (int)src[r * ss + c];
      ssd += (uint64_t)(d * d);
    }
  return ssd;
}

uint64_t vo_reconstruction_ssd(const vp8a_planes* pl, const vp8a_source* src) {
  size_t cw = (src->width + 1) / 2, ch = (src->height + 1) / 2;
  return plane_ssd(pl->y, pl->y_stride, src->y, src->y_stride, src->width, src->height) +
         plane_ssd(pl->u, pl->uv_stride, src->u, src->uv_stride, cw, ch) +
         plane_ssd(pl->v, pl->uv_stride, src->v, src->uv_stride, cw, ch);
}

/* Band list of select_filter_params_sampled (src/loop_filter.rs:2302-2330):
 * two MB rows every `every_rows` (at least 2). every_rows = 0 means one
 * whole-frame band. */
static int build_bands(int mb_rows, uint32_t every_rows, int* first, int* rows) {
  if (every_rows == 0) {
    first[0] = 0;
    rows[0] = mb_rows;
    return 1;
  }
  int step = every_rows < 2 ? 2 : (int)every_rows, n = 0;
  for (int fr = 0; fr < mb_rows; fr += step) {
    first[n] = fr;
    rows[n] = (mb_rows - fr) < 2 ? (mb_rows - fr) : 2;
    n++;
  }
  return n;
}

/* score_filter_candidate (src/loop_filter.rs:2062-2092) for every_rows = 0;
 * the sampled search's per-candidate band score (:2331-2375) otherwise. */
uint64_t vo_score_filter_candidate(const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                                   const vp8a_filter_config* base, const vp8a_source* src,
                                   uint8_t level, uint8_t sharpness, uint32_t every_rows) {
  int mb_rows = (int)planes->mb_rows;
  int* first = (int*)malloc(sizeof(int) * (mb_rows + 1));
  int* rows = (int*)malloc(sizeof(int) * (mb_rows + 1));
  int nb = build_bands(mb_rows, every_rows, first, rows);
  size_t ylen = planes->y_stride * (size_t)mb_rows * 16;
  size_t clen = planes->uv_stride * (size_t)mb_rows * 8;
  vp8a_planes cand = *planes;
  uint8_t* buf = NULL;
  if (level != 0) {
    buf = (uint8_t*)malloc(ylen + 2 * clen);
    memcpy(buf, planes->y, ylen);
    memcpy(buf + ylen, planes->u, clen);
    memcpy(buf + ylen + clen, planes->v, clen);
    cand.y = buf;
    cand.u = buf + ylen;
    cand.v = buf + ylen + clen;
  }
  vp8a_filter_config cfg = *base;
  cfg.loop_filter_level = level;
  cfg.sharpness_level = sharpness;
  uint64_t total = 0;
  for (int b = 0; b < nb; b++) {
    if (level != 0) filter_frame_rows(&cand, mbs, &cfg, first[b], first[b] + rows[b]);
    size_t y0 = (size_t)first[b] * 16;
    if (y0 >= src->height) continue;
    size_t bh = (size_t)rows[b] * 16;
    if (bh > src->height - y0) bh = src->height - y0;
    vp8a_planes bp = cand;
    bp.y = cand.y + y0 * cand.y_stride;
    bp.u = cand.u + (y0 / 2) * cand.uv_stride;
    bp.v = cand.v + (y0 / 2) * cand.uv_stride;
    vp8a_source bs = *src;
    bs.height = (uint32_t)bh;
    bs.y = src->y + y0 * src->y_stride;
    bs.u = src->u + (y0 / 2) * src->uv_stride;
    bs.v = src->v + (y0 / 2) * src->uv_stride;
    total += vo_reconstruction_ssd(&bp, &bs);
  }
  free(buf);
  free(first);
  free(rows);
  return total;
}

typedef struct {
  const vp8a_planes* planes;
  const vp8a_mb_lf_info* mbs;
  const vp8a_filter_config* base;
  const vp8a_source* src;
  uint32_t every_rows;
  uint64_t* ssd;
  const uint8_t (*cands)[2];
} sweep_job;

static void sweep_task(void* arg, uint32_t i) {
  sweep_job* j = (sweep_job*)arg;
  uint8_t level = j->cands[i][0], sharp = j->cands[i][1];
  j->ssd[level * 8 + sharp] =
      vo_score_filter_candidate(j->planes, j->mbs, j->base, j->src, level, sharp, j->every_rows);
}

static void score_list(const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                       const vp8a_filter_config* base, const vp8a_source* src,
                       uint32_t every_rows, const uint8_t (*cands)[2], uint32_t n,
                       uint64_t* ssd, uint32_t threads) {
  sweep_job j = {planes, mbs, base, src, every_rows, ssd, cands};
  vo_parallel_for(n, threads, sweep_task, &j);
}

/* Every (level, sharpness) of the 64 x 8 grid. Level 0 scores the
 * unfiltered planes for every sharpness. */
void vo_filter_sweep(const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                     const vp8a_filter_config* base, const vp8a_source* src,
                     uint32_t every_rows, uint64_t* ssd_out, uint32_t threads) {
  uint8_t(*cands)[2] = malloc(sizeof(uint8_t[2]) * 505);
  uint32_t n = 0;
  cands[n][0] = 0;
  cands[n][1] = 0;
  n++;
  for (int l = 1; l < 64; l++)
    for (int s = 0; s < 8; s++) {
      cands[n][0] = (uint8_t)l;
      cands[n][1] = (uint8_t)s;
      n++;
    }
  score_list(planes, mbs, base, src, every_rows, (const uint8_t(*)[2])cands, n, ssd_out,
             threads);
  for (int s = 1; s < 8; s++) ssd_out[s] = ssd_out[0];
  free(cands);
}

/* select_filter_params_threaded (src/loop_filter.rs:2133-2199) as a walk
 * over a table of candidate scores. */
void vo_select_from_table_full(const uint64_t* ssd, uint8_t base_sharp, uint8_t* level_out,
                               uint8_t* sharp_out) {
  uint8_t bs = base_sharp > 7 ? 7 : base_sharp;
  uint8_t best_level = 0;
  uint64_t best = ssd[0 * 8 + bs];
  for (int l = 4; l <= 60; l += 4)
    if (ssd[l * 8 + bs] < best) {
      best = ssd[l * 8 + bs];
      best_level = (uint8_t)l;
    }
  if (ssd[63 * 8 + bs] < best) {
    best = ssd[63 * 8 + bs];
    best_level = 63;
  }
  int lo = best_level >= 3 ? best_level - 3 : 0;
  int hi = best_level + 3 > 63 ? 63 : best_level + 3;
  uint8_t center = best_level;
  for (int l = lo; l <= hi; l++) {
    if (l == center) continue;
    if (ssd[l * 8 + bs] < best) {
      best = ssd[l * 8 + bs];
      best_level = (uint8_t)l;
    }
  }
  if (best_level == 0) {
    *level_out = 0;
    *sharp_out = bs;
    return;
  }
  uint8_t best_sharp = bs;
  for (int s = 0; s < 8; s++) {
    if (s == bs) continue;
    if (ssd[best_level * 8 + s] < best) {
      best = ssd[best_level * 8 + s];
      best_sharp = (uint8_t)s;
    }
  }
  *level_out = best_level;
  *sharp_out = best_sharp;
}

/* select_filter_params_sampled's coarse-to-fine walk
 * (src/loop_filter.rs:2377-2411) over a table of band scores. */
void vo_select_from_table_sampled(const uint64_t* ssd, uint8_t base_sharp, int sweep,
                                  uint8_t* level_out, uint8_t* sharp_out) {
  uint8_t bs = base_sharp > 7 ? 7 : base_sharp;
  static const uint8_t coarse[9] = {0, 8, 16, 24, 32, 40, 48, 56, 63};
  uint8_t best_level = 0;
  uint64_t best = ssd[0 * 8 + bs];
  for (int i = 1; i < 9; i++)
    if (ssd[coarse[i] * 8 + bs] < best) {
      best = ssd[coarse[i] * 8 + bs];
      best_level = coarse[i];
    }
  static const uint8_t steps[3] = {4, 2, 1};
  for (int si = 0; si < 3; si++) {
    uint8_t st = steps[si];
    uint8_t around[2];
    int na = 0;
    if (best_level >= st) around[na++] = (uint8_t)(best_level - st);
    if (best_level + st <= 63) around[na++] = (uint8_t)(best_level + st);
    for (int k = 0; k < na; k++)
      if (ssd[around[k] * 8 + bs] < best) {
        best = ssd[around[k] * 8 + bs];
        best_level = around[k];
      }
  }
  uint8_t best_sharp = bs;
  if (sweep && best_level != 0)
    for (int s = 0; s < 8; s++) {
      if (s == bs) continue;
      if (ssd[best_level * 8 + s] < best) {
        best = ssd[best_level * 8 + s];
        best_sharp = (uint8_t)s;
      }
    }
  *level_out = best_level;
  *sharp_out = best_sharp;
}

/* The reference scores only the candidates its walk visits; scoring the
 * whole table first and walking it gives the same choice. The oracle
 * follows the reference literally instead: it scores exactly the visited
 * candidates, stage by stage. */
void vo_select_filter_params(const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                             const vp8a_filter_config* base, const vp8a_source* src,
                             uint8_t* level_out, uint8_t* sharp_out, uint32_t threads) {
  uint8_t bs = base->sharpness_level > 7 ? 7 : base->sharpness_level;
  uint64_t* t = (uint64_t*)calloc(512, sizeof(uint64_t));
  uint8_t cands[32][2];
  uint32_t n = 0;
  for (int l = 0; l <= 63; l += 4) { cands[n][0] = (uint8_t)l; cands[n][1] = bs; n++; }
  cands[n][0] = 63; cands[n][1] = bs; n++;
  score_list(planes, mbs, base, src, 0, (const uint8_t(*)[2])cands, n, t, threads);
  uint8_t best_level = 0;
  uint64_t best = t[0 * 8 + bs];
  for (uint32_t i = 1; i < n; i++)
    if (t[cands[i][0] * 8 + bs] < best) { best = t[cands[i][0] * 8 + bs]; best_level = cands[i][0]; }
  int lo = best_level >= 3 ? best_level - 3 : 0, hi = best_level + 3 > 63 ? 63 : best_level + 3;
  n = 0;
  for (int l = lo; l <= hi; l++)
    if (l != best_level) { cands[n][0] = (uint8_t)l; cands[n][1] = bs; n++; }
  score_list(planes, mbs, base, src, 0, (const uint8_t(*)[2])cands, n, t, threads);
  uint8_t center = best_level;
  (void)center;
  for (uint32_t i = 0; i < n; i++)
    if (t[cands[i][0] * 8 + bs] < best) { best = t[cands[i][0] * 8 + bs]; best_level = cands[i][0]; }
  if (best_level == 0) {
    *level_out = 0;
    *sharp_out = bs;
    free(t);
    return;
  }
  n = 0;
  for (int s = 0; s < 8; s++)
    if (s != bs) { cands[n][0] = best_level; cands[n][1] = (uint8_t)s; n++; }
  score_list(planes, mbs, base, src, 0, (const uint8_t(*)[2])cands, n, t, threads);
  uint8_t best_sharp = bs;
  for (uint32_t i = 0; i < n; i++)
    if (t[best_level * 8 + cands[i][1]] < best) {
      best = t[best_level * 8 + cands[i][1]];
      best_sharp = cands[i][1];
    }
  *level_out = best_level;
  *sharp_out = best_sharp;
  free(t);
}

void vo_select_filter_params_sampled(const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                                     const vp8a_filter_config* base, const vp8a_source* src,
                                     uint32_t every_rows, uint32_t sweep_sharpness,
                                     uint8_t* level_out, uint8_t* sharp_out, uint32_t threads) {
  uint8_t bs = base->sharpness_level > 7 ? 7 : base->sharpness_level;
  uint32_t er = every_rows < 2 ? 2 : every_rows;
  uint64_t* t = (uint64_t*)calloc(512, sizeof(uint64_t));
  static const uint8_t coarse[9] = {0, 8, 16, 24, 32, 40, 48, 56, 63};
  uint8_t cands[16][2];
  uint32_t n = 0;
  for (int i = 0; i < 9; i++) { cands[n][0] = coarse[i]; cands[n][1] = bs; n++; }
  score_list(planes, mbs, base, src, er, (const uint8_t(*)[2])cands, n, t, threads);
  uint8_t best_level = 0;
  uint64_t best = t[0 * 8 + bs];
  for (int i = 1; i < 9; i++)
    if (t[coarse[i] * 8 + bs] < best) { best = t[coarse[i] * 8 + bs]; best_level = coarse[i]; }
  static const uint8_t steps[3] = {4, 2, 1};
  for (int si = 0; si < 3; si++) {
    uint8_t st = steps[si];
    n = 0;
    if (best_level >= st) { cands[n][0] = (uint8_t)(best_level - st); cands[n][1] = bs; n++; }
    if (best_level + st <= 63) { cands[n][0] = (uint8_t)(best_level + st); cands[n][1] = bs; n++; }
    score_list(planes, mbs, base, src, er, (const uint8_t(*)[2])cands, n, t, threads);
    uint8_t bl = best_level;
    for (uint32_t k = 0; k < n; k++)
      if (t[cands[k][0] * 8 + bs] < best) { best = t[cands[k][0] * 8 + bs]; bl = cands[k][0]; }
    best_level = bl;
  }
  uint8_t best_sharp = bs;
  if (sweep_sharpness && best_level != 0) {
    n = 0;
    for (int s = 0; s < 8; s++)
      if (s != bs) { cands[n][0] = best_level; cands[n][1] = (uint8_t)s; n++; }
    score_list(planes, mbs, base, src, er, (const uint8_t(*)[2])cands, n, t, threads);
    for (uint32_t k = 0; k < n; k++)
      if (t[best_level * 8 + cands[k][1]] < best) {
        best = t[best_level * 8 + cands[k][1]];
        best_sharp = cands[k][1];
      }
  }
  *level_out = best_level;
  *sharp_out = best_sharp;
  free(t);
}
