/*
 * rd_search.c — oracle restatement of the RD-effort inter search.
 *
 * TEST INFRASTRUCTURE ONLY (see vp8a_oracle.h). Follows
 * src/encoder/inter_search.rs:
 *   SearchShape per effort                 :62-162
 *   MvCostTable (f32 component bits)       :166-194
 *   whole_sad (early exit, clamped path)   :224-254
 *   fetch_window / HalfPlanes              :259-346
 *   whole_pixel_search (seeds, WIDE/NARROW):380-495
 *   sub_pixel_refine                       :499-552
 *   decide_mb_rd, search part              :846-1060
 * The early exits never change a result (a candidate that exits is
 * rejected either way), so SADs are evaluated in full here.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vp8a_oracle.h"

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int mv_eq(vp8a_mv a, vp8a_mv b) { return a.row == b.row && a.col == b.col; }
#define BB(p, v) vo_bool_bits((uint8_t)(p), (v))

typedef struct {
  uint32_t descent_rounds;
  int wide_pattern, half_diagonals, quarter, search_other_refs, refine_runner_up;
  uint64_t split_gate;
} shape_t;

/* EncodeEffort::inter_shape (src/encoder/inter_search.rs:93-161), the
 * fields the inter search reads. */
static shape_t shape_for(uint32_t effort) {
  shape_t s;
  switch (effort) {
    case VP8A_EFFORT_FASTEST: s = (shape_t){4, 0, 1, 0, 0, 0, UINT64_MAX}; break;
    case VP8A_EFFORT_FAST: s = (shape_t){8, 1, 1, 1, 1, 0, UINT64_MAX}; break;
    case VP8A_EFFORT_BALANCED: s = (shape_t){16, 1, 1, 1, 1, 1, 4}; break;
    default: s = (shape_t){32, 1, 1, 1, 1, 1, 0}; break;
  }
  return s;
}

typedef struct {
  float bits[2][2047];
} cost_table;

/* MvCostTable::new (:172-182): mv_component_bits as f32. */
static void cost_table_init(cost_table* t, const vp8a_mv_contexts* c) {
  for (int k = 0; k < 2; k++)
    for (int d = -1023; d <= 1023; d++) t->bits[k][d + 1023] = (float)vo_mv_component_bits(c->p[k], d);
}

/* MvCostTable::bits (:185-193): f32 sum, widened. Returns 0 when the
 * differential is out of range (the reference's None). */
static int cost_bits(const cost_table* t, vp8a_mv mv, vp8a_mv base, double* out) {
  int dr = mv.row - base.row, dc = mv.col - base.col;
  if (dr < -1023 || dr > 1023 || dc < -1023 || dc > 1023) return 0;
  float s = t->bits[0][dr + 1023] + t->bits[1][dc + 1023];
  *out = (double)s;
  return 1;
}

/* whole_sad (:224-254) evaluated in full: clamped 16x16 at pixel (x, y). */
static uint32_t whole_sad(const vp8a_luma_ref* r, int x, int y, const uint8_t* src) {
  int w = (int)r->width, h = (int)r->height;
  uint32_t acc = 0;
  for (int rr = 0; rr < 16; rr++) {
    int sy = clampi(y + rr, 0, h - 1);
    for (int c = 0; c < 16; c++) {
      int sx = clampi(x + c, 0, w - 1);
      int d = (int)src[rr * 16 + c] - (int)r->plane[(size_t)sy * r->stride + sx];
      acc += (uint32_t)(d < 0 ? -d : d);
    }
  }
  return acc;
}

typedef struct {
  vp8a_mv mv;
  uint32_t sad;
  double cost;
} found_t;

typedef struct {
  vp8a_mv best, nearest, near_;
  double mode_bits[5];
  int range_x0, range_x1, range_y0, range_y1;
} census_t;

/* whole_pixel_search (:380-495). */
static found_t whole_pixel_search(const vp8a_luma_ref* L, const census_t* cs, const uint8_t* src,
                                  int ox, int oy, const vp8a_mv* seeds, int nseeds,
                                  const cost_table* costs, double lambda_sad, uint32_t good_enough,
                                  const shape_t* shape, int descend) {
  found_t best = {{0, 0}, UINT32_MAX, INFINITY};
#define EVAL(PX, PY)                                                          \
  do {                                                                        \
    vp8a_mv mv_ = {(int16_t)((PY) * 4), (int16_t)((PX) * 4)};                 \
    double bits_;                                                             \
    if (cost_bits(costs, mv_, cs->best, &bits_)) {                            \
      double rate_ = lambda_sad * bits_;                                      \
      if (!(rate_ >= best.cost)) {                                            \
        uint32_t sad_ = whole_sad(L, ox + (PX), oy + (PY), src);              \
        double cost_ = (double)sad_ + rate_;                                  \
        if (cost_ < best.cost) {                                              \
          best.mv = mv_;                                                      \
          best.sad = sad_;                                                    \
          best.cost = cost_;                                                  \
          improved = 1;                                                       \
        }                                                                     \
      }                                                                       \
    }                                                                         \
  } while (0)
  int tried[8][2];
  int ntried = 0;
  int improved = 0;
  for (int s = 0; s < nseeds; s++) {
    int px = clampi((seeds[s].col + 2) >> 2, cs->range_x0, cs->range_x1);
    int py = clampi((seeds[s].row + 2) >> 2, cs->range_y0, cs->range_y1);
    int dup = 0;
    for (int k = 0; k < ntried; k++)
      if (tried[k][0] == px && tried[k][1] == py) dup = 1;
    if (dup) continue;
    if (ntried < 8) {
      tried[ntried][0] = px;
      tried[ntried][1] = py;
      ntried++;
    }
    EVAL(px, py);
  }
  if (!descend || best.sad <= good_enough) return best;
  static const int WIDE[8][2] = {{-2, 0}, {2, 0}, {0, -2}, {0, 2}, {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};
  static const int NARROW[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
  if (shape->wide_pattern && (uint64_t)best.sad > 4ull * good_enough) {
    for (uint32_t it = 0; it < shape->descent_rounds; it++) {
      int cx = best.mv.col / 4, cy = best.mv.row / 4;
      improved = 0;
      for (int k = 0; k < 8; k++) {
        int px = cx + WIDE[k][0], py = cy + WIDE[k][1];
        if (px >= cs->range_x0 && px <= cs->range_x1 && py >= cs->range_y0 && py <= cs->range_y1)
          EVAL(px, py);
      }
      if (!improved || best.sad <= good_enough) break;
    }
  }
  for (uint32_t it = 0; it < shape->descent_rounds; it++) {
    if (best.sad <= good_enough) break;
    int cx = best.mv.col / 4, cy = best.mv.row / 4;
    improved = 0;
    for (int k = 0; k < 4; k++) {
      int px = cx + NARROW[k][0], py = cy + NARROW[k][1];
      if (px >= cs->range_x0 && px <= cs->range_x1 && py >= cs->range_y0 && py <= cs->range_y1)
        EVAL(px, py);
    }
    if (!improved) break;
  }
#undef EVAL
  return best;
}

/* Six-tap half-pel run (interp with filters[4], src/motion_comp.rs:396). */
static uint8_t half_tap(const uint8_t* s, size_t step) {
  static const int f[6] = {3, -16, 77, 77, -16, 3};
  int a = 0;
  for (int i = 0; i < 6; i++) a += (int)s[i * step] * f[i];
  return (uint8_t)clampi((a + 64) >> 7, 0, 255);
}

/* sub_pixel_refine (:499-552) with fetch_window + HalfPlanes (:259-346). */
static found_t sub_pixel_refine(const vp8a_luma_ref* L, const census_t* cs, const uint8_t* src,
                                int ox, int oy, int mb_col, int mb_row, found_t start,
                                const cost_table* costs, double lambda_sad, const shape_t* shape) {
  enum { WIN = 22, HP = 17 };
  int px = start.mv.col / 4, py = start.mv.row / 4;
  int x0 = ox + px - 3, y0 = oy + py - 3;
  uint8_t win[WIN * WIN];
  for (int r = 0; r < WIN; r++) {
    int sy = clampi(y0 + r, 0, (int)L->height - 1);
    for (int c = 0; c < WIN; c++) win[r * WIN + c] = L->plane[(size_t)sy * L->stride + clampi(x0 + c, 0, (int)L->width - 1)];
  }
  uint8_t hp[WIN * HP], vp[HP * 16], dp[HP * HP];
  memset(hp, 0, sizeof hp);
  for (int r = shape->half_diagonals ? 0 : 3; r < (shape->half_diagonals ? WIN : 19); r++)
    for (int i = 0; i < HP; i++) hp[r * HP + i] = half_tap(win + r * WIN + i, 1);
  for (int r = 0; r < HP; r++)
    for (int i = 0; i < 16; i++) vp[r * 16 + i] = half_tap(win + r * WIN + 3 + i, WIN);
  if (shape->half_diagonals)
    for (int r = 0; r < HP; r++)
      for (int i = 0; i < HP; i++) dp[r * HP + i] = half_tap(hp + r * HP + i, HP);
  found_t best = start;
  for (int dy = -1; dy <= 1; dy++)
    for (int dx = -1; dx <= 1; dx++) {
      if ((dx == 0 && dy == 0) || (!shape->half_diagonals && dx != 0 && dy != 0)) continue;
      vp8a_mv mv = {(int16_t)(start.mv.row + 2 * dy), (int16_t)(start.mv.col + 2 * dx)};
      if (abs(mv.row) > 1020 || abs(mv.col) > 1020) continue;
      int cx = dx > 0, cy = dy > 0;
      const uint8_t* plane;
      int stride, off;
      if (dy == 0) {
        plane = hp, stride = HP, off = 3 * HP + cx;
      } else if (dx == 0) {
        plane = vp, stride = 16, off = cy * 16;
      } else {
        plane = dp, stride = HP, off = cy * HP + cx;
      }
      uint32_t sad = 0;
      for (int r = 0; r < 16; r++)
        for (int c = 0; c < 16; c++) {
          int d = (int)src[r * 16 + c] - (int)plane[off + r * stride + c];
          sad += (uint32_t)(d < 0 ? -d : d);
        }
      double bits;
      if (cost_bits(costs, mv, cs->best, &bits)) {
        double cost = (double)sad + lambda_sad * bits;
        if (cost < best.cost) best = (found_t){mv, sad, cost};
      }
    }
  if (shape->quarter) {
    vp8a_mv centre = best.mv;
    static const int Q[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
    for (int k = 0; k < 4; k++) {
      vp8a_mv mv = {(int16_t)(centre.row + Q[k][1]), (int16_t)(centre.col + Q[k][0])};
      if (abs(mv.row) > 1022 || abs(mv.col) > 1022) continue;
      uint32_t sad = vo_mb_luma_sad_at_mv(L, mb_col, mb_row, src, mv);
      double bits;
      if (cost_bits(costs, mv, cs->best, &bits)) {
        double cost = (double)sad + lambda_sad * bits;
        if (cost < best.cost) best = (found_t){mv, sad, cost};
      }
    }
  }
  return best;
}

static double ref_tree_bits(uint8_t ref) {
  if (ref == VP8A_REF_LAST) return BB(128, 0);
  if (ref == VP8A_REF_GOLDEN) return BB(128, 1) + BB(128, 0);
  return BB(128, 1) + BB(128, 1);
}

typedef struct {
  const vp8a_i420* frame;
  const vp8a_planes* refs;
  const uint8_t* ref_ids;
  uint32_t n_refs;
  const cost_table* costs;
  double lambda;
  uint32_t y1_ac;
  shape_t shape;
  const vp8a_mb_info* nb;
  vp8a_rd_inter* out;
  int mb_cols, mb_rows;
} rd_job;

/* decide_mb_rd's search part for one MB (:846-1060). */
static void rd_mb(void* arg, uint32_t idx) {
  rd_job* j = (rd_job*)arg;
  int mb_row = (int)idx / j->mb_cols, mb_col = (int)idx % j->mb_cols;
  const vp8a_mb_info *above = &j->nb[3 * idx], *left = &j->nb[3 * idx + 1], *al = &j->nb[3 * idx + 2];
  uint8_t src[256];
  vo_extract_mb_luma(j->frame, mb_row, mb_col, src);
  const double lambda_sad = sqrt(j->lambda);
  uint32_t qpix = j->y1_ac / 8;
  if (qpix < 1) qpix = 1;
  const uint32_t good_enough = 256 * qpix / 2;
  const int ox = mb_col * 16, oy = mb_row * 16;
  int to_left = -((mb_col + 1) << 6), to_right = (j->mb_cols - mb_col) << 6;
  int to_top = -((mb_row + 1) << 6), to_bottom = (j->mb_rows - mb_row) << 6;
  census_t cs[3];
  found_t found[3];
  double total[3];
  int have[3] = {0, 0, 0};
  int leader = 0;
  double leader_cost = INFINITY;
  vp8a_rd_inter* o = &j->out[idx];
  memset(o, 0, sizeof *o);
  for (int k = 0; k < 3; k++) o->found[k] = (vp8a_search_result){{0, 0}, UINT32_MAX};
  for (uint32_t n = 0; n < j->n_refs; n++) {
    vp8a_mv near[3];
    int32_t cnt[4];
    vo_find_near_mvs(above, left, al, j->ref_ids[n], near, cnt);
    uint8_t p[4];
    vo_mv_ref_probs(cnt, p);
    census_t* c = &cs[n];
    c->best = vo_clamp_mv_rect(near[0], mb_col, mb_row, j->mb_cols, j->mb_rows);
    c->nearest = vo_clamp_mv_rect(near[1], mb_col, mb_row, j->mb_cols, j->mb_rows);
    c->near_ = vo_clamp_mv_rect(near[2], mb_col, mb_row, j->mb_cols, j->mb_rows);
    /* The `tree` closure (:905-914): `ones` true bits then an optional last. */
    for (int m = 0; m < 5; m++) {
      double bits = 0.0;
      for (int q = 0; q < m; q++) bits += BB(p[q], 1);
      if (m < 4) bits += BB(p[m], 0);
      c->mode_bits[m] = bits;
    }
    c->range_x0 = (to_left / 4) < -255 ? -255 : to_left / 4;
    c->range_x1 = (to_right / 4) > 255 ? 255 : to_right / 4;
    c->range_y0 = (to_top / 4) < -255 ? -255 : to_top / 4;
    c->range_y1 = (to_bottom / 4) > 255 ? 255 : to_bottom / 4;
    vp8a_mv seeds[6];
    int len = 0;
    seeds[len++] = (vp8a_mv){0, 0};
    seeds[len++] = c->nearest;
    seeds[len++] = c->near_;
    seeds[len++] = c->best;
    if (left->ref_frame == j->ref_ids[n]) seeds[len++] = left->mv;
    if (above->ref_frame == j->ref_ids[n]) seeds[len++] = above->mv;
    vp8a_luma_ref L = {j->refs[n].y, j->refs[n].y_stride, j->refs[n].mb_cols * 16, j->refs[n].mb_rows * 16};
    int descend = n == 0 || j->shape.search_other_refs;
    found[n] = whole_pixel_search(&L, c, src, ox, oy, seeds, len, j->costs, lambda_sad, good_enough, &j->shape,
                                  descend);
    total[n] = found[n].cost + lambda_sad * ref_tree_bits(j->ref_ids[n]);
    if (total[n] < leader_cost) {
      leader_cost = total[n];
      leader = (int)n;
    }
    have[n] = 1;
    o->found[n].mv = found[n].mv;
    o->found[n].sad = found[n].sad;
    o->n_searched = (uint8_t)(n + 1);
    if (found[n].sad <= good_enough) break;
  }
  int have_best = 0;
  double best_cost = 0;
  for (uint32_t n = 0; n < j->n_refs; n++) {
    if (!have[n]) continue;
    int refine = (int)n == leader ||
                 (j->shape.refine_runner_up && (j->shape.split_gate == 0 || total[n] < leader_cost * 1.125));
    if (!refine) continue;
    census_t* c = &cs[n];
    double ref_bits = ref_tree_bits(j->ref_ids[n]);
    vp8a_luma_ref L = {j->refs[n].y, j->refs[n].y_stride, j->refs[n].mb_cols * 16, j->refs[n].mb_rows * 16};
    found_t f = found[n];
    if (f.sad > good_enough / 2)
      f = sub_pixel_refine(&L, c, src, ox, oy, mb_col, mb_row, f, j->costs, lambda_sad, &j->shape);
    const vp8a_mv zero = {0, 0};
    int mode;
    double mode_bits;
    if (mv_eq(f.mv, zero)) {
      mode = VP8A_MODE_ZERO;
      mode_bits = c->mode_bits[0];
    } else if (mv_eq(f.mv, c->nearest)) {
      mode = VP8A_MODE_NEAREST;
      mode_bits = c->mode_bits[1];
    } else if (mv_eq(f.mv, c->near_)) {
      mode = VP8A_MODE_NEAR;
      mode_bits = c->mode_bits[2];
    } else {
      double diff = 0.0;
      cost_bits(j->costs, f.mv, c->best, &diff);
      mode = VP8A_MODE_NEW;
      mode_bits = c->mode_bits[3] + diff;
    }
#define CONSIDER(MODE, MV, SAD, BITS)                          \
  do {                                                         \
    double bits_ = (BITS);                                     \
    double cost_ = (double)(SAD) + lambda_sad * bits_;         \
    if (!have_best || cost_ < best_cost) {                     \
      have_best = 1;                                           \
      best_cost = cost_;                                       \
      o->ref_frame = j->ref_ids[n];                            \
      o->mode = (uint8_t)(MODE);                               \
      o->mv = (MV);                                            \
      o->sad = (SAD);                                          \
      o->cost = cost_;                                         \
      o->bits = bits_;                                         \
    }                                                          \
  } while (0)
    CONSIDER(mode, f.mv, f.sad, ref_bits + mode_bits);
    const vp8a_mv fm[3] = {zero, c->nearest, c->near_};
    const int fmode[3] = {VP8A_MODE_ZERO, VP8A_MODE_NEAREST, VP8A_MODE_NEAR};
    for (int k = 0; k < 3; k++) {
      if (k == 1 && mv_eq(c->nearest, zero)) continue;
      if (k == 2 && (mv_eq(c->near_, zero) || mv_eq(c->near_, c->nearest))) continue;
      vp8a_mv mv = fm[k];
      if (mv_eq(mv, f.mv)) continue;
      uint32_t sad = (mv.row % 4 == 0 && mv.col % 4 == 0)
                         ? whole_sad(&L, ox + mv.col / 4, oy + mv.row / 4, src)
                         : vo_mb_luma_sad_at_mv(&L, mb_col, mb_row, src, mv);
      CONSIDER(fmode[k], mv, sad, ref_bits + c->mode_bits[k]);
    }
#undef CONSIDER
  }
  o->leader = (uint8_t)leader;
}

int vo_rd_inter_search(const vp8a_i420* frame, const vp8a_planes* refs, const uint8_t* ref_ids,
                       uint32_t n_refs, const vp8a_mv_contexts* mv_contexts, double lambda,
                       uint32_t y1_ac, uint32_t effort, const vp8a_mb_info* neighbours,
                       vp8a_rd_inter* out, uint32_t threads) {
  if (!frame || !refs || !ref_ids || !neighbours || !out || n_refs == 0 || n_refs > 3)
    return VP8A_E_INVALID_ARGUMENT;
  if (frame->width == 0 || frame->height == 0 || frame->width > 0x3FFF || frame->height > 0x3FFF)
    return VP8A_E_INVALID_DIMENSIONS;
  int mb_cols = (int)((frame->width + 15) / 16), mb_rows = (int)((frame->height + 15) / 16);
  for (uint32_t k = 0; k < n_refs; k++)
    if ((int)refs[k].mb_cols != mb_cols || (int)refs[k].mb_rows != mb_rows)
      return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
  vp8a_mv_contexts defctx;
  if (!mv_contexts) {
    vo_default_mv_contexts(&defctx);
    mv_contexts = &defctx;
  }
  cost_table* costs = (cost_table*)malloc(sizeof(cost_table));
  if (!costs) return VP8A_E_OUT_OF_MEMORY;
  cost_table_init(costs, mv_contexts);
  rd_job j = {frame, refs, ref_ids, n_refs, costs, lambda, y1_ac, shape_for(effort), neighbours, out,
              mb_cols, mb_rows};
  vo_parallel_for((uint32_t)(mb_cols * mb_rows), threads, rd_mb, &j);
  free(costs);
  return VP8A_OK;
}
