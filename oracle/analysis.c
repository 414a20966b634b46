/*
 * analysis.c — oracle restatement of the exhaustive inter analysis.
 *
 * TEST INFRASTRUCTURE ONLY (see vp8a_oracle.h). Follows:
 *   bool_bits + its -log2 table        src/encoder.rs:2229-2260
 *   rd_lambda                          src/encoder.rs:3742
 *   mv_component_bits                  src/motion_vector.rs:345
 *   find_near_mvs, MvClampRect,
 *   clamp_mv, mv_ref_probs             src/near_mv.rs:236-404
 *   left/above_block_mv,
 *   submv_ref_context, tables          src/near_mv.rs:539-760
 *   SPLITMV group search + scoring     src/encoder.rs:7573-8246
 *   pick_mb_for_ref (search part)      src/encoder.rs:8516-8702
 *   decide_mb_exhaustive               src/encoder/inter.rs:537-620
 *   analyse_inter_frame / analyse_row  src/encoder/inter.rs:263-513
 * RD costs are f64 in the reference's exact operation order; this file is
 * built with -ffp-contract=off so no fused multiply-add changes a result.
 */
#include <math.h>
#include <sched.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

#include "vp8a_oracle.h"

#define MV_MIN (-1023)
#define MV_MAX 1023

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int mv_eq(vp8a_mv a, vp8a_mv b) { return a.row == b.row && a.col == b.col; }
static inline int mv_zero(vp8a_mv a) { return a.row == 0 && a.col == 0; }
static const vp8a_mv MV0 = {0, 0};

/* ---------------------------------------------------------------- bit costs */

static double g_bit_cost[256];
static atomic_int g_bit_cost_ready;

static void init_bit_cost(void) {
  if (atomic_load(&g_bit_cost_ready)) return;
  double t[256];
  t[0] = -log2(1.0 / 256.0);
  for (int p = 1; p < 256; p++) t[p] = -log2((double)p / 256.0);
  memcpy(g_bit_cost, t, sizeof t);
  atomic_store(&g_bit_cost_ready, 1);
}

/* bool_bits (src/encoder.rs:2229). */
double vo_bool_bits(uint8_t prob, int value) {
  init_bit_cost();
  if (value) {
    int idx = 256 - (int)prob;
    return g_bit_cost[idx > 255 ? 255 : idx];
  }
  return g_bit_cost[prob];
}
#define BB(p, v) vo_bool_bits((uint8_t)(p), (v))

/* rd_lambda (src/encoder.rs:3742) over AC_QLOOKUP
 * (src/inverse_transform.rs:87, RFC 6386 §14.1 ac_qlookup). */
static const int16_t AC_QLOOKUP[128] = {
    4,   5,   6,   7,   8,   9,   10,  11,  12,  13,  14,  15,  16,  17,  18,  19,
    20,  21,  22,  23,  24,  25,  26,  27,  28,  29,  30,  31,  32,  33,  34,  35,
    36,  37,  38,  39,  40,  41,  42,  43,  44,  45,  46,  47,  48,  49,  50,  51,
    52,  53,  54,  55,  56,  57,  58,  60,  62,  64,  66,  68,  70,  72,  74,  76,
    78,  80,  82,  84,  86,  88,  90,  92,  94,  96,  98,  100, 102, 104, 106, 108,
    110, 112, 114, 116, 119, 122, 125, 128, 131, 134, 137, 140, 143, 146, 149, 152,
    155, 158, 161, 164, 167, 170, 173, 177, 181, 185, 189, 193, 197, 201, 205, 209,
    213, 217, 221, 225, 229, 234, 239, 245, 249, 254, 259, 264, 269, 274, 279, 284};

double vo_rd_lambda(uint32_t qi) {
  double q = (double)AC_QLOOKUP[qi > 127 ? 127 : qi];
  return q * q / 32.0;
}

/* DEFAULT_MV_CONTEXT (src/coded_header.rs:957, RFC 6386 §17.2). */
void vo_default_mv_contexts(vp8a_mv_contexts* out) {
  static const uint8_t d[2][19] = {
      {162, 128, 225, 146, 172, 147, 214, 39, 156, 128, 129, 132, 75, 145, 178, 206, 239, 254,
       254},
      {164, 128, 204, 170, 119, 235, 140, 230, 228, 128, 130, 130, 74, 148, 180, 203, 236, 254,
       254}};
  memcpy(out->p, d, sizeof d);
}

/* SMALL_MVTREE (src/motion_vector.rs:108). */
static const int8_t SMALL_MVTREE[14] = {2, 8, 4, 6, -0, -1, -2, -3, 10, 12, -4, -5, -6, -7};
enum { MVP_IS_SHORT = 0, MVP_SIGN = 1, MVP_SHORT = 2, MVP_BITS = 9 };

/* mv_component_bits (src/motion_vector.rs:345), same summation order. */
double vo_mv_component_bits(const uint8_t* p, int32_t value) {
  int32_t a = value < 0 ? -value : value;
  double bits = 0.0;
  if (a > 7) {
    bits += BB(p[MVP_IS_SHORT], 1);
    for (int i = 0; i < 3; i++) bits += BB(p[MVP_BITS + i], (a >> i) & 1);
    int i = 9;
    for (;;) {
      bits += BB(p[MVP_BITS + i], (a >> i) & 1);
      i -= 1;
      if (i <= 3) break;
    }
    if ((a & 0xfff0) != 0) bits += BB(p[MVP_BITS + 3], (a >> 3) & 1);
  } else {
    bits += BB(p[MVP_IS_SHORT], 0);
    /* small_mv_bits: a separate running sum, then added. */
    double s = 0.0;
    int i = 0;
    for (int k = 2; k >= 0; k--) {
      int bit = (a >> k) & 1;
      s += BB(p[MVP_SHORT + (i >> 1)], bit);
      int next = SMALL_MVTREE[i + bit];
      if (next <= 0) break;
      i = next;
    }
    bits += s;
  }
  if (a != 0) bits += BB(p[MVP_SIGN], value < 0);
  return bits;
}

/* ------------------------------------------------------------------ census */

/* MV_COUNTS_TO_PROBS (src/near_mv.rs, RFC 6386 §16.3 vp8_mode_contexts). */
static const uint8_t MV_COUNTS_TO_PROBS[6][4] = {{7, 1, 1, 143},    {14, 18, 14, 107},
                                                 {135, 64, 57, 68}, {60, 56, 128, 65},
                                                 {159, 134, 128, 34}, {234, 188, 128, 28}};

/* find_near_mvs (src/near_mv.rs:310-402) with the default SignBias (no
 * sign flips), as pick_mb_for_ref calls it (src/encoder.rs:8556-8562). */
void vo_find_near_mvs(const vo_mb_info* above, const vo_mb_info* left,
                      const vo_mb_info* aboveleft, uint8_t current_ref, vp8a_mv mvs_out[3],
                      int32_t cnt_out[4]) {
  (void)current_ref;
  vp8a_mv near_mvs[4] = {MV0, MV0, MV0, MV0};
  int32_t cnt[4] = {0, 0, 0, 0};
  int mv_idx = 0, cnt_idx = 0;
  if (above->ref_frame != VP8A_REF_INTRA) {
    if (!mv_zero(above->mv)) {
      mv_idx++;
      near_mvs[mv_idx] = above->mv;
      cnt_idx++;
    }
    cnt[cnt_idx] += 2;
  }
  if (left->ref_frame != VP8A_REF_INTRA) {
    if (!mv_zero(left->mv)) {
      vp8a_mv m = left->mv;
      if (!mv_eq(m, near_mvs[mv_idx])) {
        mv_idx++;
        near_mvs[mv_idx] = m;
        cnt_idx++;
      }
      cnt[cnt_idx] += 2;
    } else {
      cnt[0] += 2;
    }
  }
  if (aboveleft->ref_frame != VP8A_REF_INTRA) {
    if (!mv_zero(aboveleft->mv)) {
      vp8a_mv m = aboveleft->mv;
      if (!mv_eq(m, near_mvs[mv_idx])) {
        mv_idx++;
        near_mvs[mv_idx] = m;
        cnt_idx++;
      }
      cnt[cnt_idx] += 1;
    } else {
      cnt[0] += 1;
    }
  }
  if (cnt[3] != 0 && mv_eq(near_mvs[mv_idx], near_mvs[1])) cnt[1] += 1;
  cnt[3] = (above->is_split + left->is_split) * 2 + aboveleft->is_split;
  if (cnt[2] > cnt[1]) {
    int32_t t = cnt[1];
    cnt[1] = cnt[2];
    cnt[2] = t;
    vp8a_mv tm = near_mvs[1];
    near_mvs[1] = near_mvs[2];
    near_mvs[2] = tm;
  }
  if (cnt[1] >= cnt[0]) near_mvs[0] = near_mvs[1];
  mvs_out[0] = near_mvs[0];
  mvs_out[1] = near_mvs[1];
  mvs_out[2] = near_mvs[2];
  memcpy(cnt_out, cnt, sizeof cnt);
}

/* MvClampRect::for_mb + clamp_mv (src/near_mv.rs:236-283). */
static vp8a_mv clamp_mv_rect(vp8a_mv mv, int mb_col, int mb_row, int mb_cols, int mb_rows) {
  int to_left = -((mb_col + 1) << 6), to_right = (mb_cols - mb_col) << 6;
  int to_top = -((mb_row + 1) << 6), to_bottom = (mb_rows - mb_row) << 6;
  vp8a_mv o;
  o.col = (int16_t)clampi(mv.col, to_left, to_right);
  o.row = (int16_t)clampi(mv.row, to_top, to_bottom);
  return o;
}

/* mv_ref_probs (src/near_mv.rs:404). */
void vo_mv_ref_probs(const int32_t cnt[4], uint8_t out[4]) {
  for (int i = 0; i < 4; i++) out[i] = MV_COUNTS_TO_PROBS[cnt[i]][i];
}

vp8a_mv vo_clamp_mv_rect(vp8a_mv mv, int mb_col, int mb_row, int mb_cols, int mb_rows) {
  return clamp_mv_rect(mv, mb_col, mb_row, mb_cols, mb_rows);
}

/* ------------------------------------------------------------------ SPLITMV */

/* MV_PARTITIONS (src/near_mv.rs, RFC 6386 §20.13 mbsplits). */
static const uint8_t MV_PARTITIONS[4][16] = {
    {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1},
    {0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1},
    {0, 0, 1, 1, 0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 3, 3},
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}};
static const uint8_t MV_PARTITION_PROBS[3] = {110, 111, 150};
static const uint8_t SUBMV_REF_PROBS[5][3] = {
    {147, 136, 18}, {106, 145, 1}, {179, 121, 1}, {223, 1, 34}, {208, 1, 1}};

typedef struct {
  int members[16][16];
  int len[16];
  int row0[16], col0[16], w[16], h[16];
  int num_groups;
} part_groups;

/* PartitionGroups::build (src/encoder.rs:7912-7980). */
static void build_groups(int pid, part_groups* g) {
  memset(g, 0, sizeof *g);
  for (int idx = 0; idx < 16; idx++) {
    int gid = MV_PARTITIONS[pid][idx];
    g->members[gid][g->len[gid]++] = idx;
    if (gid + 1 > g->num_groups) g->num_groups = gid + 1;
  }
  for (int k = 0; k < g->num_groups; k++) {
    int min_r = 3, max_r = 0, min_c = 3, max_c = 0;
    for (int m = 0; m < g->len[k]; m++) {
      int b = g->members[k][m], r = b >> 2, c = b & 3;
      if (r < min_r) min_r = r;
      if (r > max_r) max_r = r;
      if (c < min_c) min_c = c;
      if (c > max_c) max_c = c;
    }
    g->row0[k] = min_r * 4;
    g->col0[k] = min_c * 4;
    g->w[k] = (max_c + 1 - min_c) * 4;
    g->h[k] = (max_r + 1 - min_r) * 4;
  }
}

/* group_sad_at_whole_mv(_shaped) (src/encoder.rs:7650-7797): every pixel
 * of the group rectangle fetched edge-clamped at the integer part of the
 * eighth-pel vector (the in-bounds fast path is the same sum). */
static uint32_t group_sad(const vp8a_luma_ref* r, int mb_col, int mb_row, const uint8_t* src_y,
                          const part_groups* g, int k, vp8a_mv mv) {
  int16_t er = (int16_t)(uint16_t)((uint16_t)mv.row * 2u);
  int16_t ec = (int16_t)(uint16_t)((uint16_t)mv.col * 2u);
  int64_t y0 = (int64_t)mb_row * 16 + (er >> 3), x0 = (int64_t)mb_col * 16 + (ec >> 3);
  uint32_t sad = 0;
  for (int rr = g->row0[k]; rr < g->row0[k] + g->h[k]; rr++) {
    int64_t sy = y0 + rr;
    if (sy < 0) sy = 0;
    if (sy > (int64_t)r->height - 1) sy = r->height - 1;
    for (int cc = g->col0[k]; cc < g->col0[k] + g->w[k]; cc++) {
      int64_t sx = x0 + cc;
      if (sx < 0) sx = 0;
      if (sx > (int64_t)r->width - 1) sx = r->width - 1;
      int d = (int)src_y[rr * 16 + cc] - (int)r->plane[(size_t)sy * r->stride + (size_t)sx];
      sad += (uint32_t)(d < 0 ? -d : d);
    }
  }
  return sad;
}

/* group_small_diamond_search (src/encoder.rs:7812-7879): snap then clamp
 * the centre; candidates clamped (not snapped); 4 iterations. */
static void group_diamond(const vp8a_luma_ref* r, int mb_col, int mb_row, const uint8_t* src_y,
                          const part_groups* g, int k, vp8a_mv center, uint32_t max_iters,
                          vp8a_mv* best_out, uint32_t* sad_out) {
  vp8a_mv best;
  best.row = (int16_t)clampi((center.row / 4) * 4, MV_MIN, MV_MAX);
  best.col = (int16_t)clampi((center.col / 4) * 4, MV_MIN, MV_MAX);
  uint32_t best_sad = group_sad(r, mb_col, mb_row, src_y, g, k, best);
  static const int off[4][2] = {{-4, 0}, {4, 0}, {0, -4}, {0, 4}};
  for (uint32_t it = 0; it < max_iters; it++) {
    int improved = 0;
    for (int o = 0; o < 4; o++) {
      vp8a_mv c;
      c.row = (int16_t)clampi(best.row + off[o][0], MV_MIN, MV_MAX);
      c.col = (int16_t)clampi(best.col + off[o][1], MV_MIN, MV_MAX);
      if (mv_eq(c, best)) continue;
      uint32_t s = group_sad(r, mb_col, mb_row, src_y, g, k, c);
      if (s < best_sad) {
        best_sad = s;
        best = c;
        improved = 1;
      }
    }
    if (!improved) break;
  }
  *best_out = best;
  *sad_out = best_sad;
}

/* above_block_mv / left_block_mv (src/near_mv.rs:722-760). */
static vp8a_mv above_block_mv(const vp8a_mv* this_split, const vo_mb_info* above, int b) {
  if (b < 4) {
    if (above->ref_frame == VP8A_REF_INTRA) return MV0;
    if (above->is_split) return above->has_split_mvs ? above->split_mvs[b + 12] : above->mv;
    return above->mv;
  }
  return this_split[b - 4];
}
static vp8a_mv left_block_mv(const vp8a_mv* this_split, const vo_mb_info* left, int b) {
  if ((b & 3) == 0) {
    if (left->ref_frame == VP8A_REF_INTRA) return MV0;
    if (left->is_split) return left->has_split_mvs ? left->split_mvs[b + 3] : left->mv;
    return left->mv;
  }
  return this_split[b - 1];
}

/* submv_ref_context (src/near_mv.rs). */
static int submv_ref_context(vp8a_mv l, vp8a_mv a) {
  int lez = mv_zero(l), aez = mv_zero(a), lea = mv_eq(l, a);
  if (lea && lez) return 4;
  if (lea) return 3;
  if (aez) return 2;
  if (lez) return 1;
  return 0;
}

/* submv_ref_bits (src/encoder.rs:8021). */
static double submv_ref_bits(const uint8_t* p, int mode) {
  switch (mode) {
    case VP8A_SUBMV_LEFT: return BB(p[0], 0);
    case VP8A_SUBMV_ABOVE: return BB(p[0], 1) + BB(p[1], 0);
    case VP8A_SUBMV_ZERO: return BB(p[0], 1) + BB(p[1], 1) + BB(p[2], 0);
    default: return BB(p[0], 1) + BB(p[1], 1) + BB(p[2], 1);
  }
}

/* mv_partition_bits (src/encoder.rs:8035). */
static double mv_partition_bits(int pid) {
  const uint8_t* p = MV_PARTITION_PROBS;
  switch (pid) {
    case VP8A_PART_MV16: return BB(p[0], 0);
    case VP8A_PART_QUARTERS: return BB(p[0], 1) + BB(p[1], 0);
    case VP8A_PART_TOP_BOTTOM: return BB(p[0], 1) + BB(p[1], 1) + BB(p[2], 0);
    default: return BB(p[0], 1) + BB(p[1], 1) + BB(p[2], 1);
  }
}

typedef struct {
  vp8a_mv split_mvs[16];
  uint8_t submv_modes[16];
  double j;
} split_cand;

/* score_split_partition (src/encoder.rs:8080-8246). Returns 0 when no
 * viable candidate exists (unreachable: ZERO4X4 always prices finite). */
static int score_split_partition(int pid, const vp8a_luma_ref* r, int mb_col, int mb_row,
                                 const uint8_t* src_y, vp8a_mv best_predictor,
                                 const vo_mb_info* above, const vo_mb_info* left,
                                 const vp8a_mv_contexts* ctx, double lambda, split_cand* out) {
  part_groups g;
  build_groups(pid, &g);
  vp8a_mv split_mvs[16];
  for (int i = 0; i < 16; i++) split_mvs[i] = MV0;
  uint8_t modes[16];
  memset(modes, VP8A_SUBMV_ZERO, sizeof modes);
  uint32_t total_sad = 0;
  double total_submv_bits = 0.0;
  for (int k = 0; k < g.num_groups; k++) {
    int anchor = g.members[k][0];
    vp8a_mv lmv = left_block_mv(split_mvs, left, anchor);
    vp8a_mv amv = above_block_mv(split_mvs, above, anchor);
    const uint8_t* probs = SUBMV_REF_PROBS[submv_ref_context(lmv, amv)];
    vp8a_mv search_mv;
    uint32_t search_sad;
    group_diamond(r, mb_col, mb_row, src_y, &g, k, best_predictor, 4, &search_mv, &search_sad);

    int best_mode = VP8A_SUBMV_ZERO;
    vp8a_mv best_mv = MV0, best_diff = MV0;
    double best_j = INFINITY;
    const vp8a_mv cmv[3] = {lmv, amv, MV0};
    for (int m = 0; m < 3; m++) {
      double sad = (double)group_sad(r, mb_col, mb_row, src_y, &g, k, cmv[m]);
      double mode_bits = submv_ref_bits(probs, m);
      double j = sad + lambda * (mode_bits + 0.0);
      if (j < best_j) {
        best_j = j;
        best_mode = m;
        best_mv = cmv[m];
        best_diff = MV0;
      }
    }
    int32_t dr = (int32_t)search_mv.row - best_predictor.row;
    int32_t dc = (int32_t)search_mv.col - best_predictor.col;
    if (dr >= -1023 && dr <= 1023 && dc >= -1023 && dc <= 1023) {
      double diff_bits = vo_mv_component_bits(ctx->p[0], dr) + vo_mv_component_bits(ctx->p[1], dc);
      double mode_bits = submv_ref_bits(probs, VP8A_SUBMV_NEW);
      double j = (double)search_sad + lambda * (mode_bits + diff_bits);
      if (j < best_j) {
        best_j = j;
        best_mode = VP8A_SUBMV_NEW;
        best_mv = search_mv;
        best_diff.row = (int16_t)dr;
        best_diff.col = (int16_t)dc;
      }
    }
    if (!isfinite(best_j)) return 0;
    uint32_t gs = group_sad(r, mb_col, mb_row, src_y, &g, k, best_mv);
    for (int m = 0; m < g.len[k]; m++) split_mvs[g.members[k][m]] = best_mv;
    total_sad += gs;
    total_submv_bits += submv_ref_bits(probs, best_mode);
    if (best_mode == VP8A_SUBMV_NEW)
      total_submv_bits += vo_mv_component_bits(ctx->p[0], best_diff.row) +
                          vo_mv_component_bits(ctx->p[1], best_diff.col);
    modes[k] = (uint8_t)best_mode;
  }
  double partition_bits = mv_partition_bits(pid);
  out->j = (double)total_sad + lambda * (partition_bits + total_submv_bits);
  memcpy(out->split_mvs, split_mvs, sizeof split_mvs);
  memcpy(out->submv_modes, modes, sizeof modes);
  return 1;
}

/* ----------------------------------------------------------- per-ref pick */

typedef struct {
  uint8_t mode, partition;
  vp8a_mv mv;
  double j;
  vp8a_mv split_mvs[16];
  uint8_t submv_modes[16];
} ref_pick;

/* pick_mb_for_ref, search and decision part (src/encoder.rs:8546-8702). */
static void pick_mb_for_ref(uint8_t ref_id, const vp8a_luma_ref* r, const uint8_t* src_y,
                            const vo_mb_info* above, const vo_mb_info* left,
                            const vo_mb_info* aboveleft, int mb_col, int mb_row, int mb_cols,
                            int mb_rows, const vp8a_mv_contexts* ctx, double lambda,
                            const vp8a_mv* prop, ref_pick* out, vp8a_ref_search* trace) {
  vp8a_mv near[3];
  int32_t cnt[4];
  vo_find_near_mvs(above, left, aboveleft, ref_id, near, cnt);
  vp8a_mv best_predictor = clamp_mv_rect(near[0], mb_col, mb_row, mb_cols, mb_rows);
  uint8_t p[4];
  for (int i = 0; i < 4; i++) p[i] = MV_COUNTS_TO_PROBS[cnt[i]][i];

  uint32_t sad_zero = vo_mb_luma_sad_at_whole_mv(r, mb_col, mb_row, src_y, MV0);
  vp8a_search_result whole =
      vo_small_diamond_search_luma(r, mb_col, mb_row, src_y, best_predictor, 8);
  vp8a_search_result half = vo_half_pixel_refine_luma(r, mb_col, mb_row, src_y, whole.mv);
  vp8a_search_result search = vo_quarter_pixel_refine_luma(r, mb_col, mb_row, src_y, half.mv);

  double bits_mode_zero = BB(p[0], 0);
  double bits_mode_nearest = BB(p[0], 1) + BB(p[1], 0);
  double bits_mode_near = BB(p[0], 1) + BB(p[1], 1) + BB(p[2], 0);
  double bits_mode_new = BB(p[0], 1) + BB(p[1], 1) + BB(p[2], 1) + BB(p[3], 0);
  int32_t dr = (int32_t)search.mv.row - best_predictor.row;
  int32_t dc = (int32_t)search.mv.col - best_predictor.col;
  int diff_in_range = dr >= -1023 && dr <= 1023 && dc >= -1023 && dc <= 1023;
  double bits_mv_diff = diff_in_range ? vo_mv_component_bits(ctx->p[0], dr) +
                                            vo_mv_component_bits(ctx->p[1], dc)
                                      : INFINITY;
  vp8a_mv nearest_mv = clamp_mv_rect(near[1], mb_col, mb_row, mb_cols, mb_rows);
  vp8a_mv near_mv = clamp_mv_rect(near[2], mb_col, mb_row, mb_cols, mb_rows);
  uint32_t sad_nearest = vo_mb_luma_sad_at_mv(r, mb_col, mb_row, src_y, nearest_mv);
  uint32_t sad_near = vo_mb_luma_sad_at_mv(r, mb_col, mb_row, src_y, near_mv);

  double j_zero = (double)sad_zero + lambda * bits_mode_zero;
  double j_nearest = (double)sad_nearest + lambda * bits_mode_nearest;
  double j_near = (double)sad_near + lambda * bits_mode_near;
  double j_new = (double)search.sad + lambda * (bits_mode_new + bits_mv_diff);

  int nearest_eligible = !mv_zero(nearest_mv);
  int near_eligible = !mv_zero(near_mv);
  int new_eligible = diff_in_range && !mv_zero(search.mv);
  vp8a_mv new_mv = search.mv;
  /* A proposed vector (the learned proposal's, for this reference) is a
   * second NEWMV candidate: its exact SAD and the same cost terms; it
   * replaces the searched vector when strictly cheaper (or when that one
   * is not eligible). Proposals beyond +-1023 are ignored. */
  if (prop && prop->row >= -1023 && prop->row <= 1023 && prop->col >= -1023 && prop->col <= 1023 &&
      !mv_zero(*prop)) {
    int32_t pr = (int32_t)prop->row - best_predictor.row, pc = (int32_t)prop->col - best_predictor.col;
    if (pr >= -1023 && pr <= 1023 && pc >= -1023 && pc <= 1023) {
      uint32_t sad_p = vo_mb_luma_sad_at_mv(r, mb_col, mb_row, src_y, *prop);
      double j_p = (double)sad_p + lambda * (bits_mode_new + (vo_mv_component_bits(ctx->p[0], pr) +
                                                               vo_mv_component_bits(ctx->p[1], pc)));
      if (!new_eligible || j_p < j_new) {
        new_mv = *prop;
        j_new = j_p;
        new_eligible = 1;
      }
    }
  }

  out->mode = VP8A_MODE_ZERO;
  out->mv = MV0;
  out->partition = VP8A_PART_NONE;
  double chosen_j = j_zero;
  if (nearest_eligible && j_nearest < chosen_j) {
    out->mode = VP8A_MODE_NEAREST;
    out->mv = nearest_mv;
    chosen_j = j_nearest;
  }
  if (near_eligible && j_near < chosen_j) {
    out->mode = VP8A_MODE_NEAR;
    out->mv = near_mv;
    chosen_j = j_near;
  }
  if (new_eligible && j_new < chosen_j) {
    out->mode = VP8A_MODE_NEW;
    out->mv = new_mv;
    chosen_j = j_new;
  }

  double bits_mode_split = BB(p[0], 1) + BB(p[1], 1) + BB(p[2], 1) + BB(p[3], 1);
  int have_split = 0;
  split_cand best_split;
  int best_pid = VP8A_PART_NONE;
  for (int pid = 0; pid < 4; pid++) {
    split_cand c;
    if (!score_split_partition(pid, r, mb_col, mb_row, src_y, best_predictor, above, left, ctx,
                               lambda, &c))
      continue;
    double total_j = c.j + lambda * bits_mode_split;
    /* The stored best already carries bits_mode_split, and the comparison
     * adds it once more (src/encoder.rs:8679-8683); kept verbatim. */
    if (!have_split || total_j < best_split.j + lambda * bits_mode_split) {
      best_split = c;
      best_split.j = total_j;
      best_pid = pid;
      have_split = 1;
    }
  }
  for (int i = 0; i < 16; i++) out->split_mvs[i] = MV0;
  memset(out->submv_modes, VP8A_SUBMV_ZERO, 16);
  if (have_split && best_split.j < chosen_j) {
    out->mode = VP8A_MODE_SPLIT;
    out->mv = best_split.split_mvs[15];
    chosen_j = best_split.j;
    out->partition = (uint8_t)best_pid;
    memcpy(out->split_mvs, best_split.split_mvs, sizeof best_split.split_mvs);
    memcpy(out->submv_modes, best_split.submv_modes, 16);
  }
  out->j = chosen_j;

  if (trace) {
    trace->best_predictor = best_predictor;
    trace->nearest_mv = nearest_mv;
    trace->near_mv = near_mv;
    trace->sad_zero = sad_zero;
    trace->whole = whole;
    trace->half = half;
    trace->quarter = search;
    trace->sad_nearest = sad_nearest;
    trace->sad_near = sad_near;
    trace->chosen_mode = out->mode;
    trace->split_partition = out->partition;
    trace->reserved[0] = trace->reserved[1] = 0;
    trace->j = chosen_j;
  }
}

/* ref_frame_tree_bits(ref, 128, 128) (src/encoder.rs:9108). */
static double ref_tree_bits(uint8_t ref) {
  if (ref == VP8A_REF_LAST) return BB(128, 0);
  if (ref == VP8A_REF_GOLDEN) return BB(128, 1) + BB(128, 0);
  return BB(128, 1) + BB(128, 1);
}

/* extract_mb (src/encoder.rs:5549-5586), luma part. */
void vo_extract_mb_luma(const vp8a_i420* f, size_t mb_row, size_t mb_col, uint8_t* out) {
  size_t w = f->width, h = f->height;
  for (int r = 0; r < 16; r++) {
    size_t y = mb_row * 16 + r;
    if (y > h - 1) y = h - 1;
    for (int c = 0; c < 16; c++) {
      size_t x = mb_col * 16 + c;
      if (x > w - 1) x = w - 1;
      out[r * 16 + c] = f->y[y * f->y_stride + x];
    }
  }
}

typedef struct {
  const vp8a_i420* frame;
  const vp8a_planes* refs;
  const uint8_t* ref_ids;
  uint32_t n_refs;
  const vp8a_mv_contexts* ctx;
  double lambda;
  vp8a_mb_decision* dec;
  vp8a_ref_search* trace;
  const vp8a_mv* props; /* n_refs proposed vectors per MB, or NULL */
  vo_mb_info* infos;
  int mb_cols, mb_rows;
  atomic_int* progress; /* per row: MBs done */
} analyse_job;

/* One MB of decide_mb_exhaustive (src/encoder/inter.rs:537-590). */
static void analyse_mb(analyse_job* j, int mb_row, int mb_col) {
  static const vo_mb_info border = {VP8A_REF_INTRA, 0, 0, 0, {0, 0}, {{0, 0}}};
  const vo_mb_info* above = mb_row > 0 ? &j->infos[(mb_row - 1) * j->mb_cols + mb_col] : &border;
  const vo_mb_info* left = mb_col > 0 ? &j->infos[mb_row * j->mb_cols + mb_col - 1] : &border;
  const vo_mb_info* aboveleft = (mb_row > 0 && mb_col > 0)
                                    ? &j->infos[(mb_row - 1) * j->mb_cols + mb_col - 1]
                                    : &border;
  uint8_t src_y[256];
  vo_extract_mb_luma(j->frame, mb_row, mb_col, src_y);
  ref_pick best;
  double best_total = INFINITY;
  int have = 0;
  uint8_t best_ref = 0;
  size_t idx = (size_t)mb_row * j->mb_cols + mb_col;
  for (uint32_t k = 0; k < j->n_refs; k++) {
    vp8a_luma_ref lr = {j->refs[k].y, j->refs[k].y_stride, j->refs[k].mb_cols * 16,
                        j->refs[k].mb_rows * 16};
    ref_pick pk;
    pick_mb_for_ref(j->ref_ids[k], &lr, src_y, above, left, aboveleft, mb_col, mb_row,
                    j->mb_cols, j->mb_rows, j->ctx, j->lambda, j->props ? &j->props[idx * j->n_refs + k] : NULL,
                    &pk,
                    j->trace ? &j->trace[idx * j->n_refs + k] : NULL);
    double total = pk.j + j->lambda * ref_tree_bits(j->ref_ids[k]);
    if (total < best_total) {
      best_total = total;
      best = pk;
      best_ref = j->ref_ids[k];
      have = 1;
    }
  }
  vp8a_mb_decision* d = &j->dec[idx];
  memset(d, 0, sizeof *d);
  vo_mb_info* info = &j->infos[idx];
  memset(info, 0, sizeof *info);
  if (!have) return;
  d->ref_frame = best_ref;
  d->mode = best.mode;
  d->partition = best.partition;
  d->mv = best.mv;
  d->j = best.j;
  d->total = best_total;
  memcpy(d->split_mvs, best.split_mvs, sizeof d->split_mvs);
  memcpy(d->submv_modes, best.submv_modes, sizeof d->submv_modes);
  /* The census record later MBs read (src/encoder/inter.rs:458-480). */
  info->ref_frame = best_ref;
  info->mv = best.mv;
  if (best.mode == VP8A_MODE_SPLIT) {
    info->is_split = 1;
    info->has_split_mvs = 1;
    memcpy(info->split_mvs, best.split_mvs, sizeof info->split_mvs);
  }
}

/* analyse_row (src/encoder/inter.rs:350-513): MB (r, c) waits until row
 * r-1 has finished min(c+2, mb_cols) MBs. */
static void analyse_row_task(void* arg, uint32_t row) {
  analyse_job* j = (analyse_job*)arg;
  for (int c = 0; c < j->mb_cols; c++) {
    if (row > 0) {
      int need = c + 2 < j->mb_cols ? c + 2 : j->mb_cols;
      while (atomic_load_explicit(&j->progress[row - 1], memory_order_acquire) < need)
        sched_yield();
    }
    analyse_mb(j, (int)row, c);
    atomic_store_explicit(&j->progress[row], c + 1, memory_order_release);
  }
}

int vo_analyse_inter_frame_proposals(const vp8a_i420* frame, const vp8a_planes* refs,
                                     const uint8_t* ref_ids, uint32_t n_refs,
                                     const vp8a_mv_contexts* mv_contexts, double lambda,
                                     const vp8a_mv* proposals, vp8a_mb_decision* decisions,
                                     vp8a_ref_search* trace, uint32_t threads);

int vo_analyse_inter_frame(const vp8a_i420* frame, const vp8a_planes* refs,
                           const uint8_t* ref_ids, uint32_t n_refs,
                           const vp8a_mv_contexts* mv_contexts, double lambda,
                           vp8a_mb_decision* decisions, vp8a_ref_search* trace,
                           uint32_t threads) {
  return vo_analyse_inter_frame_proposals(frame, refs, ref_ids, n_refs, mv_contexts, lambda, NULL,
                                          decisions, trace, threads);
}

/* vo_analyse_inter_frame with one proposed vector per (MB, reference) as a
 * second NEWMV candidate (the learned proposal's seeds into the exhaustive
 * decision; no counterpart in the reference). */
int vo_analyse_inter_frame_proposals(const vp8a_i420* frame, const vp8a_planes* refs,
                                     const uint8_t* ref_ids, uint32_t n_refs,
                                     const vp8a_mv_contexts* mv_contexts, double lambda,
                                     const vp8a_mv* proposals, vp8a_mb_decision* decisions,
                                     vp8a_ref_search* trace, uint32_t threads) {
  if (!frame || !decisions || (n_refs > 0 && (!refs || !ref_ids))) return VP8A_E_INVALID_ARGUMENT;
  if (frame->width == 0 || frame->height == 0 || frame->width > 0x3FFF || frame->height > 0x3FFF)
    return VP8A_E_INVALID_DIMENSIONS;
  if (n_refs == 0 || n_refs > 3) return VP8A_E_INVALID_ARGUMENT;
  int mb_cols = (int)((frame->width + 15) / 16), mb_rows = (int)((frame->height + 15) / 16);
  for (uint32_t k = 0; k < n_refs; k++)
    if ((int)refs[k].mb_cols != mb_cols || (int)refs[k].mb_rows != mb_rows)
      return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
  init_bit_cost();
  vp8a_mv_contexts defctx;
  if (!mv_contexts) {
    vo_default_mv_contexts(&defctx);
    mv_contexts = &defctx;
  }
  analyse_job j;
  j.frame = frame;
  j.refs = refs;
  j.ref_ids = ref_ids;
  j.n_refs = n_refs;
  j.ctx = mv_contexts;
  j.lambda = lambda;
  j.dec = decisions;
  j.trace = trace;
  j.props = proposals;
  j.mb_cols = mb_cols;
  j.mb_rows = mb_rows;
  j.infos = (vo_mb_info*)calloc((size_t)mb_cols * mb_rows, sizeof(vo_mb_info));
  j.progress = (atomic_int*)calloc((size_t)mb_rows, sizeof(atomic_int));
  if (!j.infos || !j.progress) {
    free(j.infos);
    free(j.progress);
    return VP8A_E_OUT_OF_MEMORY;
  }
  for (int r = 0; r < mb_rows; r++) atomic_init(&j.progress[r], 0);
  /* Rows are claimed in increasing order, so every waited-on row is
   * already owned by a running worker: no deadlock for any thread count. */
  vo_parallel_for((uint32_t)mb_rows, threads, analyse_row_task, &j);
  free(j.infos);
  free(j.progress);
  return VP8A_OK;
}
