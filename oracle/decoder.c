/*
 * decoder.c — oracle restatement of the oxideav-vp8 decoder (key and inter
 * frames), the encoder<->decoder lockstep checker and the bridge to the
 * libvpx-produced decode fixtures the reference vendors.
 *
 * TEST INFRASTRUCTURE ONLY (see vp8a_oracle.h). Follows:
 *   frame tag, key-frame header        src/frame_header.rs:302-360
 *   bool decoder                       src/bool_decoder.rs:100-333
 *   first-partition header             src/coded_header.rs:557-1140
 *   DCT partitions                     src/decoder.rs:502-560
 *   key-frame MB modes                 src/macroblock.rs:265-520
 *   intra MB modes in inter frames     src/macroblock.rs:580-800
 *   inter MB modes: select_ref_frame   src/motion_comp.rs:108
 *     find_near_mvs with sign bias     src/near_mv.rs:198-402
 *     read_inter_mode, split MVs       src/near_mv.rs:418-1000
 *     read_mv                          src/motion_vector.rs:100-240
 *     resolve_inter_mb_mv_after_mode   src/state.rs:1548-1600
 *   tokens and dequantisation          src/dct_tokens.rs:190-971, src/dequant.rs:383
 *   intra prediction                   src/intra_predict.rs:90-760,
 *                                      src/frame.rs:288-384, src/reconstruct.rs:295-560
 *   frame flow, probability carry,
 *     loop-filter deltas, references   src/state.rs:481-1226, :154-268
 *   FrameFilterConfig keyframe/interframe  src/loop_filter.rs:1077-1210
 * The RFC 6386 probability tables are in vp8_tables.h. Inter prediction,
 * the inverse transforms and the loop filter are the oracle's own
 * restatements (predict.c, recon.c, lf.c).
 */
#include <stdlib.h>
#include <string.h>

#include "vp8_tables.h"
#include "vp8a_oracle.h"

/* ------------------------------------------------------------ bool decoder */

typedef struct {
  const uint8_t* p;
  const uint8_t* end;
  uint32_t value, range;
  int bit_count;
} bd_t;

/* BoolDecoder::init_partition (src/bool_decoder.rs:100-135). Past the end
 * of its input the decoder shifts in zero bytes. */
static void bd_init(bd_t* d, const uint8_t* p, size_t n) {
  d->range = 255;
  d->bit_count = 0;
  if (n >= 2) {
    d->value = ((uint32_t)p[0] << 8) | p[1];
    d->p = p + 2;
    d->end = p + n;
  } else {
    d->value = 0;
    d->p = d->end = p;
  }
}

/* read_bool + renormalize (src/bool_decoder.rs:159-190, :311-333). */
static int bd_bool(bd_t* d, int prob) {
  const uint32_t split = 1 + (((d->range - 1) * (uint32_t)prob) >> 8);
  const uint32_t big = split << 8;
  int bit;
  if (d->value >= big) {
    d->value -= big;
    d->range -= split;
    bit = 1;
  } else {
    d->range = split;
    bit = 0;
  }
  while (d->range < 128) {
    d->value <<= 1;
    d->range <<= 1;
    if (++d->bit_count == 8) {
      d->bit_count = 0;
      if (d->p < d->end) d->value |= *d->p++;
    }
  }
  return bit;
}

static uint32_t bd_lit(bd_t* d, int n) {
  uint32_t v = 0;
  while (n-- > 0) v = (v << 1) | (uint32_t)bd_bool(d, 128);
  return v;
}

/* read_signed_delta (src/coded_header.rs:1037): magnitude, then sign. */
static int bd_signed(bd_t* d, int n) {
  int v = (int)bd_lit(d, n);
  return bd_bool(d, 128) ? -v : v;
}

/* treed_read (src/macroblock.rs:316-334): leaves are stored negated. */
static int bd_tree(bd_t* d, const int8_t* tree, const uint8_t* probs) {
  int i = 0;
  for (;;) {
    const int next = tree[i + bd_bool(d, probs[i >> 1])];
    if (next <= 0) return -next;
    i = next;
  }
}

/* ------------------------------------------------------------------ tables */

static const int8_t KF_YMODE_TREE[8] = {-4, 2, 4, 6, 0, -1, -2, -3};
static const uint8_t KF_YMODE_PROB[4] = {145, 156, 163, 128};
static const int8_t IF_YMODE_TREE[8] = {0, 2, 4, 6, -1, -2, -3, -4};
static const int8_t UV_MODE_TREE[6] = {0, 2, -1, 4, -2, -3};
static const uint8_t KF_UV_MODE_PROB[3] = {142, 114, 183};
static const int8_t BMODE_TREE[18] = {0, 2, -1, 4, -2, 6, 8, 12, -3, 10, -5, -6, -4, 14, -7, 16, -8, -9};
static const uint8_t IF_BMODE_PROB[9] = {120, 90, 79, 133, 87, 85, 80, 111, 151};
static const uint8_t IF_YMODE_PROB_DEFAULTS[4] = {112, 86, 140, 37};
static const uint8_t IF_UV_MODE_PROB_DEFAULTS[3] = {162, 101, 204};
static const int8_t SEGMENT_TREE[6] = {2, 4, 0, -1, -2, -3};
static const int8_t MV_REF_TREE[8] = {0, 2, -1, 4, -2, 6, -3, -4};
static const int8_t MV_PARTITION_TREE[6] = {-3, 2, -2, 4, 0, -1};
static const uint8_t MV_PARTITION_PROBS[3] = {110, 111, 150};
static const int8_t SUBMV_REF_TREE[6] = {0, 2, -1, 4, -2, -3};
static const uint8_t SUBMV_REF_PROBS[5][3] = {
    {147, 136, 18}, {106, 145, 1}, {179, 121, 1}, {223, 1, 34}, {208, 1, 1}};
static const uint8_t MV_PARTITIONS[4][16] = {
    {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1},
    {0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1},
    {0, 0, 1, 1, 0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 3, 3},
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}};
static const uint8_t MV_COUNTS_TO_PROBS[6][4] = {{7, 1, 1, 143},    {14, 18, 14, 107},
                                                 {135, 64, 57, 68}, {60, 56, 128, 65},
                                                 {159, 134, 128, 34}, {234, 188, 128, 28}};
static const uint8_t MV_UPDATE_PROBS[2][19] = {
    {237, 246, 253, 253, 254, 254, 254, 254, 254, 254, 254, 254, 254, 254, 250, 250, 252, 254, 254},
    {231, 243, 245, 253, 254, 254, 254, 254, 254, 254, 254, 254, 254, 254, 251, 251, 254, 254, 254}};
static const uint8_t DEFAULT_MV_CONTEXT[2][19] = {
    {162, 128, 225, 146, 172, 147, 214, 39, 156, 128, 129, 132, 75, 145, 178, 206, 239, 254, 254},
    {164, 128, 204, 170, 119, 235, 140, 230, 228, 128, 130, 130, 74, 148, 180, 203, 236, 254, 254}};
static const int8_t SMALL_MVTREE[14] = {2, 8, 4, 6, 0, -1, -2, -3, 10, 12, -4, -5, -6, -7};
#define COEFF_BANDS VO_COEFF_BANDS
#define ZIGZAG VO_ZIGZAG
#define PCAT VO_PCAT
#define PCAT_LEN VO_PCAT_LEN
#define CAT_BASE VO_CAT_BASE
static const uint8_t LEFT_CTX[25] = {0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3,
                                     4, 4, 5, 5, 6, 6, 7, 7, 8};
static const uint8_t ABOVE_CTX[25] = {0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3,
                                      4, 5, 4, 5, 6, 7, 6, 7, 8};

enum { YM_DC = 0, YM_V = 1, YM_H = 2, YM_TM = 3, YM_B = 4 };
enum { B_DC = 0, B_TM, B_VE, B_HE, B_LD, B_RD, B_VR, B_VL, B_HD, B_HU };
enum { BT_Y_AFTER_Y2 = 0, BT_Y2 = 1, BT_UV = 2, BT_Y_NO_Y2 = 3 };

/* ----------------------------------------------------------- decoder state */

struct vo_vp8_decoder {
  vo_vp8_capture* cap;  /* optional per-frame capture (see vo_vp8_decoder_capture) */
  int have_key;
  uint32_t width, height, mb_cols, mb_rows;
  uint8_t* slot[3][3]; /* LAST, GOLDEN, ALTREF x (y, u, v), MB-padded */
  uint8_t coef[4][8][3][11];
  uint8_t mvc[2][19];
  uint8_t ymode_prob[4], uvmode_prob[3];
  int sign_bias_golden, sign_bias_altref;
  int16_t ref_lf_deltas[4], mode_lf_deltas[4];
};

vo_vp8_decoder* vo_vp8_decoder_new(void) {
  vo_vp8_decoder* d = (vo_vp8_decoder*)calloc(1, sizeof(vo_vp8_decoder));
  return d;
}

/* Attach (or with NULL detach) caller buffers that each later decode fills
 * with that frame's intermediate state: the references in force, every
 * inter MB's prediction and decision, the reconstruction before and after
 * the loop filter, the MBs' loop-filter records and the filter
 * configuration. */
void vo_vp8_decoder_capture(vo_vp8_decoder* d, vo_vp8_capture* cap) { d->cap = cap; }

void vo_vp8_decoder_free(vo_vp8_decoder* d) {
  if (!d) return;
  for (int s = 0; s < 3; s++)
    for (int p = 0; p < 3; p++) free(d->slot[s][p]);
  free(d);
}

static int alloc_slots(vo_vp8_decoder* d);

/* Test hook: install `refs` (LAST, GOLDEN, ALTREF x (y, u, v), MB-padded
 * planes of a width x height picture) as the three reference slots, with
 * the entropy state a key frame without probability updates leaves
 * (default coefficient, MV and mode probabilities, no sign bias, no loop
 * filter deltas). Inter frames written against arbitrary references then
 * decode as they would after such a key frame. Returns 0, or -1 for a bad
 * size or an allocation failure. */
int vo_vp8_decoder_prime(vo_vp8_decoder* d, uint32_t width, uint32_t height, const uint8_t* const* refs) {
  if (!d || !width || !height || width > 0x3fff || height > 0x3fff) return -1;
  d->width = width;
  d->height = height;
  d->mb_cols = (width + 15) / 16;
  d->mb_rows = (height + 15) / 16;
  if (alloc_slots(d)) return -1;
  const size_t ly = (size_t)d->mb_cols * 16 * d->mb_rows * 16;
  for (int s = 0; s < 3; s++)
    for (int p = 0; p < 3; p++) memcpy(d->slot[s][p], refs[3 * s + p], p ? ly / 4 : ly);
  memcpy(d->coef, VO_DEFAULT_COEF_PROBS, sizeof d->coef);
  memcpy(d->ymode_prob, IF_YMODE_PROB_DEFAULTS, 4);
  memcpy(d->uvmode_prob, IF_UV_MODE_PROB_DEFAULTS, 3);
  memcpy(d->mvc, DEFAULT_MV_CONTEXT, sizeof d->mvc);
  d->sign_bias_golden = d->sign_bias_altref = 0;
  memset(d->ref_lf_deltas, 0, sizeof d->ref_lf_deltas);
  memset(d->mode_lf_deltas, 0, sizeof d->mode_lf_deltas);
  d->have_key = 1;
  return 0;
}

/* ---------------------------------------------------------------- headers */

typedef struct {
  int key, version, show;
  uint32_t first_size, hdr_bytes, width, height;
  /* first partition */
  int segmentation_enabled, update_map, update_data, seg_abs;
  int has_quant[4], quant[4], has_lf[4], lf[4];
  uint8_t seg_prob[3];
  int filter_type, level, sharpness;
  int lf_adj_enable, has_ref_delta[4], ref_delta[4], has_mode_delta[4], mode_delta[4];
  int nparts;
  vp8a_quant_indices qi;
  int refresh_entropy, refresh_golden, refresh_altref, copy_to_golden, copy_to_altref;
  int sign_bias_golden, sign_bias_altref, refresh_last;
  int no_skip_coeff, prob_skip;
  int prob_intra, prob_last, prob_gf;
  int has_ymode_prob, has_uvmode_prob;
  uint8_t ymode_prob[4], uvmode_prob[3];
  int has_mv_update[2][19];
  uint8_t mv_update[2][19];
} hdr_t;

/* Vp8CodedHeader::parse_from_decoder (src/coded_header.rs:557-740) minus the
 * token probability updates, which are applied straight to `coef`. */
static void parse_header(bd_t* d, hdr_t* h, uint8_t coef[4][8][3][11]) {
  if (h->key) {
    bd_bool(d, 128); /* color_space */
    bd_bool(d, 128); /* clamping_type */
  }
  h->segmentation_enabled = bd_bool(d, 128);
  h->seg_prob[0] = h->seg_prob[1] = h->seg_prob[2] = 255;
  if (h->segmentation_enabled) {
    h->update_map = bd_bool(d, 128);
    h->update_data = bd_bool(d, 128);
    if (h->update_data) {
      h->seg_abs = bd_bool(d, 128);
      for (int i = 0; i < 4; i++)
        if ((h->has_quant[i] = bd_bool(d, 128))) h->quant[i] = bd_signed(d, 7);
      for (int i = 0; i < 4; i++)
        if ((h->has_lf[i] = bd_bool(d, 128))) h->lf[i] = bd_signed(d, 6);
    }
    if (h->update_map)
      for (int i = 0; i < 3; i++)
        if (bd_bool(d, 128)) h->seg_prob[i] = (uint8_t)bd_lit(d, 8);
  }
  h->filter_type = bd_bool(d, 128);
  h->level = (int)bd_lit(d, 6);
  h->sharpness = (int)bd_lit(d, 3);
  h->lf_adj_enable = bd_bool(d, 128);
  if (h->lf_adj_enable && bd_bool(d, 128)) {
    for (int i = 0; i < 4; i++)
      if ((h->has_ref_delta[i] = bd_bool(d, 128))) h->ref_delta[i] = bd_signed(d, 6);
    for (int i = 0; i < 4; i++)
      if ((h->has_mode_delta[i] = bd_bool(d, 128))) h->mode_delta[i] = bd_signed(d, 6);
  }
  h->nparts = 1 << bd_lit(d, 2);
  memset(&h->qi, 0, sizeof h->qi);
  h->qi.y_ac_qi = (uint8_t)bd_lit(d, 7);
  int8_t* deltas[5] = {&h->qi.y_dc_delta, &h->qi.y2_dc_delta, &h->qi.y2_ac_delta,
                       &h->qi.uv_dc_delta, &h->qi.uv_ac_delta};
  for (int i = 0; i < 5; i++)
    if (bd_bool(d, 128)) *deltas[i] = (int8_t)bd_signed(d, 4);
  if (h->key) {
    h->refresh_entropy = bd_bool(d, 128);
  } else {
    h->refresh_golden = bd_bool(d, 128);
    h->refresh_altref = bd_bool(d, 128);
    h->copy_to_golden = h->refresh_golden ? 0 : (int)bd_lit(d, 2);
    h->copy_to_altref = h->refresh_altref ? 0 : (int)bd_lit(d, 2);
    h->sign_bias_golden = bd_bool(d, 128);
    h->sign_bias_altref = bd_bool(d, 128);
    h->refresh_entropy = bd_bool(d, 128);
    h->refresh_last = bd_bool(d, 128);
  }
  /* parse_token_prob_update (src/coded_header.rs:987) overlaid on `coef`. */
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 8; j++)
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 11; l++)
          if (bd_bool(d, VO_COEF_UPDATE_PROBS[i][j][k][l])) coef[i][j][k][l] = (uint8_t)bd_lit(d, 8);
  h->no_skip_coeff = bd_bool(d, 128);
  h->prob_skip = h->no_skip_coeff ? (int)bd_lit(d, 8) : 0;
  if (!h->key) {
    h->prob_intra = (int)bd_lit(d, 8);
    h->prob_last = (int)bd_lit(d, 8);
    h->prob_gf = (int)bd_lit(d, 8);
    if ((h->has_ymode_prob = bd_bool(d, 128)))
      for (int i = 0; i < 4; i++) h->ymode_prob[i] = (uint8_t)bd_lit(d, 8);
    if ((h->has_uvmode_prob = bd_bool(d, 128)))
      for (int i = 0; i < 3; i++) h->uvmode_prob[i] = (uint8_t)bd_lit(d, 8);
    /* parse_mv_prob_update (src/coded_header.rs:969). */
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 19; j++)
        if ((h->has_mv_update[i][j] = bd_bool(d, MV_UPDATE_PROBS[i][j]))) {
          const uint32_t x = bd_lit(d, 7);
          h->mv_update[i][j] = (uint8_t)(x ? x << 1 : 1);
        }
  }
}

/* -------------------------------------------------------------- MV helpers */

typedef struct {
  uint8_t ref; /* VP8A_REF_*; INTRA for intra / border */
  uint8_t is_split;
  vp8a_mv mv;
  vp8a_mv split[16];
} mbinfo_t;

static inline int mv_eq(vp8a_mv a, vp8a_mv b) { return a.row == b.row && a.col == b.col; }
static inline int mv_zero(vp8a_mv a) { return a.row == 0 && a.col == 0; }

/* SignBias::for_ref (src/near_mv.rs:198). */
static int sign_bias_for(const hdr_t* h, int ref) {
  return ref == VP8A_REF_GOLDEN ? h->sign_bias_golden : (ref == VP8A_REF_ALTREF ? h->sign_bias_altref : 0);
}

/* mv_bias (src/near_mv.rs:214). */
static vp8a_mv mv_bias(const hdr_t* h, int nref, int cref, vp8a_mv mv) {
  if (sign_bias_for(h, nref) ^ sign_bias_for(h, cref)) {
    mv.row = (int16_t)(uint16_t)(-(uint16_t)mv.row);
    mv.col = (int16_t)(uint16_t)(-(uint16_t)mv.col);
  }
  return mv;
}

/* find_near_mvs (src/near_mv.rs:310-402), with the frame's sign bias. */
static void near_mvs(const hdr_t* h, const mbinfo_t* above, const mbinfo_t* left,
                     const mbinfo_t* al, int cref, vp8a_mv out[3], int cnt[4]) {
  vp8a_mv nm[4];
  memset(nm, 0, sizeof nm);
  cnt[0] = cnt[1] = cnt[2] = cnt[3] = 0;
  int mi = 0, ci = 0;
  if (above->ref != VP8A_REF_INTRA) {
    if (!mv_zero(above->mv)) {
      nm[++mi] = mv_bias(h, above->ref, cref, above->mv);
      ci++;
    }
    cnt[ci] += 2;
  }
  if (left->ref != VP8A_REF_INTRA) {
    if (!mv_zero(left->mv)) {
      vp8a_mv m = mv_bias(h, left->ref, cref, left->mv);
      if (!mv_eq(m, nm[mi])) {
        nm[++mi] = m;
        ci++;
      }
      cnt[ci] += 2;
    } else {
      cnt[0] += 2;
    }
  }
  if (al->ref != VP8A_REF_INTRA) {
    if (!mv_zero(al->mv)) {
      vp8a_mv m = mv_bias(h, al->ref, cref, al->mv);
      if (!mv_eq(m, nm[mi])) {
        nm[++mi] = m;
        ci++;
      }
      cnt[ci] += 1;
    } else {
      cnt[0] += 1;
    }
  }
  if (cnt[3] != 0 && mv_eq(nm[mi], nm[1])) cnt[1] += 1;
  cnt[3] = (above->is_split + left->is_split) * 2 + al->is_split;
  if (cnt[2] > cnt[1]) {
    int t = cnt[1];
    cnt[1] = cnt[2];
    cnt[2] = t;
    vp8a_mv tm = nm[1];
    nm[1] = nm[2];
    nm[2] = tm;
  }
  if (cnt[1] >= cnt[0]) nm[0] = nm[1];
  out[0] = nm[0];
  out[1] = nm[1];
  out[2] = nm[2];
}

/* MvClampRect::for_mb + clamp_mv (src/near_mv.rs:236-283). */
static vp8a_mv clamp_mv(vp8a_mv mv, int col, int row, int cols, int rows) {
  const int to_left = -((col + 1) << 6), to_right = (cols - col) << 6;
  const int to_top = -((row + 1) << 6), to_bottom = (rows - row) << 6;
  vp8a_mv o;
  o.col = (int16_t)(mv.col < to_left ? to_left : (mv.col > to_right ? to_right : mv.col));
  o.row = (int16_t)(mv.row < to_top ? to_top : (mv.row > to_bottom ? to_bottom : mv.row));
  return o;
}

/* read_mv_component (src/motion_vector.rs:190-233). */
static int read_mv_component(bd_t* d, const uint8_t* p) {
  int a = 0;
  if (bd_bool(d, p[0])) {
    for (int i = 0; i < 3; i++) a += bd_bool(d, p[9 + i]) << i;
    for (int i = 9; i > 3; i--) a += bd_bool(d, p[9 + i]) << i;
    if ((a & 0xfff0) == 0 || bd_bool(d, p[9 + 3])) a += 8;
  } else {
    int i = 0;
    for (;;) {
      const int next = SMALL_MVTREE[i + bd_bool(d, p[2 + (i >> 1)])];
      if (next <= 0) {
        a = -next;
        break;
      }
      i = next;
    }
  }
  return (a != 0 && bd_bool(d, p[1])) ? -a : a;
}

/* read_mv (src/motion_vector.rs:236): row, then column. */
static vp8a_mv read_mv(bd_t* d, const uint8_t mvc[2][19]) {
  vp8a_mv m;
  m.row = (int16_t)read_mv_component(d, mvc[0]);
  m.col = (int16_t)read_mv_component(d, mvc[1]);
  return m;
}

static vp8a_mv mv_add(vp8a_mv a, vp8a_mv b) {
  vp8a_mv o;
  o.row = (int16_t)(uint16_t)((uint16_t)a.row + (uint16_t)b.row);
  o.col = (int16_t)(uint16_t)((uint16_t)a.col + (uint16_t)b.col);
  return o;
}

/* above_block_mv / left_block_mv (src/near_mv.rs:721-770). */
static vp8a_mv above_block_mv(const vp8a_mv* split, const mbinfo_t* above, int b) {
  if (b >= 4) return split[b - 4];
  if (above->ref == VP8A_REF_INTRA) return (vp8a_mv){0, 0};
  return above->is_split ? above->split[b + 12] : above->mv;
}

static vp8a_mv left_block_mv(const vp8a_mv* split, const mbinfo_t* left, int b) {
  if (b & 3) return split[b - 1];
  if (left->ref == VP8A_REF_INTRA) return (vp8a_mv){0, 0};
  return left->is_split ? left->split[b + 3] : left->mv;
}

/* submv_ref_context (src/near_mv.rs:640). */
static int submv_ctx(vp8a_mv l, vp8a_mv a) {
  const int lez = mv_zero(l), aez = mv_zero(a), lea = mv_eq(l, a);
  if (lea && lez) return 4;
  if (lea) return 3;
  if (aez) return 2;
  if (lez) return 1;
  return 0;
}

/* decode_split_mv (src/near_mv.rs:803-870). */
static void decode_split(bd_t* d, const mbinfo_t* above, const mbinfo_t* left, vp8a_mv best,
                         const uint8_t mvc[2][19], vp8a_mv split[16]) {
  const int part = bd_tree(d, MV_PARTITION_TREE, MV_PARTITION_PROBS);
  /* partition_id: TopBottom 0, LeftRight 1, Quarters 2, Mv16 3; the tree
   * leaves are in that order. */
  const uint8_t* table = MV_PARTITIONS[part];
  const int groups = part == 3 ? 16 : (part == 2 ? 4 : 2);
  memset(split, 0, 16 * sizeof(vp8a_mv));
  for (int j = 0; j < groups; j++) {
    int k = 0;
    while (table[k] != j) k++;
    const vp8a_mv lm = left_block_mv(split, left, k), am = above_block_mv(split, above, k);
    const int mode = bd_tree(d, SUBMV_REF_TREE, SUBMV_REF_PROBS[submv_ctx(lm, am)]);
    vp8a_mv mv;
    if (mode == 0) mv = lm;
    else if (mode == 1) mv = am;
    else if (mode == 2) mv = (vp8a_mv){0, 0};
    else mv = mv_add(best, read_mv(d, mvc));
    for (int i = 0; i < 16; i++)
      if (table[i] == j) split[i] = mv;
  }
}

/* --------------------------------------------------------------- tokens */

typedef struct {
  uint8_t nz[9];
} ectx_t;

/* decode_block_core (src/dct_tokens.rs:506-614), dequantising in place. */
static int decode_block(bd_t* d, const uint8_t probs[8][3][11], int first, int ctx3, int16_t* out,
                        int dcf, int acf) {
  int nz = 0, i = first;
  while (i < 16) {
    const uint8_t* p = probs[COEFF_BANDS[i]][ctx3];
    if (!bd_bool(d, p[0])) break;
    int zero_run_end = 0;
    while (!bd_bool(d, p[1])) {
      out[ZIGZAG[i]] = 0;
      if (++i == 16) {
        zero_run_end = 1;
        break;
      }
      p = probs[COEFF_BANDS[i]][0];
    }
    if (zero_run_end) break;
    int v;
    if (!bd_bool(d, p[2])) {
      ctx3 = 1;
      v = 1;
    } else {
      ctx3 = 2;
      int cat = -1;
      if (!bd_bool(d, p[3])) {
        if (!bd_bool(d, p[4])) v = 2;
        else v = bd_bool(d, p[5]) ? 4 : 3;
      } else if (!bd_bool(d, p[6])) {
        cat = bd_bool(d, p[7]) ? 1 : 0;
      } else if (!bd_bool(d, p[8])) {
        cat = bd_bool(d, p[9]) ? 3 : 2;
      } else {
        cat = bd_bool(d, p[10]) ? 5 : 4;
      }
      if (cat >= 0) {
        int e = 0;
        for (int k = 0; k < PCAT_LEN[cat]; k++) e = (e << 1) | bd_bool(d, PCAT[cat][k]);
        v = CAT_BASE[cat] + e;
      }
    }
    int s = bd_bool(d, 128) ? -v : v;
    const int slot = ZIGZAG[i];
    s = (int16_t)(s * (slot == 0 ? dcf : acf));
    out[slot] = (int16_t)s;
    nz++;
    i++;
  }
  return nz;
}

/* decode_mb_coeffs_inner (src/dct_tokens.rs:883-971): dequantised MbCoeffs
 * (y2[16], y[16][16], u[4][16], v[4][16]). */
static void decode_mb_tokens(bd_t* d, int has_y2, int skip, const uint8_t coef[4][8][3][11],
                             const int16_t* f, ectx_t* above, ectx_t* left, int16_t* c) {
  memset(c, 0, 400 * sizeof(int16_t));
  if (skip) {
    for (int i = 0; i < 8; i++) above->nz[i] = left->nz[i] = 0;
    if (has_y2) above->nz[8] = left->nz[8] = 0;
    return;
  }
  /* Y2 first (when present), then Y 0..15, U 16..19, V 20..23. */
  for (int k = has_y2 ? -1 : 0; k < 24; k++) {
    const int blk = k < 0 ? 24 : k;
    int type, dcf, acf;
    int16_t* out;
    if (blk == 24) {
      type = BT_Y2;
      dcf = f[2];
      acf = f[3];
      out = c;
    } else if (blk < 16) {
      type = has_y2 ? BT_Y_AFTER_Y2 : BT_Y_NO_Y2;
      dcf = f[0];
      acf = f[1];
      out = c + 16 + 16 * blk;
    } else {
      type = BT_UV;
      dcf = f[4];
      acf = f[5];
      out = c + 272 + 16 * (blk - 16);
    }
    const int first = type == BT_Y_AFTER_Y2 ? 1 : 0;
    const int ctx3 = above->nz[ABOVE_CTX[blk]] + left->nz[LEFT_CTX[blk]];
    const int nz = decode_block(d, coef[type], first, ctx3, out, dcf, acf);
    above->nz[ABOVE_CTX[blk]] = left->nz[LEFT_CTX[blk]] = nz != 0;
  }
}

/* --------------------------------------------------------- intra predict */

static inline uint8_t clamp255(int v) { return (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v)); }
static inline uint8_t avg2(int x, int y) { return (uint8_t)((x + y + 1) >> 1); }
static inline uint8_t avg3(int x, int y, int z) { return (uint8_t)((x + 2 * y + z + 2) >> 2); }

/* predict_b4x4 (src/intra_predict.rs:554-760). */
static void predict_b4x4(uint8_t* b, int mode, const uint8_t* A, const uint8_t* L, int P) {
  const uint8_t E[9] = {L[3], L[2], L[1], L[0], (uint8_t)P, A[0], A[1], A[2], A[3]};
#define B(r, c) b[(r) * 4 + (c)]
#define A3(p, i) avg3((p)[(i)-1], (p)[i], (p)[(i) + 1])
#define A2(p, i) avg2((p)[i], (p)[(i) + 1])
  switch (mode) {
    case B_DC: {
      int v = 4;
      for (int i = 0; i < 4; i++) v += A[i] + L[i];
      memset(b, v >> 3, 16);
      break;
    }
    case B_TM:
      for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) B(r, c) = clamp255(L[r] + A[c] - P);
      break;
    case B_VE: {
      const uint8_t ex[6] = {(uint8_t)P, A[0], A[1], A[2], A[3], A[4]};
      for (int c = 0; c < 4; c++) {
        const uint8_t v = avg3(ex[c], ex[c + 1], ex[c + 2]);
        for (int r = 0; r < 4; r++) B(r, c) = v;
      }
      break;
    }
    case B_HE: {
      const uint8_t ex[5] = {(uint8_t)P, L[0], L[1], L[2], L[3]};
      for (int r = 0; r < 3; r++) {
        const uint8_t v = avg3(ex[r], ex[r + 1], ex[r + 2]);
        for (int c = 0; c < 4; c++) B(r, c) = v;
      }
      const uint8_t v3 = avg3(L[2], L[3], L[3]);
      for (int c = 0; c < 4; c++) B(3, c) = v3;
      break;
    }
    case B_LD:
      B(0, 0) = A3(A, 1);
      B(0, 1) = B(1, 0) = A3(A, 2);
      B(0, 2) = B(1, 1) = B(2, 0) = A3(A, 3);
      B(0, 3) = B(1, 2) = B(2, 1) = B(3, 0) = A3(A, 4);
      B(1, 3) = B(2, 2) = B(3, 1) = A3(A, 5);
      B(2, 3) = B(3, 2) = A3(A, 6);
      B(3, 3) = avg3(A[6], A[7], A[7]);
      break;
    case B_RD:
      B(3, 0) = A3(E, 1);
      B(3, 1) = B(2, 0) = A3(E, 2);
      B(3, 2) = B(2, 1) = B(1, 0) = A3(E, 3);
      B(3, 3) = B(2, 2) = B(1, 1) = B(0, 0) = A3(E, 4);
      B(2, 3) = B(1, 2) = B(0, 1) = A3(E, 5);
      B(1, 3) = B(0, 2) = A3(E, 6);
      B(0, 3) = A3(E, 7);
      break;
    case B_VR:
      B(3, 0) = A3(E, 2);
      B(2, 0) = A3(E, 3);
      B(3, 1) = B(1, 0) = A3(E, 4);
      B(2, 1) = B(0, 0) = A2(E, 4);
      B(3, 2) = B(1, 1) = A3(E, 5);
      B(2, 2) = B(0, 1) = A2(E, 5);
      B(3, 3) = B(1, 2) = A3(E, 6);
      B(2, 3) = B(0, 2) = A2(E, 6);
      B(1, 3) = A3(E, 7);
      B(0, 3) = A2(E, 7);
      break;
    case B_VL:
      B(0, 0) = A2(A, 0);
      B(1, 0) = A3(A, 1);
      B(2, 0) = B(0, 1) = A2(A, 1);
      B(1, 1) = B(3, 0) = A3(A, 2);
      B(2, 1) = B(0, 2) = A2(A, 2);
      B(3, 1) = B(1, 2) = A3(A, 3);
      B(2, 2) = B(0, 3) = A2(A, 3);
      B(3, 2) = B(1, 3) = A3(A, 4);
      B(2, 3) = A3(A, 5);
      B(3, 3) = A3(A, 6);
      break;
    case B_HD:
      B(3, 0) = A2(E, 0);
      B(3, 1) = A3(E, 1);
      B(2, 0) = B(3, 2) = A2(E, 1);
      B(2, 1) = B(3, 3) = A3(E, 2);
      B(2, 2) = B(1, 0) = A2(E, 2);
      B(2, 3) = B(1, 1) = A3(E, 3);
      B(1, 2) = B(0, 0) = A2(E, 3);
      B(1, 3) = B(0, 1) = A3(E, 4);
      B(0, 2) = A3(E, 5);
      B(0, 3) = A3(E, 6);
      break;
    default: /* B_HU */
      B(0, 0) = A2(L, 0);
      B(0, 1) = A3(L, 1);
      B(0, 2) = B(1, 0) = A2(L, 1);
      B(0, 3) = B(1, 1) = A3(L, 2);
      B(1, 2) = B(2, 0) = A2(L, 2);
      B(1, 3) = B(2, 1) = avg3(L[2], L[3], L[3]);
      B(2, 2) = B(2, 3) = B(3, 0) = B(3, 1) = B(3, 2) = B(3, 3) = L[3];
      break;
  }
#undef B
#undef A3
#undef A2
}

/* predict_y16x16 / predict_uv8x8 (src/intra_predict.rs:371-553): n x n with
 * optional edges (NULL = outside the picture). */
static void predict_block(uint8_t* out, int n, int mode, const uint8_t* above, const uint8_t* left,
                          int p) {
  uint8_t a[16], l[16];
  for (int i = 0; i < n; i++) {
    a[i] = above ? above[i] : 127;
    l[i] = left ? left[i] : 129;
  }
  const int shift = n == 16 ? 4 : 3;
  switch (mode) {
    case YM_DC: {
      int v;
      if (above && left) {
        int s = 0;
        for (int i = 0; i < n; i++) s += above[i] + left[i];
        v = (s + (1 << shift)) >> (shift + 1);
      } else if (above || left) {
        const uint8_t* e = above ? above : left;
        int s = 0;
        for (int i = 0; i < n; i++) s += e[i];
        v = (s + (1 << (shift - 1))) >> shift;
      } else {
        v = 128;
      }
      memset(out, v, (size_t)n * n);
      break;
    }
    case YM_V:
      for (int r = 0; r < n; r++) memcpy(out + r * n, a, n);
      break;
    case YM_H:
      for (int r = 0; r < n; r++) memset(out + r * n, l[r], n);
      break;
    default: /* TM */
      for (int r = 0; r < n; r++)
        for (int c = 0; c < n; c++) out[r * n + c] = clamp255(l[r] + a[c] - p);
      break;
  }
}

/* gather_neighbors (src/frame.rs:288-383) for plane `pl` (0 Y, 1 U, 2 V). */
typedef struct {
  int has_above, has_left;
  uint8_t above[16], left[16], above_right[4];
  int topleft;
} nb_t;

static void gather(const vp8a_planes* f, int row, int col, int pl, nb_t* n) {
  const int sz = pl ? 8 : 16;
  const uint8_t* base = pl == 0 ? f->y : (pl == 1 ? f->u : f->v);
  const size_t st = pl ? f->uv_stride : f->y_stride;
  const int x0 = col * sz, y0 = row * sz;
  n->has_above = row > 0;
  n->has_left = col > 0;
  if (row > 0) memcpy(n->above, base + (size_t)(y0 - 1) * st + x0, sz);
  if (col > 0)
    for (int r = 0; r < sz; r++) n->left[r] = base[(size_t)(y0 + r) * st + x0 - 1];
  if (row == 0) n->topleft = 127;
  else if (col == 0) n->topleft = 129;
  else n->topleft = base[(size_t)(y0 - 1) * st + x0 - 1];
  if (pl == 0) {
    if (row > 0) {
      const uint8_t* ar = base + (size_t)(y0 - 1) * st;
      if ((uint32_t)col == f->mb_cols - 1)
        memset(n->above_right, ar[x0 + 15], 4);
      else
        memcpy(n->above_right, ar + x0 + 16, 4);
    } else {
      memset(n->above_right, 127, 4);
    }
  }
}

/* IDCT of a dequantised 4x4 block added onto the 4x4 block (bi, bj) of an
 * n-wide raster. */
static void idct_add(const int16_t* dq, uint8_t* px, int n, int bi, int bj) {
  int16_t res[16];
  vo_inverse_dct_4x4(dq, res);
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) {
      uint8_t* p = px + (bi * 4 + r) * n + bj * 4 + c;
      *p = clamp255(*p + res[r * 4 + c]);
    }
}

/* Residual of a non-B_PRED MB (Y2 seeding) or an inter MB: the inverse
 * transforms of reconstruct_inter_mb / reconstruct_split_mv_mb /
 * decode_keyframe_mb_non_bpred onto the prediction in `mb` (y 256, u 64,
 * v 64). */
static void add_residual(uint8_t* mb, int16_t* c, int has_y2, int skip_luma_idct) {
  if (has_y2) {
    int16_t dcs[16];
    vo_inverse_wht_4x4(c, dcs);
    for (int b = 0; b < 16; b++) c[16 + 16 * b] = dcs[b];
  }
  if (!skip_luma_idct)
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) idct_add(c + 16 + 16 * (i * 4 + j), mb, 16, i, j);
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) {
      idct_add(c + 272 + 16 * (i * 2 + j), mb + 256, 8, i, j);
      idct_add(c + 336 + 16 * (i * 2 + j), mb + 320, 8, i, j);
    }
}

/* decode_keyframe_mb_bpred's luma (src/reconstruct.rs:466-505 and
 * build_bpred_work_buffer :560-590): a 17 x 21 work buffer holds the
 * above-left, above, above-right and left edges; every 4x4 block predicts
 * from it, adds its residual and writes back, so later blocks see it. */
#define BP_STRIDE 21
static void bpred_luma(const nb_t* n, const uint8_t* modes, int skip, const int16_t* c,
                       uint8_t* out) {
  uint8_t buf[17 * BP_STRIDE];
  memset(buf, 0, sizeof buf);
  buf[0] = (uint8_t)n->topleft;
  for (int i = 0; i < 16; i++) buf[1 + i] = n->has_above ? n->above[i] : 127;
  for (int i = 0; i < 4; i++) buf[17 + i] = n->above_right[i];
  for (int r = 0; r < 16; r++) buf[(r + 1) * BP_STRIDE] = n->has_left ? n->left[r] : 129;
  for (int k = 0; k < 3; k++) memcpy(buf + (1 + 3 + 4 * k) * BP_STRIDE + 17, buf + 17, 4);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      const int sb = (1 + 4 * i) * BP_STRIDE + 1 + 4 * j;
      uint8_t above[8], left[4], pred[16];
      memcpy(above, buf + sb - BP_STRIDE, 8);
      for (int r = 0; r < 4; r++) left[r] = buf[sb + r * BP_STRIDE - 1];
      predict_b4x4(pred, modes[i * 4 + j], above, left, buf[sb - BP_STRIDE - 1]);
      if (!skip) {
        int16_t res[16];
        vo_inverse_dct_4x4(c + 16 + 16 * (i * 4 + j), res);
        for (int k = 0; k < 16; k++) pred[k] = clamp255(pred[k] + res[k]);
      }
      for (int r = 0; r < 4; r++) memcpy(buf + sb + r * BP_STRIDE, pred + 4 * r, 4);
    }
  for (int r = 0; r < 16; r++) memcpy(out + 16 * r, buf + (1 + r) * BP_STRIDE + 1, 16);
}

/* ------------------------------------------------------------- frame decode */

static int alloc_slots(vo_vp8_decoder* d) {
  const size_t ly = (size_t)d->mb_cols * 16 * d->mb_rows * 16, lc = ly / 4;
  for (int s = 0; s < 3; s++) {
    for (int p = 0; p < 3; p++) {
      free(d->slot[s][p]);
      d->slot[s][p] = (uint8_t*)calloc(p ? lc : ly, 1);
      if (!d->slot[s][p]) return -1;
    }
  }
  return 0;
}

static vp8a_planes planes_of(const vo_vp8_decoder* d, uint8_t* y, uint8_t* u, uint8_t* v) {
  vp8a_planes p;
  p.y = y;
  p.u = u;
  p.v = v;
  p.y_stride = (uint64_t)d->mb_cols * 16;
  p.uv_stride = (uint64_t)d->mb_cols * 8;
  p.mb_cols = d->mb_cols;
  p.mb_rows = d->mb_rows;
  return p;
}

/* Vp8DecoderState::decode_frame (src/state.rs:481-1226). Writes the
 * visible picture (w*h luma, then ceil(w/2)*ceil(h/2) U and V) into `out`
 * when it is not NULL; returns 0, or a negative code for a stream the
 * restatement cannot decode (truncated headers, an inter frame first). */
int vo_vp8_decode_frame(vo_vp8_decoder* d, const uint8_t* data, size_t size, uint8_t* out,
                        uint32_t* width, uint32_t* height, int* shown) {
  if (size < 3) return -1;
  hdr_t h;
  memset(&h, 0, sizeof h);
  const uint32_t tag = data[0] | ((uint32_t)data[1] << 8) | ((uint32_t)data[2] << 16);
  h.key = !(tag & 1);
  h.version = (tag >> 1) & 7;
  h.show = (tag >> 4) & 1;
  h.first_size = (tag >> 5) & 0x7ffff;
  h.hdr_bytes = 3;
  if (h.key) {
    if (size < 10 || data[3] != 0x9d || data[4] != 0x01 || data[5] != 0x2a) return -2;
    h.width = (data[6] | (data[7] << 8)) & 0x3fff;
    h.height = (data[8] | (data[9] << 8)) & 0x3fff;
    h.hdr_bytes = 10;
    if (!h.width || !h.height) return -3;
    if (!d->have_key || h.width != d->width || h.height != d->height) {
      d->width = h.width;
      d->height = h.height;
      d->mb_cols = (h.width + 15) / 16;
      d->mb_rows = (h.height + 15) / 16;
      if (alloc_slots(d)) return -4;
    }
  } else if (!d->have_key) {
    return -5;
  }
  if (h.first_size > size - h.hdr_bytes) return -6;
  const int cols = (int)d->mb_cols, rows = (int)d->mb_rows, n_mb = cols * rows;

  /* Probabilities in force for this frame. */
  uint8_t coef[4][8][3][11];
  if (h.key) memcpy(coef, VO_DEFAULT_COEF_PROBS, sizeof coef);
  else memcpy(coef, d->coef, sizeof coef);
  bd_t bd;
  bd_init(&bd, data + h.hdr_bytes, h.first_size);
  parse_header(&bd, &h, coef);
  uint8_t mvc[2][19], ymp[4], uvp[3];
  if (h.key) {
    memcpy(ymp, IF_YMODE_PROB_DEFAULTS, 4);
    memcpy(uvp, IF_UV_MODE_PROB_DEFAULTS, 3);
    memcpy(mvc, DEFAULT_MV_CONTEXT, sizeof mvc);
  } else {
    memcpy(ymp, h.has_ymode_prob ? h.ymode_prob : d->ymode_prob, 4);
    memcpy(uvp, h.has_uvmode_prob ? h.uvmode_prob : d->uvmode_prob, 3);
    memcpy(mvc, d->mvc, sizeof mvc);
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 19; j++)
        if (h.has_mv_update[i][j]) mvc[i][j] = h.mv_update[i][j];
  }

  /* carve_dct_partitions (src/decoder.rs:502-560). */
  const uint8_t* sec = data + h.hdr_bytes + h.first_size;
  size_t sec_len = size - h.hdr_bytes - h.first_size;
  const size_t tbl = (size_t)(h.nparts - 1) * 3;
  if (sec_len < tbl) return -7;
  const uint8_t* body = sec + tbl;
  size_t body_len = sec_len - tbl, off = 0;
  bd_t parts[8];
  for (int i = 0; i < h.nparts; i++) {
    size_t sz;
    if (i < h.nparts - 1) {
      sz = sec[3 * i] | ((size_t)sec[3 * i + 1] << 8) | ((size_t)sec[3 * i + 2] << 16);
      if (off + sz > body_len) return -8;
    } else {
      sz = body_len - off;
    }
    bd_init(&parts[i], body + off, sz);
    off += sz;
  }

  /* resolve_segment_dequant_factors (src/state.rs:1502-1521). */
  int16_t fac[4][6];
  for (int s = 0; s < 4; s++) {
    if (h.segmentation_enabled)
      vo_segment_factors(&h.qi, 1, h.has_quant[s] ? h.quant[s] : 0, h.seg_abs, fac[s]);
    else
      vo_segment_factors(&h.qi, 0, 0, 0, fac[s]);
  }
  const int seg_active = h.segmentation_enabled && h.update_map;
  const int full_pixel = h.version == 3, filter_set = h.version ? 1 : 0;

  const size_t ly = (size_t)cols * 16 * rows * 16, lc = ly / 4;
  uint8_t* cur_y = (uint8_t*)calloc(ly, 1);
  uint8_t* cur_u = (uint8_t*)calloc(lc, 1);
  uint8_t* cur_v = (uint8_t*)calloc(lc, 1);
  mbinfo_t* above_mb = (mbinfo_t*)calloc((size_t)cols, sizeof(mbinfo_t));
  ectx_t* above_ctx = (ectx_t*)calloc((size_t)cols, sizeof(ectx_t));
  uint8_t* above_bm = (uint8_t*)calloc((size_t)cols * 4, 1);
  vp8a_mb_lf_info* lfi = (vp8a_mb_lf_info*)calloc((size_t)n_mb, sizeof(vp8a_mb_lf_info));
  if (!cur_y || !cur_u || !cur_v || !above_mb || !above_ctx || !above_bm || !lfi) {
    free(cur_y), free(cur_u), free(cur_v), free(above_mb), free(above_ctx), free(above_bm), free(lfi);
    return -4;
  }
  vp8a_planes cur = planes_of(d, cur_y, cur_u, cur_v);
  vp8a_planes refp[4];
  refp[VP8A_REF_LAST] = planes_of(d, d->slot[0][0], d->slot[0][1], d->slot[0][2]);
  refp[VP8A_REF_GOLDEN] = planes_of(d, d->slot[1][0], d->slot[1][1], d->slot[1][2]);
  refp[VP8A_REF_ALTREF] = planes_of(d, d->slot[2][0], d->slot[2][1], d->slot[2][2]);
  for (int c = 0; c < cols; c++) above_mb[c].ref = VP8A_REF_INTRA;
  vo_vp8_capture* cap = d->cap;
  if (cap) {
    cap->captured = cap->mb_cols == cols && cap->mb_rows == rows;
    if (!cap->captured) cap = NULL;
  }
  if (cap) {
    for (int s = 0; s < 3; s++)
      for (int p = 0; p < 3; p++) memcpy(cap->refs[s][p], d->slot[s][p], p ? lc : ly);
    for (int p = 0; p < 3; p++) memset(cap->pred[p], 0, p ? lc : ly);
    memset(cap->dec, 0, (size_t)n_mb * sizeof(vp8a_mb_decision));
    cap->key = h.key;
    cap->version = h.version;
  }

  int16_t cf[400];
  uint8_t mb[384];
  for (int row = 0; row < rows; row++) {
    ectx_t left_ctx;
    memset(&left_ctx, 0, sizeof left_ctx);
    mbinfo_t left_mb, al_mb;
    memset(&left_mb, 0, sizeof left_mb);
    memset(&al_mb, 0, sizeof al_mb);
    left_mb.ref = al_mb.ref = VP8A_REF_INTRA;
    uint8_t left_bm[4] = {B_DC, B_DC, B_DC, B_DC};
    bd_t* tok = &parts[row % h.nparts];
    for (int col = 0; col < cols; col++) {
      const int idx = row * cols + col;
      const int seg = seg_active ? bd_tree(&bd, SEGMENT_TREE, h.seg_prob) : -1;
      const int skip = h.no_skip_coeff ? bd_bool(&bd, h.prob_skip) : 0;
      const int16_t* f = fac[seg < 0 ? 0 : seg];
      mbinfo_t info;
      memset(&info, 0, sizeof info);
      info.ref = VP8A_REF_INTRA;
      vp8a_mb_lf_info* L = &lfi[idx];
      memset(L, 0, sizeof *L);
      L->segment_id = (int8_t)seg;
      int is_inter = !h.key && bd_bool(&bd, h.prob_intra);
      if (is_inter) {
        /* select_ref_frame (src/motion_comp.rs:108). */
        const int ref = !bd_bool(&bd, h.prob_last)
                            ? VP8A_REF_LAST
                            : (!bd_bool(&bd, h.prob_gf) ? VP8A_REF_GOLDEN : VP8A_REF_ALTREF);
        vp8a_mv nm[3];
        int cnt[4];
        near_mvs(&h, &above_mb[col], &left_mb, &al_mb, ref, nm, cnt);
        uint8_t p[4];
        for (int i = 0; i < 4; i++) p[i] = MV_COUNTS_TO_PROBS[cnt[i]][i];
        const int mode = bd_tree(&bd, MV_REF_TREE, p); /* Zero, Nearest, Near, New, Split */
        info.ref = (uint8_t)ref;
        L->ref_frame = (uint8_t)ref;
        L->inter_mode = (uint8_t)mode;
        const vp8a_mv best = clamp_mv(nm[0], col, row, cols, rows);
        vp8a_mv mv = {0, 0};
        if (mode == VP8A_MODE_NEAREST) mv = clamp_mv(nm[1], col, row, cols, rows);
        else if (mode == VP8A_MODE_NEAR) mv = clamp_mv(nm[2], col, row, cols, rows);
        else if (mode == VP8A_MODE_NEW) mv = mv_add(best, read_mv(&bd, mvc));
        const int split = mode == VP8A_MODE_SPLIT;
        if (split) {
          decode_split(&bd, &above_mb[col], &left_mb, best, mvc, info.split);
          info.is_split = 1;
          mv = info.split[15];
        }
        info.mv = mv;
        L->y_mode_is_bpred = (uint8_t)split;
        decode_mb_tokens(tok, !split, skip, coef, f, &above_ctx[col], &left_ctx, cf);
        if (split)
          vo_predict_split_mv(&refp[ref], (uint32_t)col, (uint32_t)row, info.split, full_pixel, filter_set, mb);
        else
          vo_predict_inter_mb(&refp[ref], (uint32_t)col, (uint32_t)row, mv, full_pixel, filter_set, mb);
        if (cap) {
          vp8a_mb_decision* dd = &cap->dec[idx];
          dd->ref_frame = (uint8_t)ref;
          dd->mode = (uint8_t)mode;
          dd->mv = mv;
          if (split) memcpy(dd->split_mvs, info.split, sizeof info.split);
          for (int r = 0; r < 16; r++)
            memcpy(cap->pred[0] + ((size_t)row * 16 + r) * cur.y_stride + col * 16, mb + 16 * r, 16);
          for (int r = 0; r < 8; r++) {
            memcpy(cap->pred[1] + ((size_t)row * 8 + r) * cur.uv_stride + col * 8, mb + 256 + 8 * r, 8);
            memcpy(cap->pred[2] + ((size_t)row * 8 + r) * cur.uv_stride + col * 8, mb + 320 + 8 * r, 8);
          }
        }
        if (!skip) add_residual(mb, cf, !split, 0);
      } else {
        if (cap) cap->dec[idx].ref_frame = VP8A_REF_INTRA;
        int ymode, uvmode;
        uint8_t bm[16];
        if (h.key) {
          ymode = bd_tree(&bd, KF_YMODE_TREE, KF_YMODE_PROB);
          if (ymode == YM_B)
            for (int j = 0; j < 16; j++) {
              const int a = (j >> 2) == 0 ? above_bm[col * 4 + (j & 3)] : bm[j - 4];
              const int l = (j & 3) == 0 ? left_bm[j >> 2] : bm[j - 1];
              bm[j] = (uint8_t)bd_tree(&bd, BMODE_TREE, VO_KF_BMODE_PROBS[a][l]);
            }
          uvmode = bd_tree(&bd, UV_MODE_TREE, KF_UV_MODE_PROB);
          /* B-mode contexts for the next MBs (project_to_subblock_context). */
          static const uint8_t proj[4] = {B_DC, B_VE, B_HE, B_TM};
          for (int k = 0; k < 4; k++) {
            above_bm[col * 4 + k] = ymode == YM_B ? bm[12 + k] : proj[ymode];
            left_bm[k] = ymode == YM_B ? bm[4 * k + 3] : proj[ymode];
          }
        } else {
          ymode = bd_tree(&bd, IF_YMODE_TREE, ymp);
          if (ymode == YM_B)
            for (int j = 0; j < 16; j++) bm[j] = (uint8_t)bd_tree(&bd, BMODE_TREE, IF_BMODE_PROB);
          uvmode = bd_tree(&bd, UV_MODE_TREE, uvp);
        }
        L->ref_frame = VP8A_REF_INTRA;
        L->inter_mode = VP8A_MODE_NONE;
        L->y_mode_is_bpred = (uint8_t)(ymode == YM_B);
        decode_mb_tokens(tok, ymode != YM_B, skip, coef, f, &above_ctx[col], &left_ctx, cf);
        nb_t ny, nu, nv;
        gather(&cur, row, col, 0, &ny);
        gather(&cur, row, col, 1, &nu);
        gather(&cur, row, col, 2, &nv);
        if (ymode == YM_B) {
          bpred_luma(&ny, bm, skip, cf, mb);
        } else {
          predict_block(mb, 16, ymode, ny.has_above ? ny.above : NULL, ny.has_left ? ny.left : NULL,
                        ny.topleft);
        }
        predict_block(mb + 256, 8, uvmode, nu.has_above ? nu.above : NULL, nu.has_left ? nu.left : NULL,
                      nu.topleft);
        predict_block(mb + 320, 8, uvmode, nv.has_above ? nv.above : NULL, nv.has_left ? nv.left : NULL,
                      nv.topleft);
        if (!skip) add_residual(mb, cf, ymode != YM_B, ymode == YM_B);
      }
      /* mb_has_coeffs (src/loop_filter.rs:1500) on the dequantised bundle. */
      int has = 0;
      for (int k = 0; k < 400; k++) has |= cf[k] != 0;
      L->has_coeffs = (uint8_t)has;
      /* write_mb (src/frame.rs:404-421). */
      for (int r = 0; r < 16; r++) memcpy(cur_y + ((size_t)row * 16 + r) * cur.y_stride + col * 16, mb + 16 * r, 16);
      for (int r = 0; r < 8; r++) {
        memcpy(cur_u + ((size_t)row * 8 + r) * cur.uv_stride + col * 8, mb + 256 + 8 * r, 8);
        memcpy(cur_v + ((size_t)row * 8 + r) * cur.uv_stride + col * 8, mb + 320 + 8 * r, 8);
      }
      al_mb = above_mb[col];
      left_mb = info;
      above_mb[col] = info;
    }
  }

  /* FrameFilterConfig::keyframe / ::interframe (src/loop_filter.rs:1077-1190). */
  vp8a_filter_config lc_;
  memset(&lc_, 0, sizeof lc_);
  lc_.simple = (uint8_t)h.filter_type;
  lc_.key_frame = (uint8_t)h.key;
  lc_.loop_filter_level = (uint8_t)h.level;
  lc_.sharpness_level = (uint8_t)h.sharpness;
  lc_.segmentation_enabled = (uint8_t)h.segmentation_enabled;
  if (h.segmentation_enabled) {
    lc_.segment_abs = (uint8_t)h.seg_abs;
    for (int i = 0; i < 4; i++) lc_.segment_lf_level[i] = (int16_t)(h.has_lf[i] ? h.lf[i] : 0);
  }
  lc_.delta_enabled = (uint8_t)h.lf_adj_enable;
  int16_t rd[4], md[4];
  if (h.key) {
    for (int i = 0; i < 4; i++) rd[i] = md[i] = 0;
    if (h.lf_adj_enable)
      for (int i = 0; i < 4; i++) {
        if (h.has_ref_delta[i]) rd[i] = (int16_t)h.ref_delta[i];
        if (h.has_mode_delta[i]) md[i] = (int16_t)h.mode_delta[i];
      }
    lc_.ref_delta_current = rd[0];
    lc_.bpred_mode_delta = md[0];
  } else {
    memcpy(rd, d->ref_lf_deltas, sizeof rd);
    memcpy(md, d->mode_lf_deltas, sizeof md);
    if (h.lf_adj_enable)
      for (int i = 0; i < 4; i++) {
        if (h.has_ref_delta[i]) rd[i] = (int16_t)h.ref_delta[i];
        if (h.has_mode_delta[i]) md[i] = (int16_t)h.mode_delta[i];
      }
    lc_.ref_delta_current = rd[0];
    lc_.bpred_mode_delta = md[0];
    lc_.ref_delta_last = rd[1];
    lc_.ref_delta_golden = rd[2];
    lc_.ref_delta_altref = rd[3];
    lc_.zero_mv_mode_delta = md[1];
    lc_.other_mv_mode_delta = md[2];
    lc_.split_mv_mode_delta = md[3];
  }
  memcpy(d->ref_lf_deltas, rd, sizeof rd);
  memcpy(d->mode_lf_deltas, md, sizeof md);
  if (cap) {
    memcpy(cap->pre[0], cur_y, ly);
    memcpy(cap->pre[1], cur_u, lc);
    memcpy(cap->pre[2], cur_v, lc);
    memcpy(cap->lf, lfi, (size_t)n_mb * sizeof(vp8a_mb_lf_info));
    *cap->cfg = lc_;
    cap->filtered = h.level != 0;
  }
  if (h.level != 0) vo_filter_frame(&cur, lfi, &lc_);
  if (cap) {
    memcpy(cap->post[0], cur_y, ly);
    memcpy(cap->post[1], cur_u, lc);
    memcpy(cap->post[2], cur_v, lc);
  }

  /* Probability carry (src/state.rs:628-640, :1163-1171). */
  if (h.key) {
    if (h.refresh_entropy) memcpy(d->coef, coef, sizeof coef);
    else memcpy(d->coef, VO_DEFAULT_COEF_PROBS, sizeof coef);
    memcpy(d->ymode_prob, IF_YMODE_PROB_DEFAULTS, 4);
    memcpy(d->uvmode_prob, IF_UV_MODE_PROB_DEFAULTS, 3);
    memcpy(d->mvc, DEFAULT_MV_CONTEXT, sizeof d->mvc);
    d->sign_bias_golden = d->sign_bias_altref = 0;
  } else {
    if (h.refresh_entropy) {
      memcpy(d->coef, coef, sizeof coef);
      memcpy(d->mvc, mvc, sizeof mvc);
      memcpy(d->ymode_prob, ymp, 4);
      memcpy(d->uvmode_prob, uvp, 3);
    }
    d->sign_bias_golden = h.sign_bias_golden;
    d->sign_bias_altref = h.sign_bias_altref;
  }

  /* Visible picture (crop_to_visible, src/decoder.rs:692). */
  const uint32_t w = d->width, hh = d->height, cw = (w + 1) / 2, ch = (hh + 1) / 2;
  if (out) {
    for (uint32_t r = 0; r < hh; r++) memcpy(out + (size_t)r * w, cur_y + (size_t)r * cur.y_stride, w);
    uint8_t* ou = out + (size_t)w * hh;
    uint8_t* ov = ou + (size_t)cw * ch;
    for (uint32_t r = 0; r < ch; r++) {
      memcpy(ou + (size_t)r * cw, cur_u + (size_t)r * cur.uv_stride, cw);
      memcpy(ov + (size_t)r * cw, cur_v + (size_t)r * cur.uv_stride, cw);
    }
  }
  if (width) *width = w;
  if (height) *height = hh;
  if (shown) *shown = h.show;

  /* Reference update: key frames fill all three slots; inter frames
   * rotate_reference_slots (src/state.rs:154-268). */
  uint8_t* cur_p[3] = {cur_y, cur_u, cur_v};
  const size_t psz[3] = {ly, lc, lc};
  if (h.key) {
    for (int s = 0; s < 3; s++)
      for (int p = 0; p < 3; p++) memcpy(d->slot[s][p], cur_p[p], psz[p]);
  } else {
    /* Sources: 0 = previous LAST, 1 = previous GOLDEN, 2 = previous ALTREF, 3 = current. */
    int src_alt = h.copy_to_altref == 1 ? 0 : (h.copy_to_altref == 2 ? 1 : 2);
    int src_gold = h.copy_to_golden == 1 ? 0 : (h.copy_to_golden == 2 ? 2 : 1);
    if (h.refresh_golden) src_gold = 3;
    if (h.refresh_altref) src_alt = 3;
    const int src_last = h.refresh_last ? 3 : 0;
    const int src[3] = {src_last, src_gold, src_alt};
    uint8_t* nw[3][3];
    for (int s = 0; s < 3; s++)
      for (int p = 0; p < 3; p++) {
        nw[s][p] = (uint8_t*)malloc(psz[p]);
        memcpy(nw[s][p], src[s] == 3 ? cur_p[p] : d->slot[src[s]][p], psz[p]);
      }
    for (int s = 0; s < 3; s++)
      for (int p = 0; p < 3; p++) {
        free(d->slot[s][p]);
        d->slot[s][p] = nw[s][p];
      }
  }
  d->have_key = 1;
  free(cur_y), free(cur_u), free(cur_v), free(above_mb), free(above_ctx), free(above_bm), free(lfi);
  return 0;
}
