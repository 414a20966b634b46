/*
 * recon.c — oracle restatement of the §14 inter reconstruction the encoder
 * runs after its mode decision, with the trellis off.
 *
 * TEST INFRASTRUCTURE ONLY (see vp8a_oracle.h). Follows:
 *   DC_QLOOKUP / AC_QLOOKUP, clamp_qindex      src/inverse_transform.rs:72-107
 *   MbDequantFactors::from_base_and_deltas,
 *     for_segment, dequantize, dequant_block   src/dequant.rs:118-290
 *   forward_dct_4x4_scalar, forward_wht_4x4,
 *     c_mul, s_mul, round_div2                 src/forward_transform.rs:134-260, :486-604, :765-790
 *   inverse_wht_4x4_scalar                     src/inverse_transform.rs:190-252
 *   inverse_dct_4x4_scalar (wrapping i32)      src/inverse_transform.rs:609-712
 *   add_residue_4x4                            src/inverse_transform.rs:871
 *   enc_round_div, enc_quantize_block          src/encoder.rs:2112-2132
 *   transform_whole_block_luma_rd              src/encoder.rs:3815-3885
 *   transform_chroma_plane_rd                  src/encoder.rs:4133-4172
 *   transform_split_mv_mb_rd                   src/encoder.rs:8259-8315
 *   I420Frame::extract_mb                      src/encoder.rs:5526-5586
 *   the §18/§14 step of pick_mb_for_ref        src/encoder.rs:8704-8800
 *     (skip detection, dequantise, reconstruct_inter_mb /
 *      reconstruct_split_mv_mb, src/motion_comp.rs:2098-2160, :2340-2386)
 *   mb_has_coeffs                              src/loop_filter.rs:1500
 * TrellisStrength::OFF (src/encoder.rs:2677) makes every block take
 * enc_quantize_block, the plain round-half-away-from-zero quantiser.
 */
#include <string.h>

#include "vp8a_oracle.h"

static const int16_t DC_Q[128] = {
    4,   5,   6,   7,   8,   9,   10,  10,  11,  12,  13,  14,  15,  16,  17,  17,  18,  19,  20,
    20,  21,  21,  22,  22,  23,  23,  24,  25,  25,  26,  27,  28,  29,  30,  31,  32,  33,  34,
    35,  36,  37,  37,  38,  39,  40,  41,  42,  43,  44,  45,  46,  46,  47,  48,  49,  50,  51,
    52,  53,  54,  55,  56,  57,  58,  59,  60,  61,  62,  63,  64,  65,  66,  67,  68,  69,  70,
    71,  72,  73,  74,  75,  76,  76,  77,  78,  79,  80,  81,  82,  83,  84,  85,  86,  87,  88,
    89,  91,  93,  95,  96,  98,  100, 101, 102, 104, 106, 108, 110, 112, 114, 116, 118, 122, 124,
    126, 128, 130, 132, 134, 136, 138, 140, 143, 145, 148, 151, 154, 157};

static const int16_t AC_Q[128] = {
    4,   5,   6,   7,   8,   9,   10,  11,  12,  13,  14,  15,  16,  17,  18,  19,  20,  21,  22,
    23,  24,  25,  26,  27,  28,  29,  30,  31,  32,  33,  34,  35,  36,  37,  38,  39,  40,  41,
    42,  43,  44,  45,  46,  47,  48,  49,  50,  51,  52,  53,  54,  55,  56,  57,  58,  60,  62,
    64,  66,  68,  70,  72,  74,  76,  78,  80,  82,  84,  86,  88,  90,  92,  94,  96,  98,  100,
    102, 104, 106, 108, 110, 112, 114, 116, 119, 122, 125, 128, 131, 134, 137, 140, 143, 146, 149,
    152, 155, 158, 161, 164, 167, 170, 173, 177, 181, 185, 189, 193, 197, 201, 205, 209, 213, 217,
    221, 225, 229, 234, 239, 245, 249, 254, 259, 264, 269, 274, 279, 284};

#define COSPI8_SQRT2_MINUS1 20091
#define SINPI8_SQRT2 35468

static inline int clamp_qindex(int64_t q) { return q < 0 ? 0 : (q > 127 ? 127 : (int)q); }
static inline int64_t sat_add(int64_t a, int64_t b) {
  int64_t s = a + b;  /* i32 saturating add of the reference, widened */
  return s > 2147483647LL ? 2147483647LL : (s < -2147483648LL ? -2147483648LL : s);
}

/* MbDequantFactors::from_base_and_deltas (src/dequant.rs:118-165): out =
 * {y1_dc, y1_ac, y2_dc, y2_ac, uv_dc, uv_ac}. */
void vo_dequant_factors(int32_t q, int32_t ydc, int32_t y2dc, int32_t y2ac, int32_t uvdc,
                        int32_t uvac, int16_t* out) {
  int y1_dc = DC_Q[clamp_qindex(sat_add(q, ydc))];
  int y1_ac = AC_Q[clamp_qindex(q)];
  int y2_dc = DC_Q[clamp_qindex(sat_add(q, y2dc))] * 2;
  int y2_ac = AC_Q[clamp_qindex(sat_add(q, y2ac))] * 155 / 100;
  if (y2_ac < 8) y2_ac = 8;
  int uv_dc = DC_Q[clamp_qindex(sat_add(q, uvdc))];
  if (uv_dc > 132) uv_dc = 132;
  int uv_ac = AC_Q[clamp_qindex(sat_add(q, uvac))];
  out[0] = (int16_t)y1_dc;
  out[1] = (int16_t)y1_ac;
  out[2] = (int16_t)y2_dc;
  out[3] = (int16_t)y2_ac;
  out[4] = (int16_t)uv_dc;
  out[5] = (int16_t)uv_ac;
}

/* MbDequantFactors::from_quant_indices / for_segment (src/dequant.rs:169-230). */
void vo_segment_factors(const vp8a_quant_indices* qi, int has_segment, int32_t segment_quant,
                        int absolute, int16_t* out) {
  int32_t q = qi->y_ac_qi;
  if (has_segment) q = absolute ? segment_quant : (int32_t)sat_add(qi->y_ac_qi, segment_quant);
  vo_dequant_factors(q, qi->y_dc_delta, qi->y2_dc_delta, qi->y2_ac_delta, qi->uv_dc_delta,
                     qi->uv_ac_delta, out);
}

static inline int c_mul(int i) { return i + ((i * COSPI8_SQRT2_MINUS1) >> 16); }
static inline int s_mul(int i) { return (i * SINPI8_SQRT2) >> 16; }

static inline int16_t round_div2(int v) {
  int r = v >= 0 ? (v + 1) >> 1 : -((-v + 1) >> 1);
  return (int16_t)(r < -32768 ? -32768 : (r > 32767 ? 32767 : r));
}

/* forward_dct_4x4_scalar (src/forward_transform.rs:486-604). */
void vo_forward_dct_4x4(const int16_t* in, int16_t* out) {
  int tmp[16];
  for (int col = 0; col < 4; col++) {
    int i0 = in[col], i4 = in[4 + col], i8 = in[8 + col], i12 = in[12 + col];
    int a1 = i0 + i12, b1 = i4 + i8;
    int c1 = (c_mul(i0) - c_mul(i12)) + (s_mul(i4) - s_mul(i8));
    int d1 = (s_mul(i0) - s_mul(i12)) - (c_mul(i4) - c_mul(i8));
    tmp[col] = a1 + b1;
    tmp[4 + col] = c1;
    tmp[8 + col] = a1 - b1;
    tmp[12 + col] = d1;
  }
  for (int row = 0; row < 4; row++) {
    int r0 = tmp[row * 4], r1 = tmp[row * 4 + 1], r2 = tmp[row * 4 + 2], r3 = tmp[row * 4 + 3];
    int a1 = r0 + r3, b1 = r1 + r2;
    int c1 = (c_mul(r0) - c_mul(r3)) + (s_mul(r1) - s_mul(r2));
    int d1 = (s_mul(r0) - s_mul(r3)) - (c_mul(r1) - c_mul(r2));
    out[row * 4] = round_div2(a1 + b1);
    out[row * 4 + 1] = round_div2(c1);
    out[row * 4 + 2] = round_div2(a1 - b1);
    out[row * 4 + 3] = round_div2(d1);
  }
}

/* forward_wht_4x4_scalar (src/forward_transform.rs:173-260). */
void vo_forward_wht_4x4(const int16_t* in, int16_t* out) {
  int tmp[16];
  for (int col = 0; col < 4; col++) {
    int i0 = in[col], i4 = in[4 + col], i8 = in[8 + col], i12 = in[12 + col];
    int a1 = i0 + i12, b1 = i4 + i8, c1 = i4 - i8, d1 = i0 - i12;
    tmp[col] = a1 + b1;
    tmp[4 + col] = c1 + d1;
    tmp[8 + col] = a1 - b1;
    tmp[12 + col] = d1 - c1;
  }
  for (int row = 0; row < 4; row++) {
    int r0 = tmp[row * 4], r1 = tmp[row * 4 + 1], r2 = tmp[row * 4 + 2], r3 = tmp[row * 4 + 3];
    int a1 = r0 + r3, b1 = r1 + r2, c1 = r1 - r2, d1 = r0 - r3;
    out[row * 4] = round_div2(a1 + b1);
    out[row * 4 + 1] = round_div2(c1 + d1);
    out[row * 4 + 2] = round_div2(a1 - b1);
    out[row * 4 + 3] = round_div2(d1 - c1);
  }
}

/* inverse_wht_4x4_scalar (src/inverse_transform.rs:190-252). */
void vo_inverse_wht_4x4(const int16_t* in, int16_t* out) {
  int tmp[16];
  for (int col = 0; col < 4; col++) {
    int i0 = in[col], i4 = in[4 + col], i8 = in[8 + col], i12 = in[12 + col];
    int a1 = i0 + i12, b1 = i4 + i8, c1 = i4 - i8, d1 = i0 - i12;
    tmp[col] = a1 + b1;
    tmp[4 + col] = c1 + d1;
    tmp[8 + col] = a1 - b1;
    tmp[12 + col] = d1 - c1;
  }
  for (int row = 0; row < 4; row++) {
    int r0 = tmp[row * 4], r1 = tmp[row * 4 + 1], r2 = tmp[row * 4 + 2], r3 = tmp[row * 4 + 3];
    int a1 = r0 + r3, b1 = r1 + r2, c1 = r1 - r2, d1 = r0 - r3;
    int a2 = a1 + b1, b2 = c1 + d1, c2 = a1 - b1, d2 = d1 - c1;
    out[row * 4] = (int16_t)((a2 + 3) >> 3);
    out[row * 4 + 1] = (int16_t)((b2 + 3) >> 3);
    out[row * 4 + 2] = (int16_t)((c2 + 3) >> 3);
    out[row * 4 + 3] = (int16_t)((d2 + 3) >> 3);
  }
}

/* Two's-complement i32 arithmetic of the reference's wrapping_* ops. */
static inline int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static inline int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
static inline int32_t wmul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }

/* inverse_dct_4x4_scalar (src/inverse_transform.rs:609-712). */
void vo_inverse_dct_4x4(const int16_t* in, int16_t* out) {
  int32_t tmp[16];
  for (int col = 0; col < 4; col++) {
    int32_t i0 = in[col], i4 = in[4 + col], i8 = in[8 + col], i12 = in[12 + col];
    int32_t a1 = wadd(i0, i8), b1 = wsub(i0, i8);
    int32_t t1 = wmul(i4, SINPI8_SQRT2) >> 16;
    int32_t t2 = wadd(i12, wmul(i12, COSPI8_SQRT2_MINUS1) >> 16);
    int32_t c1 = wsub(t1, t2);
    t1 = wadd(i4, wmul(i4, COSPI8_SQRT2_MINUS1) >> 16);
    t2 = wmul(i12, SINPI8_SQRT2) >> 16;
    int32_t d1 = wadd(t1, t2);
    tmp[col] = wadd(a1, d1);
    tmp[12 + col] = wsub(a1, d1);
    tmp[4 + col] = wadd(b1, c1);
    tmp[8 + col] = wsub(b1, c1);
  }
  for (int row = 0; row < 4; row++) {
    int32_t r0 = tmp[row * 4], r1 = tmp[row * 4 + 1], r2 = tmp[row * 4 + 2], r3 = tmp[row * 4 + 3];
    int32_t a1 = wadd(r0, r2), b1 = wsub(r0, r2);
    int32_t t1 = wmul(r1, SINPI8_SQRT2) >> 16;
    int32_t t2 = wadd(r3, wmul(r3, COSPI8_SQRT2_MINUS1) >> 16);
    int32_t c1 = wsub(t1, t2);
    t1 = wadd(r1, wmul(r1, COSPI8_SQRT2_MINUS1) >> 16);
    t2 = wmul(r3, SINPI8_SQRT2) >> 16;
    int32_t d1 = wadd(t1, t2);
    out[row * 4] = (int16_t)(wadd(wadd(a1, d1), 4) >> 3);
    out[row * 4 + 3] = (int16_t)(wadd(wsub(a1, d1), 4) >> 3);
    out[row * 4 + 1] = (int16_t)(wadd(wadd(b1, c1), 4) >> 3);
    out[row * 4 + 2] = (int16_t)(wadd(wsub(b1, c1), 4) >> 3);
  }
}

/* enc_round_div (src/encoder.rs:2112-2120). */
static inline int16_t enc_round_div(int32_t num, int32_t den) {
  int32_t r = num >= 0 ? (num + den / 2) / den : -(((-num) + den / 2) / den);
  return (int16_t)r;
}

/* enc_quantize_block (src/encoder.rs:2127-2132). */
void vo_enc_quantize_block(int16_t* blk, int16_t dc, int16_t ac) {
  blk[0] = enc_round_div(blk[0], dc);
  for (int i = 1; i < 16; i++) blk[i] = enc_round_div(blk[i], ac);
}

/* dequant_block_scalar (src/dequant.rs:284-290). */
static void dequant_block(int16_t* blk, int16_t dc, int16_t ac) {
  blk[0] = (int16_t)((int32_t)blk[0] * dc);
  for (int i = 1; i < 16; i++) blk[i] = (int16_t)((int32_t)blk[i] * ac);
}

static inline uint8_t clamp255(int v) { return (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v)); }

/* I420Frame::extract_mb (src/encoder.rs:5526-5586): 16x16 luma and two 8x8
 * chroma blocks, edge-replicated past the visible picture. */
static void extract_mb(const vp8a_i420* f, size_t mb_row, size_t mb_col, uint8_t* y, uint8_t* u,
                       uint8_t* v) {
  const size_t w = f->width, h = f->height, cw = (w + 1) / 2, ch = (h + 1) / 2;
  for (int r = 0; r < 16; r++)
    for (int c = 0; c < 16; c++) {
      size_t x = mb_col * 16 + c, yy = mb_row * 16 + r;
      if (x > w - 1) x = w - 1;
      if (yy > h - 1) yy = h - 1;
      y[r * 16 + c] = f->y[yy * f->y_stride + x];
    }
  for (int r = 0; r < 8; r++)
    for (int c = 0; c < 8; c++) {
      size_t x = mb_col * 8 + c, yy = mb_row * 8 + r;
      if (x > cw - 1) x = cw - 1;
      if (yy > ch - 1) yy = ch - 1;
      u[r * 8 + c] = f->u[yy * f->uv_stride + x];
      v[r * 8 + c] = f->v[yy * f->uv_stride + x];
    }
}

/* Residual of the 4x4 block (bi, bj) of an n-wide block. */
static void residual_4x4(const uint8_t* src, const uint8_t* pred, int n, int bi, int bj,
                         int16_t* out) {
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) {
      int off = (bi * 4 + r) * n + bj * 4 + c;
      out[r * 4 + c] = (int16_t)((int)src[off] - (int)pred[off]);
    }
}

/* IDCT of a dequantised block, added onto the 4x4 block (bi, bj) of an
 * n-wide raster (inverse_dct_4x4 + add_residue_4x4). */
static void idct_add(const int16_t* dq, uint8_t* plane, int n, int bi, int bj) {
  int16_t res[16];
  vo_inverse_dct_4x4(dq, res);
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) {
      uint8_t* p = plane + (bi * 4 + r) * n + bj * 4 + c;
      *p = clamp255((int)*p + res[r * 4 + c]);
    }
}

/* The §14 half of pick_mb_for_ref's chosen-mode step (src/encoder.rs:8704-8800)
 * for one MB with the trellis off. `pred` holds the §18 prediction (y 256,
 * u 64, v 64) and receives the reconstruction. coeffs gets the quantised
 * MbCoeffs (y2[16], y[16][16], u[4][16], v[4][16]); returns bit 0 = the
 * §11.1 mb_skip_coeff, bit 1 = mb_has_coeffs. */
void vo_trellis_quantize_block(int16_t* block, int16_t dc, int16_t ac, int first_coeff, int entry_ctx3, int plane,
                               double lambda);

/* Quantise one block: plain rounding, or the §13 trellis when tlambda > 0
 * (every inter call site uses entry context 0; planes are BlockType
 * indices: 0 YAfterY2, 1 Y2, 2 UV, 3 YNoY2). */
static void quantize(int16_t* blk, int16_t dc, int16_t ac, int first_coeff, int plane, double tlambda) {
  if (tlambda > 0.0) vo_trellis_quantize_block(blk, dc, ac, first_coeff, 0, plane, tlambda);
  else vo_enc_quantize_block(blk, dc, ac);
}

int vo_reconstruct_inter_mb_trellis(const uint8_t* src384, uint8_t* pred, const int16_t* f, int split,
                                    int16_t* coeffs, double tlambda);

int vo_reconstruct_inter_mb(const uint8_t* src384, uint8_t* pred, const int16_t* f, int split,
                            int16_t* coeffs) {
  return vo_reconstruct_inter_mb_trellis(src384, pred, f, split, coeffs, 0.0);
}

/* vo_reconstruct_inter_mb with the §13 trellis at `tlambda`
 * (MbRdCtx::trellis_lambda; 0 = plain rounding). */
int vo_reconstruct_inter_mb_trellis(const uint8_t* src384, uint8_t* pred, const int16_t* f, int split,
                                    int16_t* coeffs, double tlambda) {
  int16_t* y2 = coeffs;
  int16_t* y = coeffs + 16;
  int16_t* u = coeffs + 272;
  int16_t* v = coeffs + 336;
  memset(coeffs, 0, 400 * sizeof(int16_t));
  /* transform_whole_block_luma_rd / transform_split_mv_mb_rd */
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      int16_t res[16];
      residual_4x4(src384, pred, 16, i, j, res);
      vo_forward_dct_4x4(res, y + (i * 4 + j) * 16);
    }
  if (!split) {
    int16_t dcs[16];
    for (int b = 0; b < 16; b++) {
      dcs[b] = y[b * 16];
      y[b * 16] = 0;
    }
    vo_forward_wht_4x4(dcs, y2);
    quantize(y2, f[2], f[3], 0, 1, tlambda);
  }
  for (int b = 0; b < 16; b++) quantize(y + b * 16, f[0], f[1], split ? 0 : 1, split ? 3 : 0, tlambda);
  /* transform_chroma_plane_rd, U then V */
  for (int p = 0; p < 2; p++) {
    int16_t* dst = p ? v : u;
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) {
        int16_t res[16];
        residual_4x4(src384 + 256 + 64 * p, pred + 256 + 64 * p, 8, i, j, res);
        vo_forward_dct_4x4(res, dst + (i * 2 + j) * 16);
        quantize(dst + (i * 2 + j) * 16, f[4], f[5], 0, 2, tlambda);
      }
  }
  /* §11.1 skip detection (src/encoder.rs:8745-8769) */
  int nonzero = 0;
  if (split == 0)
    for (int k = 0; k < 16; k++) nonzero += y2[k] != 0;
  for (int b = 0; b < 16; b++)
    for (int k = split ? 0 : 1; k < 16; k++) nonzero += y[b * 16 + k] != 0;
  for (int k = 0; k < 128; k++) nonzero += u[k] != 0;
  const int skip = nonzero == 0;
  /* factors.dequantize on a copy (src/dequant.rs:240-252) */
  int16_t dq[400];
  memcpy(dq, coeffs, sizeof dq);
  dequant_block(dq, f[2], f[3]);
  for (int b = 0; b < 16; b++) dequant_block(dq + 16 + b * 16, f[0], f[1]);
  for (int b = 0; b < 8; b++) dequant_block(dq + 272 + b * 16, f[4], f[5]);
  int has = 0;
  for (int k = 0; k < 400; k++) has |= dq[k] != 0;
  if (!skip) {
    /* reconstruct_inter_mb / reconstruct_split_mv_mb */
    if (!split) {
      int16_t dcs[16];
      vo_inverse_wht_4x4(dq, dcs);
      for (int b = 0; b < 16; b++) dq[16 + b * 16] = dcs[b];
    }
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) idct_add(dq + 16 + (i * 4 + j) * 16, pred, 16, i, j);
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) {
        idct_add(dq + 272 + (i * 2 + j) * 16, pred + 256, 8, i, j);
        idct_add(dq + 336 + (i * 2 + j) * 16, pred + 320, 8, i, j);
      }
  }
  return skip | (has << 1);
}

/* The chosen-mode §18 + §14 step for every MB of a frame: predict_split_mv
 * / predict_inter_mb from the decision's reference, then
 * vo_reconstruct_inter_mb, written into the MB-padded `out` planes.
 * mb_segment (optional) selects per-MB factors: -1 = the frame's, k = the
 * segment quant segment_quant[k] (absolute or a delta). lf (optional)
 * receives each MB's §15 side information. MBs without an inter reference
 * are left untouched (flags 0, their lf record kept). Every MB is
 * independent, so MB rows are spread over `threads` (same outputs for any
 * count). Returns the number of MBs left untouched. */
typedef struct {
  const vp8a_i420* frame;
  const vp8a_planes* refs;
  const uint8_t* ref_ids;
  uint32_t n_refs;
  const vp8a_mb_decision* dec;
  const int8_t* mb_segment;
  int16_t fset[5][6];
  double tlambda[5];
  int full_pixel, filter_set;
  vp8a_planes* out;
  int16_t* coeffs;
  uint8_t* flags;
  vp8a_mb_lf_info* lf;
  _Atomic int skipped;
} recon_job;

static void recon_row(void* arg, uint32_t row) {
  recon_job* j = (recon_job*)arg;
  vp8a_planes* out = j->out;
  uint8_t src[384], mb[384];
  int16_t cf[400];
  for (uint32_t col = 0; col < out->mb_cols; col++) {
    const size_t idx = (size_t)row * out->mb_cols + col;
    const vp8a_mb_decision* d = &j->dec[idx];
    const vp8a_planes* ref = NULL;
    for (uint32_t k = 0; k < j->n_refs; k++)
      if (d->ref_frame != VP8A_REF_INTRA && j->ref_ids[k] == d->ref_frame) ref = &j->refs[k];
    if (!ref) {
      j->skipped++;
      if (j->flags) j->flags[idx] = 0;
      continue;
    }
    const int split = d->mode == VP8A_MODE_SPLIT;
    if (split)
      vo_predict_split_mv(ref, col, row, d->split_mvs, j->full_pixel, j->filter_set, mb);
    else
      vo_predict_inter_mb(ref, col, row, d->mv, j->full_pixel, j->filter_set, mb);
    extract_mb(j->frame, row, col, src, src + 256, src + 320);
    const int seg = j->mb_segment ? j->mb_segment[idx] : -1;
    const int16_t* f = j->fset[(seg >= 0 && seg < 4) ? 1 + seg : 0];
    const int fl = vo_reconstruct_inter_mb_trellis(src, mb, f, split, cf,
                                                   j->tlambda[(seg >= 0 && seg < 4) ? 1 + seg : 0]);
    if (j->flags) j->flags[idx] = (uint8_t)fl;
    if (j->lf) {
      /* The §15 side information of the MB (SPLITMV as B_PRED,
       * src/loop_filter.rs:1258-1266). */
      memset(&j->lf[idx], 0, sizeof j->lf[idx]);
      j->lf[idx].y_mode_is_bpred = (uint8_t)split;
      j->lf[idx].has_coeffs = (uint8_t)(fl >> 1);
      j->lf[idx].ref_frame = d->ref_frame;
      j->lf[idx].inter_mode = d->mode;
      j->lf[idx].segment_id = (int8_t)seg;
    }
    if (j->coeffs) memcpy(j->coeffs + idx * 400, cf, sizeof cf);
    for (int r = 0; r < 16; r++)
      memcpy(out->y + ((size_t)row * 16 + r) * out->y_stride + (size_t)col * 16, mb + r * 16, 16);
    for (int r = 0; r < 8; r++) {
      memcpy(out->u + ((size_t)row * 8 + r) * out->uv_stride + (size_t)col * 8, mb + 256 + r * 8, 8);
      memcpy(out->v + ((size_t)row * 8 + r) * out->uv_stride + (size_t)col * 8, mb + 320 + r * 8, 8);
    }
  }
}

double vo_trellis_lambda(int16_t y1_ac, double strength);

int vo_reconstruct_inter_frame_trellis(const vp8a_i420* frame, const vp8a_planes* refs,
                                       const uint8_t* ref_ids, uint32_t n_refs,
                                       const vp8a_mb_decision* dec, const vp8a_quant_indices* qi,
                                       const int8_t* mb_segment, const int16_t* segment_quant,
                                       int segment_abs, int full_pixel, int filter_set,
                                       vp8a_planes* out, int16_t* coeffs, uint8_t* flags,
                                       vp8a_mb_lf_info* lf, double trellis_strength, uint32_t threads);

int vo_reconstruct_inter_frame(const vp8a_i420* frame, const vp8a_planes* refs,
                               const uint8_t* ref_ids, uint32_t n_refs,
                               const vp8a_mb_decision* dec, const vp8a_quant_indices* qi,
                               const int8_t* mb_segment, const int16_t* segment_quant,
                               int segment_abs, int full_pixel, int filter_set,
                               vp8a_planes* out, int16_t* coeffs, uint8_t* flags,
                               vp8a_mb_lf_info* lf, uint32_t threads) {
  return vo_reconstruct_inter_frame_trellis(frame, refs, ref_ids, n_refs, dec, qi, mb_segment, segment_quant,
                                            segment_abs, full_pixel, filter_set, out, coeffs, flags, lf, 0.0,
                                            threads);
}

/* vo_reconstruct_inter_frame with the §13 trellis at TrellisStrength
 * `trellis_strength` (clamped to 0..=8, NaN = 1.0; 0 = off): each factor
 * set's trellis lambda is rd_lambda(factors) * strength * 0.04. */
int vo_reconstruct_inter_frame_trellis(const vp8a_i420* frame, const vp8a_planes* refs,
                                       const uint8_t* ref_ids, uint32_t n_refs,
                                       const vp8a_mb_decision* dec, const vp8a_quant_indices* qi,
                                       const int8_t* mb_segment, const int16_t* segment_quant,
                                       int segment_abs, int full_pixel, int filter_set,
                                       vp8a_planes* out, int16_t* coeffs, uint8_t* flags,
                                       vp8a_mb_lf_info* lf, double trellis_strength, uint32_t threads) {
  recon_job j;
  memset(&j, 0, sizeof j);
  j.frame = frame;
  j.refs = refs;
  j.ref_ids = ref_ids;
  j.n_refs = n_refs;
  j.dec = dec;
  j.mb_segment = mb_segment;
  vo_segment_factors(qi, 0, 0, 0, j.fset[0]);
  for (int k = 0; k < 4; k++)
    vo_segment_factors(qi, 1, segment_quant ? segment_quant[k] : 0, segment_abs, j.fset[1 + k]);
  double s = trellis_strength != trellis_strength ? 1.0 : trellis_strength;
  s = s < 0.0 ? 0.0 : (s > 8.0 ? 8.0 : s);
  for (int k = 0; k < 5; k++) j.tlambda[k] = vo_trellis_lambda(j.fset[k][1], s);
  j.full_pixel = full_pixel;
  j.filter_set = filter_set;
  j.out = out;
  j.coeffs = coeffs;
  j.flags = flags;
  j.lf = lf;
  vo_parallel_for(out->mb_rows, threads, recon_row, &j);
  return j.skipped;
}
