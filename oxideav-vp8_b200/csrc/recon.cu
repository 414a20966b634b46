// recon.cu — the §14 inter reconstruction of the encoder's chosen mode
// (trellis off) on the GPU:
//   vp8a_reconstruct_inter_frame  (the §18 + §14 step of pick_mb_for_ref,
//                                  src/encoder.rs:8704-8800, TrellisStrength::OFF)
//   vp8a_dequant_factors          (MbDequantFactors, src/dequant.rs:118-230; host)
//
// The prediction is queued first (predict.cu) into the output planes; this
// kernel then turns each MB's prediction into its reconstruction in place.
// One warp per MB, one lane per 4x4 block: lanes 0-15 the luma blocks in
// raster order, 16-19 U, 20-23 V, lane 24 the Y2 block of a non-SPLITMV MB.
// A lane forms its block's residual against the source MB (edge-replicated
// as I420Frame::extract_mb does), runs the forward DCT, hands its DC to lane
// 24 for the forward WHT (non-SPLITMV), quantises with the plain rounding
// quantiser, votes on the §11.1 skip decision, dequantises, takes its DC back
// from lane 24's inverse WHT, runs the inverse DCT and adds onto the
// prediction. All arithmetic is the reference's integer listing: the
// forward transforms in int, the inverse DCT in wrapping 32-bit int.
#include <algorithm>
#include <mutex>

#include "coeff_tables.h"
#include "vp8a_internal.cuh"

namespace {

constexpr int RC_WARPS = 4;
constexpr int COS8 = 20091;  // sqrt(2) cos(pi/8) - 1, 16-bit fixed point
constexpr int SIN8 = 35468;  // sqrt(2) sin(pi/8), 16-bit fixed point

// §14.1 dc_qlookup / ac_qlookup (src/inverse_transform.rs:72-103).
const int16_t DC_Q[128] = {
    4,   5,   6,   7,   8,   9,   10,  10,  11,  12,  13,  14,  15,  16,  17,  17,  18,  19,  20,
    20,  21,  21,  22,  22,  23,  23,  24,  25,  25,  26,  27,  28,  29,  30,  31,  32,  33,  34,
    35,  36,  37,  37,  38,  39,  40,  41,  42,  43,  44,  45,  46,  46,  47,  48,  49,  50,  51,
    52,  53,  54,  55,  56,  57,  58,  59,  60,  61,  62,  63,  64,  65,  66,  67,  68,  69,  70,
    71,  72,  73,  74,  75,  76,  76,  77,  78,  79,  80,  81,  82,  83,  84,  85,  86,  87,  88,
    89,  91,  93,  95,  96,  98,  100, 101, 102, 104, 106, 108, 110, 112, 114, 116, 118, 122, 124,
    126, 128, 130, 132, 134, 136, 138, 140, 143, 145, 148, 151, 154, 157};
const int16_t AC_Q[128] = {
    4,   5,   6,   7,   8,   9,   10,  11,  12,  13,  14,  15,  16,  17,  18,  19,  20,  21,  22,
    23,  24,  25,  26,  27,  28,  29,  30,  31,  32,  33,  34,  35,  36,  37,  38,  39,  40,  41,
    42,  43,  44,  45,  46,  47,  48,  49,  50,  51,  52,  53,  54,  55,  56,  57,  58,  60,  62,
    64,  66,  68,  70,  72,  74,  76,  78,  80,  82,  84,  86,  88,  90,  92,  94,  96,  98,  100,
    102, 104, 106, 108, 110, 112, 114, 116, 119, 122, 125, 128, 131, 134, 137, 140, 143, 146, 149,
    152, 155, 158, 161, 164, 167, 170, 173, 177, 181, 185, 189, 193, 197, 201, 205, 209, 213, 217,
    221, 225, 229, 234, 239, 245, 249, 254, 259, 264, 269, 274, 279, 284};

int qclamp(int64_t q) { return q < 0 ? 0 : (q > 127 ? 127 : (int)q); }
int64_t sat32(int64_t v) { return std::max<int64_t>(INT32_MIN, std::min<int64_t>(INT32_MAX, v)); }

// MbDequantFactors::from_base_and_deltas (src/dequant.rs:118-165).
void factors_from(int64_t q, int ydc, int y2dc, int y2ac, int uvdc, int uvac, int16_t* out) {
  int y2_ac = AC_Q[qclamp(sat32(q + y2ac))] * 155 / 100;
  int uv_dc = DC_Q[qclamp(sat32(q + uvdc))];
  out[0] = DC_Q[qclamp(sat32(q + ydc))];
  out[1] = AC_Q[qclamp(q)];
  out[2] = (int16_t)(DC_Q[qclamp(sat32(q + y2dc))] * 2);
  out[3] = (int16_t)(y2_ac < 8 ? 8 : y2_ac);
  out[4] = (int16_t)(uv_dc > 132 ? 132 : uv_dc);
  out[5] = AC_Q[qclamp(sat32(q + uvac))];
}

struct RcArgs {
  const uint8_t *fy, *fu, *fv;  // visible source
  uint64_t fys, fuvs;
  int fw, fh, fcw, fch;
  uint8_t *ry, *ru, *rv;  // MB-padded planes: prediction in, reconstruction out
  uint64_t rys, ruvs;
  int aligned;  // recon plane bases and pitches are 4-byte aligned
  int mb_cols;
  uint32_t n;
  const vp8a_mb_decision* dec;
  uint8_t ref_ids[3];
  int n_refs;
  const int8_t* mb_segment;
  int16_t f[5][6];  // frame factors, then segments 0..3
  uint32_t m[5][6];  // ceil(2^32 / f): the quantiser's reciprocals
  int16_t* coeffs;
  uint8_t* flags;
  vp8a_mb_lf_info* lf;
  // §13 trellis: lambda per factor set (0 = plain rounding), the
  // bool_bits cost table and the IDCT basis norms by scan position.
  double tl[5];
  const double* bit_cost;
  double norm[16];
};

__device__ __forceinline__ int cmul(int i) { return i + ((i * COS8) >> 16); }
__device__ __forceinline__ int smul(int i) { return (i * SIN8) >> 16; }
__device__ __forceinline__ int rdiv2(int v) {
  const int r = v >= 0 ? (v + 1) >> 1 : -((-v + 1) >> 1);
  return r < -32768 ? -32768 : (r > 32767 ? 32767 : r);
}
__host__ __device__ __forceinline__ int to16(int v) { return (int)(short)v; }

// forward_dct_4x4_scalar (src/forward_transform.rs:486-604), in place.
__device__ __forceinline__ void fdct4x4(int* b) {
  int t[16];
#pragma unroll
  for (int col = 0; col < 4; col++) {
    const int i0 = b[col], i4 = b[4 + col], i8 = b[8 + col], i12 = b[12 + col];
    t[col] = (i0 + i12) + (i4 + i8);
    t[4 + col] = (cmul(i0) - cmul(i12)) + (smul(i4) - smul(i8));
    t[8 + col] = (i0 + i12) - (i4 + i8);
    t[12 + col] = (smul(i0) - smul(i12)) - (cmul(i4) - cmul(i8));
  }
#pragma unroll
  for (int row = 0; row < 4; row++) {
    const int r0 = t[4 * row], r1 = t[4 * row + 1], r2 = t[4 * row + 2], r3 = t[4 * row + 3];
    b[4 * row] = rdiv2((r0 + r3) + (r1 + r2));
    b[4 * row + 1] = rdiv2((cmul(r0) - cmul(r3)) + (smul(r1) - smul(r2)));
    b[4 * row + 2] = rdiv2((r0 + r3) - (r1 + r2));
    b[4 * row + 3] = rdiv2((smul(r0) - smul(r3)) - (cmul(r1) - cmul(r2)));
  }
}

// forward_wht_4x4_scalar (src/forward_transform.rs:173-260), in place.
__device__ __forceinline__ void fwht4x4(int* b) {
  int t[16];
#pragma unroll
  for (int col = 0; col < 4; col++) {
    const int a1 = b[col] + b[12 + col], b1 = b[4 + col] + b[8 + col];
    const int c1 = b[4 + col] - b[8 + col], d1 = b[col] - b[12 + col];
    t[col] = a1 + b1;
    t[4 + col] = c1 + d1;
    t[8 + col] = a1 - b1;
    t[12 + col] = d1 - c1;
  }
#pragma unroll
  for (int row = 0; row < 4; row++) {
    const int a1 = t[4 * row] + t[4 * row + 3], b1 = t[4 * row + 1] + t[4 * row + 2];
    const int c1 = t[4 * row + 1] - t[4 * row + 2], d1 = t[4 * row] - t[4 * row + 3];
    b[4 * row] = rdiv2(a1 + b1);
    b[4 * row + 1] = rdiv2(c1 + d1);
    b[4 * row + 2] = rdiv2(a1 - b1);
    b[4 * row + 3] = rdiv2(d1 - c1);
  }
}

// inverse_wht_4x4_scalar (src/inverse_transform.rs:190-252), in place.
__device__ __forceinline__ void iwht4x4(int* b) {
  int t[16];
#pragma unroll
  for (int col = 0; col < 4; col++) {
    const int a1 = b[col] + b[12 + col], b1 = b[4 + col] + b[8 + col];
    const int c1 = b[4 + col] - b[8 + col], d1 = b[col] - b[12 + col];
    t[col] = a1 + b1;
    t[4 + col] = c1 + d1;
    t[8 + col] = a1 - b1;
    t[12 + col] = d1 - c1;
  }
#pragma unroll
  for (int row = 0; row < 4; row++) {
    const int a1 = t[4 * row] + t[4 * row + 3], b1 = t[4 * row + 1] + t[4 * row + 2];
    const int c1 = t[4 * row + 1] - t[4 * row + 2], d1 = t[4 * row] - t[4 * row + 3];
    b[4 * row] = to16((a1 + b1 + 3) >> 3);
    b[4 * row + 1] = to16((c1 + d1 + 3) >> 3);
    b[4 * row + 2] = to16((a1 - b1 + 3) >> 3);
    b[4 * row + 3] = to16((d1 - c1 + 3) >> 3);
  }
}

// Two's-complement 32-bit arithmetic (the reference's wrapping_* ops).
__host__ __device__ __forceinline__ int wa(int a, int b) { return (int)((unsigned)a + (unsigned)b); }
__host__ __device__ __forceinline__ int ws(int a, int b) { return (int)((unsigned)a - (unsigned)b); }
__host__ __device__ __forceinline__ int wm(int a, int b) { return (int)((unsigned)a * (unsigned)b); }

// inverse_dct_4x4_scalar (src/inverse_transform.rs:609-712), in place.
__host__ __device__ __forceinline__ void idct4x4(int* b) {
  int t[16];
#pragma unroll
  for (int col = 0; col < 4; col++) {
    const int i0 = b[col], i4 = b[4 + col], i8 = b[8 + col], i12 = b[12 + col];
    const int a1 = wa(i0, i8), b1 = ws(i0, i8);
    const int c1 = ws(wm(i4, SIN8) >> 16, wa(i12, wm(i12, COS8) >> 16));
    const int d1 = wa(wa(i4, wm(i4, COS8) >> 16), wm(i12, SIN8) >> 16);
    t[col] = wa(a1, d1);
    t[12 + col] = ws(a1, d1);
    t[4 + col] = wa(b1, c1);
    t[8 + col] = ws(b1, c1);
  }
#pragma unroll
  for (int row = 0; row < 4; row++) {
    const int r0 = t[4 * row], r1 = t[4 * row + 1], r2 = t[4 * row + 2], r3 = t[4 * row + 3];
    const int a1 = wa(r0, r2), b1 = ws(r0, r2);
    const int c1 = ws(wm(r1, SIN8) >> 16, wa(r3, wm(r3, COS8) >> 16));
    const int d1 = wa(wa(r1, wm(r1, COS8) >> 16), wm(r3, SIN8) >> 16);
    b[4 * row] = to16(wa(wa(a1, d1), 4) >> 3);
    b[4 * row + 3] = to16(wa(ws(a1, d1), 4) >> 3);
    b[4 * row + 1] = to16(wa(wa(b1, c1), 4) >> 3);
    b[4 * row + 2] = to16(wa(ws(b1, c1), 4) >> 3);
  }
}

// enc_round_div (src/encoder.rs:2112): round half away from zero, as i16.
// The quotient floor(a / den) of a = |num| + den / 2 < 2^17 is taken as
// the high word of a * m with m = ceil(2^32 / den): with e = m * den - 2^32
// in [0, den), a * m / 2^32 = a / den + a * e / (den * 2^32), and the excess
// stays below 1 / den because a * den < 2^27 (den <= 440), so the floor is
// exact.
__device__ __forceinline__ int rdiv(int num, int den, uint32_t m) {
  const uint32_t q = __umulhi((uint32_t)abs(num) + (uint32_t)(den >> 1), m);
  return to16(num >= 0 ? (int)q : -(int)q);
}

// ---------------------------------------------- §13 trellis quantiser
//
// trellis_quantize_block with the direct scan (src/encoder.rs:3095-3129,
// :3468-3582), one block per lane: a Viterbi pass over the scan positions
// up to the last one whose rounded level is non-zero, the survivors keyed
// by the carried §13.3 context (0 / 1 / >= 2), candidates round, round - 1
// and 0, cost = distortion (IDCT basis norm x transform-domain error^2) +
// lambda x token bits (coeff_token_bits, :2789-2817, priced against the
// §13.5 default probabilities through bool_bits), and the end of the block
// chosen among the positions that hold a non-zero level. Every f64
// expression keeps the reference's operation order (the library is built
// without fused multiply-adds). Every inter call site uses entry
// context 0.
static __constant__ uint8_t c_tprobs[4][8][3][11] = VP8A_DEFAULT_COEFF_PROBS_INIT;
static __constant__ uint8_t c_tbands[16] = {0, 1, 2, 3, 6, 4, 5, 6, 6, 6, 6, 6, 6, 6, 6, 7};
static __constant__ uint8_t c_zigzag[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};
// Each token's (probability index, bit) path through the §13.2 coefficient
// tree from the root (DCT_0..DCT_4, cat1..cat6); the first step is the "not
// EOB" branch, skipped after a DCT_0.
static __constant__ uint8_t c_tpath_len[11] = {2, 3, 5, 6, 6, 6, 6, 7, 7, 7, 7};
static __constant__ uint8_t c_tpath[11][7][2] = {
    {{0, 1}, {1, 0}},
    {{0, 1}, {1, 1}, {2, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 0}, {4, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 0}, {4, 1}, {5, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 0}, {4, 1}, {5, 1}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 0}, {7, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 0}, {7, 1}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 1}, {8, 0}, {9, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 1}, {8, 0}, {9, 1}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 1}, {8, 1}, {10, 0}},
    {{0, 1}, {1, 1}, {2, 1}, {3, 1}, {6, 1}, {8, 1}, {10, 1}},
};
// DCT_extra categories: extra-bit probabilities, their count, base values.
static __constant__ uint8_t c_pcat[6][11] = {{159},
                                             {165, 145},
                                             {173, 148, 140},
                                             {176, 155, 140, 135},
                                             {180, 157, 141, 134, 130},
                                             {254, 254, 243, 230, 196, 177, 153, 140, 133, 130, 129}};
static __constant__ uint8_t c_pcat_len[6] = {1, 2, 3, 4, 5, 11};
static __constant__ uint16_t c_cat_base[6] = {5, 7, 11, 19, 35, 67};

// bool_bits (src/encoder.rs:2229).
__device__ __forceinline__ double tbb(const double* t, int prob, int v) {
  if (v) {
    const int idx = 256 - prob;
    return t[idx > 255 ? 255 : idx];
  }
  return t[prob];
}

// coeff_token_bits (src/encoder.rs:2789-2817).
__device__ double token_bits(const double* t, int plane, int i, int ctx3, bool pwz, uint32_t level) {
  const uint8_t* probs = c_tprobs[plane][c_tbands[i]][ctx3];
  const int token = level <= 4 ? (int)level
                               : (level <= 6 ? 5 : (level <= 10 ? 6 : (level <= 18 ? 7 : (level <= 34 ? 8 : (level <= 66 ? 9 : 10)))));
  double bits = 0.0;
  for (int s = pwz ? 1 : 0; s < c_tpath_len[token]; s++)
    bits += tbb(t, probs[c_tpath[token][s][0]], c_tpath[token][s][1]);
  if (token >= 5) {
    const int cat = token - 5, n = c_pcat_len[cat];
    const uint32_t extra = level - c_cat_base[cat];
    for (int j = 0; j < n; j++) bits += tbb(t, c_pcat[cat][j], (int)((extra >> (n - 1 - j)) & 1u));
  }
  if (level != 0) bits += tbb(t, 128, 0);
  return bits;
}

// eob_token_bits (src/encoder.rs:2825-2831).
__device__ __forceinline__ double eob_bits(const double* t, int plane, int i, int ctx3) {
  return tbb(t, c_tprobs[plane][c_tbands[i]][ctx3][0], 0);
}

// The trellis on one raster block `b` (the transform's output; replaced by
// the chosen levels).
__device__ void trellis_block(int* b, int dc, int ac, int first, int plane, double lambda, const RcArgs& a) {
  const double* t = a.bit_cost;
  const uint32_t dc_q = (uint32_t)dc, ac_q = (uint32_t)ac;
  uint32_t ax[16], mr[16];
  double zd[16], suffix[17];
  unsigned negative = 0;
  int last = -1;
  suffix[16] = 0.0;
#pragma unroll
  for (int k = 15; k >= 0; k--) {
    if (k < first) {
      suffix[k] = 0.0;
      ax[k] = mr[k] = 0;
      zd[k] = 0.0;
      continue;
    }
    const int x = b[c_zigzag[k]];
    const uint32_t q = k == 0 ? dc_q : ac_q;
    ax[k] = (uint32_t)(x < 0 ? -x : x);
    if (x < 0) negative |= 1u << k;
    mr[k] = (ax[k] + q / 2) / q;  // rounded_level (:3608-3615)
    if (mr[k] != 0 && last < 0) last = k;
    zd[k] = a.norm[k] * (double)((unsigned long long)ax[k] * ax[k]);
    suffix[k] = suffix[k + 1] + zd[k];
  }
#pragma unroll
  for (int k = 0; k < 16; k++) b[k] = 0;
  if (last < 0) return;
  const double INF = __longlong_as_double(0x7ff0000000000000LL);
  double sc[3] = {0.0, INF, INF};  // entry context 0
  bool sp[3] = {false, false, false};
  uint16_t cl[16][3];
  uint8_t cp[16][3];
  double best_term = 0.0 + lambda * eob_bits(t, plane, first, 0) + suffix[first];
  int best_pos = -1, best_ctx = 0;
  for (int k = first; k <= last; k++) {
    const uint32_t m = mr[k];
    const uint32_t q = k == 0 ? dc_q : ac_q;
    const uint32_t cands[3] = {m, m > 0 ? m - 1 : 0u, 0u};
    const int ncand = (int)(m < 2 ? m : 2) + 1;
    double cd[3];
    for (int c = 0; c < ncand; c++) {
      if (cands[c] == 0) {
        cd[c] = zd[k];
      } else {
        const long long err = (long long)ax[k] - (long long)cands[c] * (long long)q;
        cd[c] = a.norm[k] * (double)(err * err);
      }
    }
    double nc[3] = {INF, INF, INF};
    bool np[3] = {false, false, false};
    uint16_t nl[3] = {0, 0, 0};
    uint8_t npv[3] = {0, 0, 0};
    for (int in_ctx = 0; in_ctx < 3; in_ctx++) {
      const double base = sc[in_ctx];
      if (base >= INF) continue;
      for (int c = 0; c < ncand; c++) {
        const uint32_t level = cands[c];
        const double r = token_bits(t, plane, k, in_ctx, sp[in_ctx], level);
        const double cost = base + cd[c] + lambda * r;
        const int out = level == 0 ? 0 : (level == 1 ? 1 : 2);
        if (cost < nc[out]) {
          nc[out] = cost;
          np[out] = level == 0;
          nl[out] = (uint16_t)level;
          npv[out] = (uint8_t)in_ctx;
        }
      }
    }
    for (int c = 0; c < 3; c++) {
      cl[k][c] = nl[c];
      cp[k][c] = npv[c];
    }
    for (int out = 1; out < 3; out++) {
      const double cost = nc[out];
      if (cost >= INF) continue;
      const double term = k + 1 < 16 ? cost + lambda * eob_bits(t, plane, k + 1, out) + suffix[k + 1] : cost;
      if (term < best_term) {
        best_term = term;
        best_pos = k;
        best_ctx = out;
      }
    }
    for (int c = 0; c < 3; c++) {
      sc[c] = nc[c];
      sp[c] = np[c];
    }
  }
  if (best_pos >= 0) {
    int k = best_pos, ctx = best_ctx;
    for (;;) {
      const int level = cl[k][ctx];
      b[c_zigzag[k]] = (negative >> k & 1u) ? -level : level;
      if (k == first) break;
      ctx = cp[k][ctx];
      k--;
    }
  }
}

// CTA `cta` of the `ncta` working on `a`: one warp per MB, grid-stride.
__device__ __forceinline__ void recon_body(const RcArgs& a, uint32_t cta, uint32_t ncta) {
  const int lane = threadIdx.x & 31;
  const unsigned full = 0xffffffffu;
  for (uint32_t item = cta * RC_WARPS + (threadIdx.x >> 5); item < a.n; item += ncta * RC_WARPS) {
    const vp8a_mb_decision& d = a.dec[item];
    bool have = false;
    for (int k = 0; k < a.n_refs; k++) have |= d.ref_frame != VP8A_REF_INTRA && a.ref_ids[k] == d.ref_frame;
    if (!have) {  // warp-uniform: no inter reference, no reconstruction
      if (a.flags && lane == 0) a.flags[item] = 0;
      if (a.coeffs && lane < 25) {
        int16_t* dst = a.coeffs + (size_t)item * 400 + (lane == 24 ? 0 : 16 + 16 * lane);
#pragma unroll
        for (int k = 0; k < 16; k += 2) *reinterpret_cast<uint32_t*>(dst + k) = 0u;
      }
      continue;
    }
    const bool split = d.mode == VP8A_MODE_SPLIT;
    const int seg = a.mb_segment ? a.mb_segment[item] : -1;
    const int fs = (seg >= 0 && seg < 4) ? 1 + seg : 0;
    const int16_t* f = a.f[fs];
    const uint32_t* fm = a.m[fs];
    const int mbx = (int)(item % (uint32_t)a.mb_cols), mby = (int)(item / (uint32_t)a.mb_cols);

    // This lane's block: plane, top-left pixel in the plane.
    const bool luma = lane < 16, chroma = lane >= 16 && lane < 24;
    const int cb = (lane - 16) & 3;
    int px = 0, py = 0;
    uint8_t* rp = nullptr;
    uint64_t rs = 0;
    const uint8_t* sp = nullptr;
    uint64_t ss = 0;
    int sw = 1, sh = 1;
    if (luma) {
      px = mbx * 16 + 4 * (lane & 3);
      py = mby * 16 + 4 * (lane >> 2);
      rp = a.ry;
      rs = a.rys;
      sp = a.fy;
      ss = a.fys;
      sw = a.fw;
      sh = a.fh;
    } else if (chroma) {
      px = mbx * 8 + 4 * (cb & 1);
      py = mby * 8 + 4 * (cb >> 1);
      rp = lane < 20 ? a.ru : a.rv;
      rs = a.ruvs;
      sp = lane < 20 ? a.fu : a.fv;
      ss = a.fuvs;
      sw = a.fcw;
      sh = a.fch;
    }
    int blk[16];
    uint8_t pred[16];
    if (luma || chroma) {
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const uint8_t* prow = rp + (uint64_t)(py + r) * rs + px;
        if (a.aligned) {
          const uint32_t w = *reinterpret_cast<const uint32_t*>(prow);
#pragma unroll
          for (int c = 0; c < 4; c++) pred[4 * r + c] = (uint8_t)(w >> (8 * c));
        } else {
#pragma unroll
          for (int c = 0; c < 4; c++) pred[4 * r + c] = prow[c];
        }
        const int sy = min(py + r, sh - 1);
        const uint8_t* srow = sp + (uint64_t)sy * ss;
#pragma unroll
        for (int c = 0; c < 4; c++) blk[4 * r + c] = (int)__ldg(srow + min(px + c, sw - 1)) - (int)pred[4 * r + c];
      }
      fdct4x4(blk);
    } else {
#pragma unroll
      for (int k = 0; k < 16; k++) blk[k] = 0;
    }

    // Y2: lane 24 collects the sixteen luma DCs (non-SPLITMV).
    if (!split) {
#pragma unroll
      for (int k = 0; k < 16; k++) {
        const int v = __shfl_sync(full, blk[0], k);
        if (lane == 24) blk[k] = v;
      }
      if (lane == 24) fwht4x4(blk);
      if (luma) blk[0] = 0;
    }
    // Plain quantisation (enc_quantize_block) with this block's factors.
    const int fi = lane == 24 ? 2 : (chroma ? 4 : 0);
    const int qdc = f[fi], qac = f[fi + 1];
    const uint32_t mdc = fm[fi], mac = fm[fi + 1];
    const bool active = luma || chroma || (lane == 24 && !split);
    int nz = 0;
    if (active) {
      const double tl = a.tl[fs];
      if (tl > 0.0) {
        // BlockType planes: 0 YAfterY2 (from coefficient 1), 1 Y2, 2 UV,
        // 3 YNoY2 (SPLITMV luma).
        trellis_block(blk, qdc, qac, (luma && !split) ? 1 : 0, lane == 24 ? 1 : (chroma ? 2 : (split ? 3 : 0)), tl,
                      a);
      } else {
        blk[0] = rdiv(blk[0], qdc, mdc);
#pragma unroll
        for (int k = 1; k < 16; k++) blk[k] = rdiv(blk[k], qac, mac);
      }
#pragma unroll
      for (int k = 0; k < 16; k++) nz |= blk[k];
    }
    // §11.1 skip: no non-zero coefficient in Y2, the Y blocks (from index 1
    // with Y2; their DC is already 0) or the chroma blocks.
    const bool skip = !__any_sync(full, nz != 0);
    if (a.coeffs && (active || lane == 24)) {
      // MbCoeffs order: y2, y[16], u[4], v[4].
      const int off = lane == 24 ? 0 : (luma ? 16 + 16 * lane : 272 + 16 * (lane - 16));
      int16_t* dst = a.coeffs + (size_t)item * 400 + off;
#pragma unroll
      for (int k = 0; k < 16; k += 2)
        *reinterpret_cast<uint32_t*>(dst + k) = (uint32_t)(uint16_t)blk[k] | ((uint32_t)(uint16_t)blk[k + 1] << 16);
    }
    // Dequantise (dequant_block: (c * factor) as i16).
    int dnz = 0;
    if (active) {
      blk[0] = to16(blk[0] * qdc);
#pragma unroll
      for (int k = 1; k < 16; k++) blk[k] = to16(blk[k] * qac);
#pragma unroll
      for (int k = 0; k < 16; k++) dnz |= blk[k];
    }
    const bool has = __any_sync(full, dnz != 0);
    if (a.flags && lane == 0) a.flags[item] = (uint8_t)((skip ? VP8A_MB_SKIP : 0) | (has ? VP8A_MB_HAS_COEFFS : 0));
    if (a.lf && lane == 0) {
      vp8a_mb_lf_info m{};
      m.y_mode_is_bpred = split;
      m.has_coeffs = has;
      m.ref_frame = d.ref_frame;
      m.inter_mode = d.mode;
      m.segment_id = (int8_t)seg;
      a.lf[item] = m;
    }
    if (skip) continue;  // warp-uniform: the reconstruction is the prediction
    if (!split) {
      if (lane == 24) iwht4x4(blk);
#pragma unroll
      for (int k = 0; k < 16; k++) {
        const int v = __shfl_sync(full, blk[k], 24);
        if (lane == k) blk[0] = v;
      }
    }
    if (luma || chroma) {
      idct4x4(blk);
#pragma unroll
      for (int r = 0; r < 4; r++) {
        uint8_t* prow = rp + (uint64_t)(py + r) * rs + px;
        uint32_t w = 0;
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const int v = (int)pred[4 * r + c] + blk[4 * r + c];
          w |= (uint32_t)(v < 0 ? 0 : (v > 255 ? 255 : v)) << (8 * c);
        }
        if (a.aligned) {
          *reinterpret_cast<uint32_t*>(prow) = w;
        } else {
#pragma unroll
          for (int c = 0; c < 4; c++) prow[c] = (uint8_t)(w >> (8 * c));
        }
      }
    }
  }
}

__global__ void __launch_bounds__(RC_WARPS * 32) recon_kernel(RcArgs a) { recon_body(a, blockIdx.x, gridDim.x); }

__global__ void __launch_bounds__(RC_WARPS * 32)
    recon_frames_kernel(const RcArgs* __restrict__ jobs, const uint32_t* __restrict__ cta_start, int n_jobs) {
  __shared__ RcArgs sa;
  __shared__ uint32_t first[2];
  vp8a_dev::find_job(jobs, cta_start, n_jobs, &sa, first);
  recon_body(sa, blockIdx.x - first[0], first[1]);
}

int g_rc_blocks_per_sm = 0;

// IDCT_BASIS_NORM_SQ (src/encoder.rs:2763-2777): the energy of the §14.4
// inverse DCT of a 256 impulse at each scan position's raster index, over
// 256^2 (exact in f64).
const double* idct_basis_norms() {
  static double norms[16];
  static std::once_flag once;
  std::call_once(once, [] {
    static const int zz[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};
    for (int k = 0; k < 16; k++) {
      int b[16] = {0};
      b[zz[k]] = 256;
      idct4x4(b);
      double e = 0.0;
      for (int i = 0; i < 16; i++) e += (double)b[i] * (double)b[i];
      norms[k] = e / (256.0 * 256.0);
    }
  });
  return norms;
}

// Validate one frame's arguments, queue (or, with `defer`, prepare) its
// prediction into `recon`, and fill the reconstruction kernel's arguments
// and CTA count.
vp8a_status prepare_recon(vp8a_ctx* ctx, vp8a::Stager& st, const vp8a_i420* frame, const vp8a_planes* refs,
                          const uint8_t* ref_ids, uint32_t n_refs, const vp8a_mb_decision* decisions,
                          const vp8a_quant_indices* quant, const int8_t* mb_segment, const int16_t* segment_quant,
                          uint32_t segment_abs, uint32_t full_pixel, uint32_t filter_set, const vp8a_planes* recon,
                          int16_t* coeffs, uint8_t* mb_flags, vp8a_mb_lf_info* lf_info, bool defer,
                          vp8a::FramePrediction* fp, RcArgs* out, uint32_t* ctas);

}  // namespace

extern "C" {

void vp8a_dequant_factors(const vp8a_quant_indices* qi, uint32_t has_segment, int32_t segment_quant,
                          uint32_t absolute, int16_t* out) {
  if (!qi || !out) return;
  int64_t q = qi->y_ac_qi;
  if (has_segment) q = absolute ? (int64_t)segment_quant : sat32((int64_t)qi->y_ac_qi + segment_quant);
  factors_from(q, qi->y_dc_delta, qi->y2_dc_delta, qi->y2_ac_delta, qi->uv_dc_delta, qi->uv_ac_delta, out);
}

}  // extern "C"

namespace {
vp8a_status prepare_recon(vp8a_ctx* ctx, vp8a::Stager& st, const vp8a_i420* frame, const vp8a_planes* refs,
                          const uint8_t* ref_ids, uint32_t n_refs, const vp8a_mb_decision* decisions,
                          const vp8a_quant_indices* quant, const int8_t* mb_segment, const int16_t* segment_quant,
                          uint32_t segment_abs, uint32_t full_pixel, uint32_t filter_set, const vp8a_planes* recon,
                          int16_t* coeffs, uint8_t* mb_flags, vp8a_mb_lf_info* lf_info, bool defer,
                          vp8a::FramePrediction* fp_out, RcArgs* out, uint32_t* ctas) {
  if (!ctx || !frame || !quant || !recon) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (frame->width == 0 || frame->height == 0 || frame->width > 0x3FFF || frame->height > 0x3FFF) {
    vp8a::set_error("invalid dimensions");
    return VP8A_E_INVALID_DIMENSIONS;
  }
  if (quant->y_ac_qi > 127) {
    vp8a::set_error("y_ac_qi must be 0..=127");
    return VP8A_E_QUANT_INDEX_OUT_OF_RANGE;
  }
  if (!frame->y || !frame->u || !frame->v || frame->y_stride < frame->width ||
      frame->uv_stride < (frame->width + 1) / 2) {
    vp8a::set_error("bad source plane");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (recon->mb_cols != (frame->width + 15) / 16 || recon->mb_rows != (frame->height + 15) / 16) {
    vp8a::set_error("reconstruction planes do not match the frame's MB grid");
    return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
  }
  vp8a::FramePrediction& fp = *fp_out;
  vp8a_status s = vp8a::predict_frame(ctx, st, refs, ref_ids, n_refs, decisions, full_pixel, filter_set, recon, &fp,
                                      defer);
  if (s != VP8A_OK) return s;

  RcArgs a{};
  const size_t cw = (frame->width + 1) / 2, ch = (frame->height + 1) / 2;
  const void* d;
  if ((s = st.in(frame->y, frame->y_stride * (size_t)(frame->height - 1) + frame->width, &d)) != VP8A_OK) return s;
  a.fy = (const uint8_t*)d;
  if ((s = st.in(frame->u, frame->uv_stride * (ch - 1) + cw, &d)) != VP8A_OK) return s;
  a.fu = (const uint8_t*)d;
  if ((s = st.in(frame->v, frame->uv_stride * (ch - 1) + cw, &d)) != VP8A_OK) return s;
  a.fv = (const uint8_t*)d;
  a.fys = frame->y_stride;
  a.fuvs = frame->uv_stride;
  a.fw = (int)frame->width;
  a.fh = (int)frame->height;
  a.fcw = (int)cw;
  a.fch = (int)ch;
  a.ry = fp.planes.y;
  a.ru = fp.planes.u;
  a.rv = fp.planes.v;
  a.rys = fp.planes.y_stride;
  a.ruvs = fp.planes.uv_stride;
  a.aligned = (((uintptr_t)a.ry | (uintptr_t)a.ru | (uintptr_t)a.rv | a.rys | a.ruvs) & 3) == 0;
  a.mb_cols = (int)recon->mb_cols;
  a.n = recon->mb_cols * recon->mb_rows;
  a.dec = fp.dec;
  for (uint32_t k = 0; k < fp.n_refs; k++) a.ref_ids[k] = fp.ref_ids[k];
  a.n_refs = (int)fp.n_refs;
  int16_t sq[4] = {0, 0, 0, 0};
  if (segment_quant && (s = st.read_to_host(segment_quant, sizeof sq, sq)) != VP8A_OK) return s;
  vp8a_dequant_factors(quant, 0, 0, 0, a.f[0]);
  for (int k = 0; k < 4; k++) vp8a_dequant_factors(quant, 1, sq[k], segment_abs, a.f[1 + k]);
  for (int k = 0; k < 5; k++)
    for (int i = 0; i < 6; i++) a.m[k][i] = (uint32_t)((((uint64_t)1 << 32) + a.f[k][i] - 1) / a.f[k][i]);
  // The trellis price per factor set: MbRdCtx::trellis_lambda, rd_lambda
  // (y1_ac^2 / 32, src/encoder.rs:3742) x strength x TRELLIS_LAMBDA_SCALE.
  for (int k = 0; k < 5; k++) {
    const double q = (double)a.f[k][1];
    const double lambda = q * q / 32.0;
    a.tl[k] = ctx->trellis_strength > 0.0 ? lambda * (ctx->trellis_strength * 0.04) : 0.0;
  }
  a.bit_cost = ctx->d_bit_cost;
  memcpy(a.norm, idct_basis_norms(), sizeof a.norm);
  if (mb_segment) {
    if ((s = st.in(mb_segment, a.n, &d)) != VP8A_OK) return s;
    a.mb_segment = (const int8_t*)d;
  }
  void* o;
  if (coeffs) {
    if ((s = st.out(coeffs, (size_t)a.n * 400 * sizeof(int16_t), &o)) != VP8A_OK) return s;
    if (((uintptr_t)o & 3) != 0) {
      vp8a::set_error("coeffs must be 4-byte aligned");
      return VP8A_E_INVALID_ARGUMENT;
    }
    a.coeffs = (int16_t*)o;
  }
  if (mb_flags) {
    if ((s = st.out(mb_flags, a.n, &o)) != VP8A_OK) return s;
    a.flags = (uint8_t*)o;
  }
  if (lf_info) {
    // In/out: MBs without an inter reference keep the caller's record.
    if ((s = st.inout(lf_info, (size_t)a.n * sizeof(vp8a_mb_lf_info), &o)) != VP8A_OK) return s;
    a.lf = (vp8a_mb_lf_info*)o;
  }
  if (!g_rc_blocks_per_sm) {
    int b = 0;
    VP8A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, recon_kernel, RC_WARPS * 32, 0));
    g_rc_blocks_per_sm = std::max(b, 1);
  }
  *ctas = (unsigned)std::min<size_t>((a.n + RC_WARPS - 1) / RC_WARPS, (size_t)ctx->sm_count * g_rc_blocks_per_sm);
  *out = a;
  return VP8A_OK;
}
}  // namespace

extern "C" {

vp8a_status vp8a_reconstruct_inter_frame(vp8a_ctx* ctx, const vp8a_i420* frame, const vp8a_planes* refs,
                                         const uint8_t* ref_ids, uint32_t n_refs, const vp8a_mb_decision* decisions,
                                         const vp8a_quant_indices* quant, const int8_t* mb_segment,
                                         const int16_t* segment_quant, uint32_t segment_abs, uint32_t full_pixel,
                                         uint32_t filter_set, vp8a_planes* recon, int16_t* coeffs,
                                         uint8_t* mb_flags, vp8a_mb_lf_info* lf_info) {
  if (!ctx) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  vp8a::FramePrediction fp;
  RcArgs a;
  uint32_t grid = 0;
  vp8a_status s = prepare_recon(ctx, st, frame, refs, ref_ids, n_refs, decisions, quant, mb_segment, segment_quant,
                                segment_abs, full_pixel, filter_set, recon, coeffs, mb_flags, lf_info, false, &fp, &a,
                                &grid);
  if (s != VP8A_OK) return s;
  recon_kernel<<<grid, RC_WARPS * 32, 0, ctx->stream>>>(a);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return st.finish();
}

vp8a_status vp8a_reconstruct_inter_frames(vp8a_ctx* ctx, const vp8a_recon_job* jobs, uint32_t n_jobs) {
  if (!ctx || (!jobs && n_jobs)) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (n_jobs > VP8A_MAX_BATCH_JOBS) {
    vp8a::set_error("more jobs than VP8A_MAX_BATCH_JOBS");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (n_jobs == 0) return VP8A_OK;
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  std::vector<vp8a::FramePrediction> fps(n_jobs);
  std::vector<RcArgs> table(n_jobs);
  std::vector<uint32_t> start{0};
  vp8a_status s;
  for (uint32_t j = 0; j < n_jobs; j++) {
    const vp8a_recon_job& J = jobs[j];
    uint32_t ctas = 0;
    if ((s = prepare_recon(ctx, st, &J.frame, J.refs, J.ref_ids, J.n_refs, J.decisions, &J.quant, J.mb_segment,
                           J.segment_quant, J.segment_abs, J.full_pixel, J.filter_set, &J.recon, J.coeffs, J.mb_flags,
                           J.lf_info, true, &fps[j], &table[j], &ctas)) != VP8A_OK)
      return s;
    start.push_back(start.back() + ctas);
  }
  if ((s = vp8a::predict_frames(ctx, st, fps.data(), n_jobs)) != VP8A_OK) return s;
  const size_t o_start = sizeof(RcArgs) * n_jobs, total = o_start + sizeof(uint32_t) * start.size();
  std::vector<uint8_t> blob(total);
  memcpy(blob.data(), table.data(), o_start);
  memcpy(blob.data() + o_start, start.data(), sizeof(uint32_t) * start.size());
  void* d;
  if ((s = st.upload(blob.data(), total, &d)) != VP8A_OK) return s;
  recon_frames_kernel<<<start.back(), RC_WARPS * 32, 0, ctx->stream>>>(
      (const RcArgs*)d, (const uint32_t*)((const uint8_t*)d + o_start), (int)n_jobs);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return st.finish();
}

}  // extern "C"
