// census.cuh — §16.3 census and RD bit costs on the device, shared by the
// exhaustive analysis (analysis.cu) and the RD-effort search (rd_search.cu).
#pragma once

#include "me_common.cuh"

namespace vp8a_dev {

// The census record of one MB (MbInfo, src/near_mv.rs:127); layout equals
// vp8a_mb_info.
struct MbInfoDev {
  uint8_t ref_frame;  // VP8A_REF_INTRA = None
  uint8_t is_split;
  uint8_t has_split_mvs;
  uint8_t reserved;
  vp8a_mv mv;
  vp8a_mv split_mvs[16];
};

static_assert(sizeof(MbInfoDev) == sizeof(vp8a_mb_info), "MbInfoDev layout");

static __constant__ uint8_t c_counts_to_probs[6][4] = {{7, 1, 1, 143},    {14, 18, 14, 107}, {135, 64, 57, 68},
                                                {60, 56, 128, 65}, {159, 134, 128, 34}, {234, 188, 128, 28}};
static __constant__ uint8_t c_partitions[4][16] = {{0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1},
                                            {0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1},
                                            {0, 0, 1, 1, 0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 3, 3},
                                            {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}};
static __constant__ uint8_t c_partition_probs[3] = {110, 111, 150};
static __constant__ uint8_t c_submv_probs[5][3] = {{147, 136, 18}, {106, 145, 1}, {179, 121, 1}, {223, 1, 34}, {208, 1, 1}};
static __constant__ int8_t c_small_mvtree[14] = {2, 8, 4, 6, -0, -1, -2, -3, 10, 12, -4, -5, -6, -7};

static __device__ __forceinline__ bool mv_eq(vp8a_mv a, vp8a_mv b) { return a.row == b.row && a.col == b.col; }
static __device__ __forceinline__ bool mv_zero(vp8a_mv a) { return a.row == 0 && a.col == 0; }

// bool_bits (src/encoder.rs:2229).
static __device__ __forceinline__ double bb(const double* t, int prob, int v) {
  if (v) {
    int idx = 256 - prob;
    return t[idx > 255 ? 255 : idx];
  }
  return t[prob];
}

// mv_component_bits (src/motion_vector.rs:345), same summation order.
static __device__ double mv_component_bits(const double* t, const uint8_t* p, int value) {
  const int a = value < 0 ? -value : value;
  double bits = 0.0;
  if (a > 7) {
    bits += bb(t, p[0], 1);
    for (int i = 0; i < 3; i++) bits += bb(t, p[9 + i], (a >> i) & 1);
    int i = 9;
    for (;;) {
      bits += bb(t, p[9 + i], (a >> i) & 1);
      i -= 1;
      if (i <= 3) break;
    }
    if ((a & 0xfff0) != 0) bits += bb(t, p[9 + 3], (a >> 3) & 1);
  } else {
    bits += bb(t, p[0], 0);
    double s = 0.0;
    int i = 0;
    for (int k = 2; k >= 0; k--) {
      int bit = (a >> k) & 1;
      s += bb(t, p[2 + (i >> 1)], bit);
      int next = c_small_mvtree[i + bit];
      if (next <= 0) break;
      i = next;
    }
    bits += s;
  }
  if (a != 0) bits += bb(t, p[1], value < 0);
  return bits;
}

// mv_component_bits of both components for every value -1023..1023,
// written to out[k * 2047 + value + 1023]: the searches read the table
// instead of walking the tree per candidate. The entries come from the
// same device function, so they are bit-identical.
constexpr int MV_BITS_SPAN = 2047;
static __global__ void mv_bits_table_kernel(const double* t, vp8a_mv_contexts ctx, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * MV_BITS_SPAN) return;
  const int k = i >= MV_BITS_SPAN, v = i - k * MV_BITS_SPAN - 1023;
  out[i] = mv_component_bits(t, ctx.p[k], v);
}

// Table lookup; value must lie in -1023..1023.
static __device__ __forceinline__ double mv_bits_lookup(const double* tab, int k, int v) {
  return __ldg(tab + k * MV_BITS_SPAN + v + 1023);
}

struct Census {
  vp8a_mv best_predictor, nearest, near_;
  uint8_t p[4];
};

// find_near_mvs (src/near_mv.rs:310-402; default SignBias) + clamps
// (MvClampRect::for_mb / clamp_mv, :236-283) + mv_ref_probs (:404).
// The reference's near-MV list index and count index always advance
// together, so one index `mi` drives both; the list and the counts live in
// registers (every index is resolved with selects).
static __device__ __forceinline__ Census census(const MbInfoDev& above, const MbInfoDev& left, const MbInfoDev& al,
                                                int mb_col, int mb_row, int mb_cols, int mb_rows) {
  vp8a_mv n0 = {0, 0}, n1 = {0, 0}, n2 = {0, 0}, n3 = {0, 0};
  int c0 = 0, c1 = 0, c2 = 0, c3 = 0, mi = 0;
  auto last = [&]() { return mi == 0 ? n0 : (mi == 1 ? n1 : (mi == 2 ? n2 : n3)); };
  auto push = [&](vp8a_mv v) {
    mi++;
    if (mi == 1) n1 = v;
    else if (mi == 2) n2 = v;
    else n3 = v;
  };
  auto count = [&](int w) {
    if (mi == 0) c0 += w;
    else if (mi == 1) c1 += w;
    else if (mi == 2) c2 += w;
    else c3 += w;
  };
  if (above.ref_frame != VP8A_REF_INTRA) {
    if (!mv_zero(above.mv)) push(above.mv);
    count(2);
  }
  if (left.ref_frame != VP8A_REF_INTRA) {
    if (!mv_zero(left.mv)) {
      if (!mv_eq(left.mv, last())) push(left.mv);
      count(2);
    } else {
      c0 += 2;
    }
  }
  if (al.ref_frame != VP8A_REF_INTRA) {
    if (!mv_zero(al.mv)) {
      if (!mv_eq(al.mv, last())) push(al.mv);
      count(1);
    } else {
      c0 += 1;
    }
  }
  if (c3 != 0 && mv_eq(last(), n1)) c1 += 1;
  c3 = (above.is_split + left.is_split) * 2 + al.is_split;
  if (c2 > c1) {
    const int t = c1;
    c1 = c2;
    c2 = t;
    const vp8a_mv tm = n1;
    n1 = n2;
    n2 = tm;
  }
  if (c1 >= c0) n0 = n1;
  const int to_left = -((mb_col + 1) << 6), to_right = (mb_cols - mb_col) << 6;
  const int to_top = -((mb_row + 1) << 6), to_bottom = (mb_rows - mb_row) << 6;
  Census c;
  c.best_predictor.col = (int16_t)clampi(n0.col, to_left, to_right);
  c.best_predictor.row = (int16_t)clampi(n0.row, to_top, to_bottom);
  c.nearest.col = (int16_t)clampi(n1.col, to_left, to_right);
  c.nearest.row = (int16_t)clampi(n1.row, to_top, to_bottom);
  c.near_.col = (int16_t)clampi(n2.col, to_left, to_right);
  c.near_.row = (int16_t)clampi(n2.row, to_top, to_bottom);
  c.p[0] = c_counts_to_probs[c0][0];
  c.p[1] = c_counts_to_probs[c1][1];
  c.p[2] = c_counts_to_probs[c2][2];
  c.p[3] = c_counts_to_probs[c3][3];
  return c;
}


}  // namespace vp8a_dev
