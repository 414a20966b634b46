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
static __device__ Census census(const MbInfoDev& above, const MbInfoDev& left, const MbInfoDev& al, int mb_col, int mb_row,
                         int mb_cols, int mb_rows) {
  vp8a_mv nm[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  int cnt[4] = {0, 0, 0, 0};
  int mi = 0, ci = 0;
  if (above.ref_frame != VP8A_REF_INTRA) {
    if (!mv_zero(above.mv)) {
      mi++;
      nm[mi] = above.mv;
      ci++;
    }
    cnt[ci] += 2;
  }
  if (left.ref_frame != VP8A_REF_INTRA) {
    if (!mv_zero(left.mv)) {
      if (!mv_eq(left.mv, nm[mi])) {
        mi++;
        nm[mi] = left.mv;
        ci++;
      }
      cnt[ci] += 2;
    } else {
      cnt[0] += 2;
    }
  }
  if (al.ref_frame != VP8A_REF_INTRA) {
    if (!mv_zero(al.mv)) {
      if (!mv_eq(al.mv, nm[mi])) {
        mi++;
        nm[mi] = al.mv;
        ci++;
      }
      cnt[ci] += 1;
    } else {
      cnt[0] += 1;
    }
  }
  if (cnt[3] != 0 && mv_eq(nm[mi], nm[1])) cnt[1] += 1;
  cnt[3] = (above.is_split + left.is_split) * 2 + al.is_split;
  if (cnt[2] > cnt[1]) {
    int t = cnt[1];
    cnt[1] = cnt[2];
    cnt[2] = t;
    vp8a_mv tm = nm[1];
    nm[1] = nm[2];
    nm[2] = tm;
  }
  if (cnt[1] >= cnt[0]) nm[0] = nm[1];
  const int to_left = -((mb_col + 1) << 6), to_right = (mb_cols - mb_col) << 6;
  const int to_top = -((mb_row + 1) << 6), to_bottom = (mb_rows - mb_row) << 6;
  Census c;
  vp8a_mv* outs[3] = {&c.best_predictor, &c.nearest, &c.near_};
  for (int k = 0; k < 3; k++) {
    outs[k]->col = (int16_t)clampi(nm[k].col, to_left, to_right);
    outs[k]->row = (int16_t)clampi(nm[k].row, to_top, to_bottom);
  }
  for (int k = 0; k < 4; k++) c.p[k] = c_counts_to_probs[cnt[k]][k];
  return c;
}


}  // namespace vp8a_dev
