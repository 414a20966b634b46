// me.cu — batched §17/§18 motion-search entry points:
//   vp8a_mb_luma_sad_at_mv          (mb_luma_sad_at_mv, src/motion_search.rs:470)
//   vp8a_small_diamond_search_luma  (src/motion_search.rs:381)
//   vp8a_half_pixel_refine_luma     (src/motion_search.rs:564)
//   vp8a_quarter_pixel_refine_luma  (src/motion_search.rs:666)
//   vp8a_motion_descent             (diamond -> half -> quarter, src/encoder.rs:8576-8596)
//   vp8a_motion_descent_masked      (the same for the items an active mask selects)
// One warp per item, four warps per CTA; the reference window of each item
// is staged in shared memory (me_common.cuh).
#include "me_common.cuh"

namespace {
using namespace vp8a_dev;

enum MeMode { MODE_SAD = 0, MODE_DIAMOND = 1, MODE_HALF = 2, MODE_QUARTER = 3, MODE_DESCENT = 4 };

struct MeBatch {
  MePlane P;
  const uint8_t* src_mbs;
  const uint32_t* mb_xy;
  const vp8a_mv* mvs;
  uint32_t n;
  uint32_t max_iters;
  uint32_t* sad_out;
  vp8a_search_result* out0;
  vp8a_search_result* out1;
  vp8a_search_result* out2;
  const uint8_t* active;  // optional: items whose byte is 0 are skipped
};

constexpr int ME_WARPS = 4;

template <int MODE>
__global__ void __launch_bounds__(ME_WARPS * 32) me_batch_kernel(MeBatch a) {
  __shared__ WarpScratch scratch[ME_WARPS];
  __shared__ __align__(16) uint8_t srcs[ME_WARPS][256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t item = blockIdx.x * ME_WARPS + warp;
  if (item >= a.n) return;  // warp-uniform
  if (a.active && !a.active[item]) return;
  WarpScratch& S = scratch[warp];
  uint8_t* src = srcs[warp];
  const uint8_t* gsrc = a.src_mbs + (size_t)item * 256;
#pragma unroll
  for (int k = 0; k < 8; k++) src[lane + 32 * k] = gsrc[lane + 32 * k];
  const int mbx = (int)a.mb_xy[2 * item] * 16, mby = (int)a.mb_xy[2 * item + 1] * 16;
  const vp8a_mv c = a.mvs[item];
  __syncwarp();

  if (MODE == MODE_SAD) {
    // No window: every fetch is a clamped global fetch.
    uint32_t s = sad_at_mv(a.P, S, -(1 << 28), -(1 << 28), mbx, mby, c.row, c.col, src, lane);
    if (lane == 0) a.sad_out[item] = s;
    return;
  }
  // Window around the integer part of the centre.
  int cx, cy;
  if (MODE == MODE_DIAMOND || MODE == MODE_DESCENT) {
    cx = snap_whole(clamp_component(c.col)) / 4;
    cy = snap_whole(clamp_component(c.row)) / 4;
  } else {
    cx = eighth(c.col) >> 3;
    cy = eighth(c.row) >> 3;
  }
  const int wx0 = mbx + cx - WIN_LEAD, wy0 = mby + cy - WIN_LEAD;
  load_window(a.P, S.win, wx0, wy0, lane);

  if (MODE == MODE_DIAMOND) {
    vp8a_search_result r = diamond(a.P, S, wx0, wy0, mbx, mby, c, a.max_iters, src, lane);
    if (lane == 0) a.out0[item] = r;
  } else if (MODE == MODE_HALF) {
    vp8a_search_result r;
    if (!half_refine_planes(S, wx0, wy0, mbx, mby, c, src, lane, &r))
      r = refine(a.P, S, wx0, wy0, mbx, mby, c, 2, src, lane);
    if (lane == 0) a.out0[item] = r;
  } else if (MODE == MODE_QUARTER) {
    vp8a_search_result r = refine(a.P, S, wx0, wy0, mbx, mby, c, 1, src, lane);
    if (lane == 0) a.out0[item] = r;
  } else {
    vp8a_search_result w = diamond(a.P, S, wx0, wy0, mbx, mby, c, a.max_iters, src, lane);
    vp8a_search_result h;
    if (!half_refine_planes(S, wx0, wy0, mbx, mby, w.mv, src, lane, &h))
      h = refine(a.P, S, wx0, wy0, mbx, mby, w.mv, 2, src, lane);
    vp8a_search_result q = refine(a.P, S, wx0, wy0, mbx, mby, h.mv, 1, src, lane, h.sad);
    if (lane == 0) {
      if (a.out0) a.out0[item] = w;
      if (a.out1) a.out1[item] = h;
      if (a.out2) a.out2[item] = q;
    }
  }
}

using vp8a::Stager;

vp8a_status run_batch(vp8a_ctx* ctx, int mode, const vp8a_luma_ref* ref, const uint8_t* src_mbs,
                      const uint32_t* mb_xy, const vp8a_mv* mvs, uint32_t max_iters, uint32_t n,
                      uint32_t* sad_out, vp8a_search_result* o0, vp8a_search_result* o1,
                      vp8a_search_result* o2, const uint8_t* active = nullptr) {
  if (!ctx || !ref || !ref->plane) {
    vp8a::set_error("null context or reference");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (ref->width == 0 || ref->height == 0 || ref->stride < ref->width) {
    vp8a::set_error("reference plane must be non-empty with stride >= width");
    return VP8A_E_INVALID_DIMENSIONS;
  }
  if (n == 0) return VP8A_OK;
  if (!src_mbs || !mb_xy || !mvs) {
    vp8a::set_error("null batch input");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  Stager st(ctx);
  MeBatch a{};
  const void* d = nullptr;
  vp8a_status s;
  size_t plane_bytes = ref->stride * (size_t)(ref->height - 1) + ref->width;
  if ((s = st.in(ref->plane, plane_bytes, &d)) != VP8A_OK) return s;
  a.P.plane = (const uint8_t*)d;
  a.P.stride = ref->stride;
  a.P.width = (int)ref->width;
  a.P.height = (int)ref->height;
  if ((s = st.in(src_mbs, (size_t)n * 256, &d)) != VP8A_OK) return s;
  a.src_mbs = (const uint8_t*)d;
  if ((s = st.in(mb_xy, (size_t)n * 8, &d)) != VP8A_OK) return s;
  a.mb_xy = (const uint32_t*)d;
  if ((s = st.in(mvs, (size_t)n * sizeof(vp8a_mv), &d)) != VP8A_OK) return s;
  a.mvs = (const vp8a_mv*)d;
  if (active) {
    if ((s = st.in(active, (size_t)n, &d)) != VP8A_OK) return s;
    a.active = (const uint8_t*)d;
  }
  void* o = nullptr;
  if (sad_out) {
    if ((s = st.out(sad_out, (size_t)n * 4, &o)) != VP8A_OK) return s;
    a.sad_out = (uint32_t*)o;
  }
  vp8a_search_result* outs[3] = {o0, o1, o2};
  vp8a_search_result** douts[3] = {&a.out0, &a.out1, &a.out2};
  for (int k = 0; k < 3; k++)
    if (outs[k]) {
      // With a mask, skipped items keep their values: host outputs go both ways.
      if ((s = active ? st.inout(outs[k], (size_t)n * sizeof(vp8a_search_result), &o)
                      : st.out(outs[k], (size_t)n * sizeof(vp8a_search_result), &o)) != VP8A_OK)
        return s;
      *douts[k] = (vp8a_search_result*)o;
    }
  a.n = n;
  a.max_iters = max_iters;
  dim3 grid(vp8a::grid_for(n, ME_WARPS)), block(ME_WARPS * 32);
  switch (mode) {
    case MODE_SAD: me_batch_kernel<MODE_SAD><<<grid, block, 0, ctx->stream>>>(a); break;
    case MODE_DIAMOND: me_batch_kernel<MODE_DIAMOND><<<grid, block, 0, ctx->stream>>>(a); break;
    case MODE_HALF: me_batch_kernel<MODE_HALF><<<grid, block, 0, ctx->stream>>>(a); break;
    case MODE_QUARTER: me_batch_kernel<MODE_QUARTER><<<grid, block, 0, ctx->stream>>>(a); break;
    default: me_batch_kernel<MODE_DESCENT><<<grid, block, 0, ctx->stream>>>(a); break;
  }
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return st.finish();
}

}  // namespace

extern "C" {

vp8a_status vp8a_mb_luma_sad_at_mv(vp8a_ctx* ctx, const vp8a_luma_ref* ref, const uint8_t* src_mbs,
                                   const uint32_t* mb_xy, const vp8a_mv* mvs, uint32_t n,
                                   uint32_t* sad_out) {
  if (n && !sad_out) return VP8A_E_INVALID_ARGUMENT;
  return run_batch(ctx, MODE_SAD, ref, src_mbs, mb_xy, mvs, 0, n, sad_out, nullptr, nullptr, nullptr);
}

vp8a_status vp8a_small_diamond_search_luma(vp8a_ctx* ctx, const vp8a_luma_ref* ref,
                                           const uint8_t* src_mbs, const uint32_t* mb_xy,
                                           const vp8a_mv* centers, uint32_t max_iters, uint32_t n,
                                           vp8a_search_result* out) {
  if (n && !out) return VP8A_E_INVALID_ARGUMENT;
  return run_batch(ctx, MODE_DIAMOND, ref, src_mbs, mb_xy, centers, max_iters, n, nullptr, out, nullptr,
                   nullptr);
}

vp8a_status vp8a_half_pixel_refine_luma(vp8a_ctx* ctx, const vp8a_luma_ref* ref, const uint8_t* src_mbs,
                                        const uint32_t* mb_xy, const vp8a_mv* whole_centers, uint32_t n,
                                        vp8a_search_result* out) {
  if (n && !out) return VP8A_E_INVALID_ARGUMENT;
  return run_batch(ctx, MODE_HALF, ref, src_mbs, mb_xy, whole_centers, 0, n, nullptr, out, nullptr, nullptr);
}

vp8a_status vp8a_quarter_pixel_refine_luma(vp8a_ctx* ctx, const vp8a_luma_ref* ref,
                                           const uint8_t* src_mbs, const uint32_t* mb_xy,
                                           const vp8a_mv* half_centers, uint32_t n, vp8a_search_result* out) {
  if (n && !out) return VP8A_E_INVALID_ARGUMENT;
  return run_batch(ctx, MODE_QUARTER, ref, src_mbs, mb_xy, half_centers, 0, n, nullptr, out, nullptr,
                   nullptr);
}

vp8a_status vp8a_motion_descent(vp8a_ctx* ctx, const vp8a_luma_ref* ref, const uint8_t* src_mbs,
                                const uint32_t* mb_xy, const vp8a_mv* centers, uint32_t max_iters,
                                uint32_t n, vp8a_search_result* whole_out, vp8a_search_result* half_out,
                                vp8a_search_result* quarter_out) {
  return run_batch(ctx, MODE_DESCENT, ref, src_mbs, mb_xy, centers, max_iters, n, nullptr, whole_out,
                   half_out, quarter_out);
}

vp8a_status vp8a_motion_descent_masked(vp8a_ctx* ctx, const vp8a_luma_ref* ref, const uint8_t* src_mbs,
                                       const uint32_t* mb_xy, const vp8a_mv* centers, uint32_t max_iters,
                                       uint32_t n, const uint8_t* active, vp8a_search_result* whole_out,
                                       vp8a_search_result* half_out, vp8a_search_result* quarter_out) {
  if (n && !active) {
    vp8a::set_error("null active mask");
    return VP8A_E_INVALID_ARGUMENT;
  }
  return run_batch(ctx, MODE_DESCENT, ref, src_mbs, mb_xy, centers, max_iters, n, nullptr, whole_out,
                   half_out, quarter_out, active);
}

}  // extern "C"
