// arnr.cu — the ARNR temporal filter (build_arnr_altref, src/arnr.rs:476).
//
// Two kernels:
//  * arnr_search_kernel — refine_search (src/arnr.rs:264-300) for every
//    (window frame != centre, 16x16 block): one warp per block, the +/-15 px
//    neighbourhood of the block staged edge-clamped in shared memory, the
//    eight candidates of each 8/4/2/1 round scored in parallel (four lanes
//    each) and folded in the reference's candidate order with strict '<'.
//  * arnr_blend_kernel — the per-pixel weighted temporal mean
//    (accumulate_* :337-459 + resolve_plane :670): every output pixel
//    gathers its block's alignment from each frame, applies the SAD
//    occlusion guard (:605) and the weight table (:307-323), and resolves in
//    one pass. Integer sums are order-free, so gathering per pixel equals
//    the reference's frame-then-raster scatter. Every chroma pixel lies in
//    exactly one chroma block (block k covers [8k, 8k + ceil(bw/2)) and
//    ceil((bx+bw)/2) <= ceil(w/2)), so the clamped-overhang branch of
//    accumulate_chroma_block never adds a second contribution.
#include "vp8a_internal.cuh"

namespace {
using namespace vp8a_dev;
constexpr unsigned FULL = 0xffffffffu;

struct ArnrFrame {
  const uint8_t* y;
  const uint8_t* u;
  const uint8_t* v;
  uint64_t y_stride;
  uint64_t uv_stride;
};

struct BlockMv {
  int16_t mvx;
  int16_t mvy;
  uint32_t sad;
};

constexpr int AW = 46;       // window extent: 16 + 2 * 15
constexpr int AWS = 48;      // window stride
constexpr int ARNR_WARPS = 4;

__device__ __forceinline__ void load8u(const uint8_t* p, uint32_t& o0, uint32_t& o1) {
  uintptr_t a = (uintptr_t)p;
  const uint32_t* w = (const uint32_t*)(a & ~(uintptr_t)3);
  unsigned sh = (unsigned)(a & 3) * 8u;
  uint32_t w0 = w[0], w1 = w[1], w2 = w[2];
  o0 = __funnelshift_r(w0, w1, sh);
  o1 = __funnelshift_r(w1, w2, sh);
}

struct SearchArgs {
  const ArnrFrame* frames;
  uint32_t n, center;
  int w, h, bcols, brows;
  BlockMv* out;  // [n][brows][bcols]
};

__global__ void __launch_bounds__(ARNR_WARPS * 32) arnr_search_kernel(SearchArgs a) {
  __shared__ __align__(16) uint8_t win[ARNR_WARPS][AWS * AW + 16];
  __shared__ __align__(16) uint8_t srcb[ARNR_WARPS][256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t nblk = (uint32_t)a.bcols * a.brows;
  const uint32_t item = blockIdx.x * ARNR_WARPS + warp;
  if (item >= nblk * (a.n - 1)) return;
  uint32_t fi = item / nblk;
  if (fi >= a.center) fi++;  // skip the centre frame
  const uint32_t blk = item % nblk;
  const int bcol = (int)(blk % a.bcols), brow = (int)(blk / a.bcols);
  const int bx = bcol * 16, by = brow * 16;
  const int bw = min(16, a.w - bx), bh = min(16, a.h - by);
  const ArnrFrame ctr = a.frames[a.center];
  const ArnrFrame ref = a.frames[fi];
  uint8_t* W = win[warp];
  uint8_t* S = srcb[warp];
  // Source block (centre frame), zero outside bw x bh.
  for (int i = lane; i < 256; i += 32) {
    int r = i >> 4, c = i & 15;
    S[i] = (r < bh && c < bw) ? ctr.y[(size_t)(by + r) * ctr.y_stride + bx + c] : 0;
  }
  // Reference neighbourhood, edge-clamped to the visible plane (pel,
  // src/arnr.rs:149).
  for (int r = 0; r < AW; r++) {
    int yy = clampi(by - 15 + r, 0, a.h - 1);
    const uint8_t* row = ref.y + (size_t)yy * ref.y_stride;
    for (int c = lane; c < AW; c += 32) W[r * AWS + c] = row[clampi(bx - 15 + c, 0, a.w - 1)];
  }
  __syncwarp();
  const int k = lane >> 2, q = lane & 3;
  // Byte masks for the partial-width columns.
  uint32_t m[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    uint32_t mm = 0;
#pragma unroll
    for (int b = 0; b < 4; b++)
      if (4 * j + b < bw) mm |= 0xffu << (8 * b);
    m[j] = mm;
  }
  // SAD of candidate (x, y) over this lane's four rows.
  auto part = [&](int x, int y) -> uint32_t {
    uint32_t s = 0;
    const uint8_t* base = W + (15 + y + q * 4) * AWS + 15 + x;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      if (q * 4 + r < bh) {
        uint32_t a0, a1, a2, a3;
        load8u(base + r * AWS, a0, a1);
        load8u(base + r * AWS + 8, a2, a3);
        const uint32_t* sp = (const uint32_t*)(S + (q * 4 + r) * 16);
        s += __vsadu4(a0 & m[0], sp[0]) + __vsadu4(a1 & m[1], sp[1]) + __vsadu4(a2 & m[2], sp[2]) +
             __vsadu4(a3 & m[3], sp[3]);
      }
    }
    return s;
  };
  // Zero vector (all groups compute it; group 0's value is used).
  uint32_t s0 = part(0, 0);
  s0 += __shfl_xor_sync(FULL, s0, 1);
  s0 += __shfl_xor_sync(FULL, s0, 2);
  uint32_t best_sad = __shfl_sync(FULL, s0, 0);
  int bestx = 0, besty = 0;
  for (int step = 8; step >= 1; step >>= 1) {
    const int cx = bestx, cy = besty;
    // Candidate order (src/arnr.rs:274-283): (-s,-s) (0,-s) (s,-s) (-s,0)
    // (s,0) (-s,s) (0,s) (s,s) as (dx, dy).
    const int dx = (k == 0 || k == 3 || k == 5) ? -step : ((k == 1 || k == 6) ? 0 : step);
    const int dy = (k < 3) ? -step : (k < 5 ? 0 : step);
    const int x = cx + dx, y = cy + dy;
    const bool valid = x >= -15 && x <= 15 && y >= -15 && y <= 15;
    uint32_t s = valid ? part(x, y) : 0;
    s += __shfl_xor_sync(FULL, s, 1);
    s += __shfl_xor_sync(FULL, s, 2);
#pragma unroll
    for (int j = 0; j < 8; j++) {
      uint32_t sj = __shfl_sync(FULL, s, j * 4);
      const int jdx = (j == 0 || j == 3 || j == 5) ? -step : ((j == 1 || j == 6) ? 0 : step);
      const int jdy = (j < 3) ? -step : (j < 5 ? 0 : step);
      const int jx = cx + jdx, jy = cy + jdy;
      const bool jv = jx >= -15 && jx <= 15 && jy >= -15 && jy <= 15;
      if (jv && sj < best_sad) {
        best_sad = sj;
        bestx = jx;
        besty = jy;
      }
    }
  }
  if (lane == 0) {
    BlockMv o;
    o.mvx = (int16_t)bestx;
    o.mvy = (int16_t)besty;
    o.sad = best_sad;
    a.out[((size_t)fi * a.brows + brow) * a.bcols + bcol] = o;
  }
}

struct BlendArgs {
  const ArnrFrame* frames;
  const BlockMv* mv;
  uint32_t n, center, s_scale;
  int w, h, cw, ch, bcols, brows;
  uint8_t* y_out;
  uint8_t* u_out;
  uint8_t* v_out;
};

// One thread per output pixel of the three planes (luma first).
__global__ void __launch_bounds__(256) arnr_blend_kernel(BlendArgs a) {
  __shared__ uint32_t wt[256];
  for (int d = threadIdx.x; d < 256; d += blockDim.x)
    wt[d] = (16u * a.s_scale) / (a.s_scale + (uint32_t)(d * d));
  __syncthreads();
  const size_t ny = (size_t)a.w * a.h, nc = (size_t)a.cw * a.ch;
  const size_t total = ny + 2 * nc;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    int plane, x, y, pw, ph;
    if (i < ny) {
      plane = 0;
      y = (int)(i / a.w);
      x = (int)(i % a.w);
      pw = a.w;
      ph = a.h;
    } else {
      size_t j = i - ny;
      plane = j < nc ? 1 : 2;
      if (j >= nc) j -= nc;
      y = (int)(j / a.cw);
      x = (int)(j % a.cw);
      pw = a.cw;
      ph = a.ch;
    }
    const int blk_x = plane ? x >> 3 : x >> 4, blk_y = plane ? y >> 3 : y >> 4;
    const ArnrFrame c = a.frames[a.center];
    const uint8_t* cp = plane == 0 ? c.y : (plane == 1 ? c.u : c.v);
    const uint64_t cs = plane == 0 ? c.y_stride : c.uv_stride;
    const int ctr = cp[(size_t)y * cs + x];
    uint32_t acc = 16u * (uint32_t)ctr, ws = 16u;
    const int bw = min(16, a.w - blk_x * 16), bh = min(16, a.h - blk_y * 16);
    const uint32_t area = (uint32_t)(bw * bh);
    for (uint32_t fi = 0; fi < a.n; fi++) {
      if (fi == a.center) continue;
      const BlockMv m = a.mv[((size_t)fi * a.brows + blk_y) * a.bcols + blk_x];
      if (m.sad / area > 12u) continue;  // BLOCK_SAD_PER_PIXEL_CUTOFF
      int mvx = m.mvx, mvy = m.mvy;
      if (plane) {
        mvx /= 2;  // toward zero (src/arnr.rs:622)
        mvy /= 2;
      }
      const ArnrFrame f = a.frames[fi];
      const uint8_t* fp = plane == 0 ? f.y : (plane == 1 ? f.u : f.v);
      const uint64_t fs = plane == 0 ? f.y_stride : f.uv_stride;
      const int rx = clampi(x + mvx, 0, pw - 1), ry = clampi(y + mvy, 0, ph - 1);
      const int ref = fp[(size_t)ry * fs + rx];
      const int d = ref - ctr;
      const uint32_t wgt = wt[d < 0 ? -d : d];
      acc += wgt * (uint32_t)ref;
      ws += wgt;
    }
    const uint8_t o = (uint8_t)((acc + ws / 2) / ws);
    if (plane == 0) a.y_out[(size_t)y * a.w + x] = o;
    else if (plane == 1) a.u_out[(size_t)y * a.cw + x] = o;
    else a.v_out[(size_t)y * a.cw + x] = o;
  }
}

}  // namespace

extern "C" vp8a_status vp8a_build_arnr_altref(vp8a_ctx* ctx, const vp8a_i420* frames, uint32_t n,
                                              uint32_t center, uint32_t strength, uint8_t* y_out,
                                              uint8_t* u_out, uint8_t* v_out) {
  if (!ctx || !frames || !y_out || !u_out || !v_out) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (n == 0 || center >= n) {
    vp8a::set_error("build_arnr_altref: center index out of range");
    return VP8A_E_INVALID_ARGUMENT;
  }
  const vp8a_i420& c = frames[center];
  if (c.width == 0 || c.height == 0 || c.width > 0x3FFF || c.height > 0x3FFF) {
    vp8a::set_error("invalid dimensions");
    return VP8A_E_INVALID_DIMENSIONS;
  }
  for (uint32_t i = 0; i < n; i++)
    if (frames[i].width != c.width || frames[i].height != c.height) {
      vp8a::set_error("window frame dimensions differ from the centre frame");
      return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
    }
  const int w = (int)c.width, h = (int)c.height, cw = (w + 1) / 2, ch = (h + 1) / 2;
  for (uint32_t i = 0; i < n; i++)
    if (!frames[i].y || !frames[i].u || !frames[i].v || frames[i].y_stride < (uint64_t)w ||
        frames[i].uv_stride < (uint64_t)cw) {
      vp8a::set_error("frame planes missing or stride below width");
      return VP8A_E_INVALID_ARGUMENT;
    }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  vp8a_status s;
  std::vector<ArnrFrame> hf(n);
  for (uint32_t i = 0; i < n; i++) {
    const void* d;
    size_t yb = frames[i].y_stride * (size_t)(h - 1) + w, cb = frames[i].uv_stride * (size_t)(ch - 1) + cw;
    if ((s = st.in(frames[i].y, yb, &d)) != VP8A_OK) return s;
    hf[i].y = (const uint8_t*)d;
    if ((s = st.in(frames[i].u, cb, &d)) != VP8A_OK) return s;
    hf[i].u = (const uint8_t*)d;
    if ((s = st.in(frames[i].v, cb, &d)) != VP8A_OK) return s;
    hf[i].v = (const uint8_t*)d;
    hf[i].y_stride = frames[i].y_stride;
    hf[i].uv_stride = frames[i].uv_stride;
  }
  void* dframes = nullptr;
  if ((s = st.scratch(sizeof(ArnrFrame) * n, &dframes)) != VP8A_OK) return s;
  VP8A_CUDA(cudaMemcpyAsync(dframes, hf.data(), sizeof(ArnrFrame) * n, cudaMemcpyHostToDevice, ctx->stream));
  st.force_sync();  // hf must outlive the copy
  void *dy, *du, *dv;
  if ((s = st.out(y_out, (size_t)w * h, &dy)) != VP8A_OK) return s;
  if ((s = st.out(u_out, (size_t)cw * ch, &du)) != VP8A_OK) return s;
  if ((s = st.out(v_out, (size_t)cw * ch, &dv)) != VP8A_OK) return s;

  const int bcols = (w + 15) / 16, brows = (h + 15) / 16;
  const bool filter = strength != 0 && n >= 2;
  const uint32_t str = strength > 6 ? 6 : strength;
  void* dmv = nullptr;
  if ((s = st.scratch(sizeof(BlockMv) * (size_t)n * bcols * brows, &dmv)) != VP8A_OK) return s;
  if (filter) {
    SearchArgs sa{(const ArnrFrame*)dframes, n, center, w, h, bcols, brows, (BlockMv*)dmv};
    size_t items = (size_t)bcols * brows * (n - 1);
    arnr_search_kernel<<<vp8a::grid_for(items, ARNR_WARPS), ARNR_WARPS * 32, 0, ctx->stream>>>(sa);
    VP8A_CUDA(cudaGetLastError());
    ctx->launches++;
  }
  BlendArgs ba{(const ArnrFrame*)dframes, (const BlockMv*)dmv, filter ? n : 0u, filter ? center : 0u,
               8u << str, w, h, cw, ch, bcols, brows, (uint8_t*)dy, (uint8_t*)du, (uint8_t*)dv};
  if (!filter) {
    // Pass-through (src/arnr.rs:527-529): the blend with no window frames
    // reproduces the centre exactly. The centre is frames[0] of a
    // one-entry view.
    ba.frames = (const ArnrFrame*)dframes + center;
    ba.n = 1;
    ba.center = 0;
  }
  size_t total = (size_t)w * h + 2 * (size_t)cw * ch;
  unsigned grid = (unsigned)std::min<size_t>(vp8a::grid_for(total, 256), (size_t)ctx->sm_count * 16);
  arnr_blend_kernel<<<grid, 256, 0, ctx->stream>>>(ba);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return st.finish();
}
