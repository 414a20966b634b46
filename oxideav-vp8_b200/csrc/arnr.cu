// arnr.cu — the ARNR temporal filter (build_arnr_altref, src/arnr.rs:476).
//
// Two kernels:
//  * arnr_search_kernel — refine_search (src/arnr.rs:264-300) for every
//    (window frame != centre, 16x16 block): one CTA per strip of 8 blocks
//    of one frame, whose shared +/-15 px neighbourhood is staged
//    edge-clamped in shared memory once; one warp per block, the eight
//    candidates of each 8/4/2/1 round scored in parallel (four lanes each)
//    and folded in the reference's candidate order with strict '<'.
//  * arnr_blend_kernel — the per-pixel weighted temporal mean
//    (accumulate_* :337-459 + resolve_plane :670): each thread takes four
//    horizontally adjacent output pixels of one block, gathers the block's
//    alignment from each frame, applies the SAD occlusion guard (:605) and
//    the weight table (:307-323) to one motion-compensated word per frame,
//    and resolves in one pass. Integer sums are order-free, so gathering per pixel equals
//    the reference's frame-then-raster scatter. Every chroma pixel lies in
//    exactly one chroma block (block k covers [8k, 8k + ceil(bw/2)) and
//    ceil((bx+bw)/2) <= ceil(w/2)), so the clamped-overhang branch of
//    accumulate_chroma_block never adds a second contribution.
#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

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
  int aligned;  // every window plane base and row pitch is 4-byte aligned
  BlockMv* out;  // [n][brows][bcols]
};

constexpr int STRIP = 8;                    // blocks per CTA (one warp each)
constexpr int SWS = 164;  // row stride: rows four apart fall four banks apart
constexpr int SWW = SWS / 4;                // words per staged row

// One CTA per (window frame != centre, strip of 8 horizontally adjacent
// blocks). The strip's +-15 px neighbourhood in the frame (46 rows x 158
// columns, staged 164 wide, edge-clamped to the visible plane as pel does, src/arnr.rs:149)
// and its 16 source rows of the centre frame are staged once as 32-bit
// words; warp j then runs refine_search for block j of the strip on the
// staged window.
__device__ __forceinline__ void search_body(const SearchArgs& a, uint32_t bid) {
  __shared__ __align__(16) uint8_t win[AW * SWS + 16];
  __shared__ __align__(16) uint8_t srcs[16 * STRIP * 16];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int strips = (a.bcols + STRIP - 1) / STRIP;
  uint32_t fi = bid / ((uint32_t)strips * a.brows);
  const uint32_t rest = bid % ((uint32_t)strips * a.brows);
  if (fi >= a.center) fi++;  // skip the centre frame
  const int brow = (int)(rest / strips), strip = (int)(rest % strips);
  const int bx0 = strip * STRIP * 16, by = brow * 16;
  const ArnrFrame ctr = a.frames[a.center];
  const ArnrFrame ref = a.frames[fi];
  // Window: word k of row r holds columns x0 + 4k .. x0 + 4k + 3.
  const int x0 = bx0 - 15;
  const bool words = a.aligned && x0 >= 0 && x0 + SWS + 4 <= a.w;
  for (int i = threadIdx.x; i < AW * SWW; i += blockDim.x) {
    const int r = i / SWW, k = i - SWW * r;
    const uint8_t* row = ref.y + (size_t)clampi(by - 15 + r, 0, a.h - 1) * ref.y_stride;
    uint32_t v;
    if (words) {
      const int x = x0 + 4 * k;
      const uint32_t* p = reinterpret_cast<const uint32_t*>(row + (x & ~3));
      v = __funnelshift_r(__ldg(p), __ldg(p + 1), 8 * (x & 3));
    } else {
      v = 0;
#pragma unroll
      for (int c = 0; c < 4; c++) v |= (uint32_t)__ldg(row + clampi(x0 + 4 * k + c, 0, a.w - 1)) << (8 * c);
    }
    *reinterpret_cast<uint32_t*>(win + r * SWS + 4 * k) = v;
  }
  // Source rows of the strip (centre frame), zero outside the picture.
  for (int i = threadIdx.x; i < 16 * STRIP * 4; i += blockDim.x) {
    const int r = i / (STRIP * 4), k = i - STRIP * 4 * r, x = bx0 + 4 * k;
    uint32_t v = 0;
    if (by + r < a.h) {
      const uint8_t* row = ctr.y + (size_t)(by + r) * ctr.y_stride;
      if (a.aligned && x + 4 <= a.w) {
        v = __ldg(reinterpret_cast<const uint32_t*>(row + x));
      } else {
#pragma unroll
        for (int c = 0; c < 4; c++)
          if (x + c < a.w) v |= (uint32_t)__ldg(row + x + c) << (8 * c);
      }
    }
    // Stored block-major: block j's 16 x 16 source at srcs + 256 j.
    const int j = k >> 2, kk = k & 3;
    *reinterpret_cast<uint32_t*>(srcs + 256 * j + 16 * r + 4 * kk) = v;
  }
  __syncthreads();
  const int bcol = strip * STRIP + warp;
  if (bcol >= a.bcols) return;  // past the picture's last block (after the only barrier)
  const int bx = bcol * 16;
  const int bw = min(16, a.w - bx), bh = min(16, a.h - by);
  const uint8_t* W = win + 16 * warp;  // this block's 46 x 46 window
  const uint8_t* S = srcs + 256 * warp;
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
    const uint8_t* base = W + (15 + y + q * 4) * SWS + 15 + x;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      if (q * 4 + r < bh) {
        uint32_t a0, a1, a2, a3;
        load8u(base + r * SWS, a0, a1);
        load8u(base + r * SWS + 8, a2, a3);
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
    // The reference folds the eight candidates in order with a strict '<'
    // against the running best: that is the smallest (sad, order) pair,
    // taken when its sad beats the incumbent. SADs are < 2^17.
    const uint32_t r = __reduce_min_sync(FULL, valid ? (s << 3) | (uint32_t)k : 0xffffffffu);
    if (r != 0xffffffffu && (r >> 3) < best_sad) {
      const int j = (int)(r & 7);
      best_sad = r >> 3;
      bestx = cx + ((j == 0 || j == 3 || j == 5) ? -step : ((j == 1 || j == 6) ? 0 : step));
      besty = cy + ((j < 3) ? -step : (j < 5 ? 0 : step));
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

__global__ void __launch_bounds__(STRIP * 32) arnr_search_kernel(SearchArgs a) { search_body(a, blockIdx.x); }

__global__ void __launch_bounds__(STRIP * 32)
    arnr_search_batch_kernel(const SearchArgs* __restrict__ jobs, const uint32_t* __restrict__ cta_start, int n_jobs) {
  __shared__ SearchArgs sa;
  __shared__ uint32_t first[2];
  find_job(jobs, cta_start, n_jobs, &sa, first);
  search_body(sa, blockIdx.x - first[0]);
}

struct BlendArgs {
  const ArnrFrame* frames;
  const BlockMv* mv;
  uint32_t n, center, s_scale;
  int w, h, cw, ch, bcols, brows;
  int aligned_in;  // every window plane base and row pitch is 4-byte aligned
  int aligned_out;  // the output planes' rows start 4-byte aligned
  uint8_t* y_out;
  uint8_t* u_out;
  uint8_t* v_out;
  uint64_t ys, cs;  // output row pitches
  int ow, oh;       // output luma extent (w x h, or the MB-padded size)
  int ocw, och;     // output chroma extent
};

constexpr int BLEND_BLOCKS = 2;                 // 16x16 blocks per CTA step
constexpr int BLEND_THREADS = 96 * BLEND_BLOCKS;  // 64 luma + 2 x 16 chroma words per block

// Four bytes of row `row` at columns x .. x+3, each clamped to [0, pw). The
// word form needs a row whose base and pitch are 4-byte aligned and the
// aligned pair [x & ~3, (x & ~3) + 8) inside [0, pw): that pair covers the
// four bytes and never leaves the row.
__device__ __forceinline__ uint32_t row4(const uint8_t* row, int x, int pw, bool words) {
  if (words && x >= 0 && x + 8 <= pw) {
    const uint32_t* p = reinterpret_cast<const uint32_t*>(row + (x & ~3));
    return __funnelshift_r(__ldg(p), __ldg(p + 1), 8 * (x & 3));
  }
  uint32_t v = 0;
#pragma unroll
  for (int c = 0; c < 4; c++) v |= (uint32_t)__ldg(row + clampi(x + c, 0, pw - 1)) << (8 * c);
  return v;
}

// floor(a / d) for a < 2^24, 16 <= d < 2^16: the single-precision estimate
// is within one below the quotient; the remainder test corrects it.
__device__ __forceinline__ uint32_t udiv_small(uint32_t a, uint32_t d) {
  uint32_t q = __float2uint_rz(__uint2float_rn(a) * __frcp_rn(__uint2float_rn(d)));
  const int r = (int)a - (int)(q * d);
  if (r < 0) q--;
  else if (r >= (int)d) q++;
  return q;
}

// Each thread blends four horizontally adjacent output pixels of one block:
// threads 0-63 of a block's group the 16x16 luma block (row t / 4, columns
// 4 (t % 4) ..), 64-79 the 8x8 U block and 80-95 the 8x8 V block. The
// block's alignment per window frame is uniform, so every frame's four
// motion-compensated samples are one unaligned word of one row. The
// alignments of the CTA's blocks are staged in shared memory first (frames
// past BLEND_MAX_FRAMES are read from global memory).
constexpr int BLEND_MAX_FRAMES = 32;

// CTA `cta` of the `ncta` that blend job `a` (grid-stride over its blocks).
__device__ __forceinline__ void blend_body(const BlendArgs& a, uint32_t cta, uint32_t ncta) {
  __shared__ uint32_t wt[256];
  __shared__ int2 smv[BLEND_BLOCKS][BLEND_MAX_FRAMES];  // (mvx, mvy); mvx = INT_MIN: frame not used
  for (int d = threadIdx.x; d < 256; d += blockDim.x)
    wt[d] = (16u * a.s_scale) / (a.s_scale + (uint32_t)(d * d));
  const int g = threadIdx.x / 96, t = threadIdx.x % 96;
  const uint32_t nblk = (uint32_t)a.bcols * a.brows;
  const ArnrFrame c = a.frames[a.center];
  const uint32_t nst = min(a.n, (uint32_t)BLEND_MAX_FRAMES);
  for (uint32_t b0 = cta * BLEND_BLOCKS; b0 < nblk; b0 += ncta * BLEND_BLOCKS) {
    const uint32_t b = b0 + g;
    const int bcol = (int)(b % (uint32_t)a.bcols), brow = (int)(b / (uint32_t)a.bcols);
    // Occlusion guard: sad / (bw * bh) > 12 (BLOCK_SAD_PER_PIXEL_CUTOFF)
    // is sad >= 13 * area for integers.
    const uint32_t area = (uint32_t)(min(16, a.w - bcol * 16) * min(16, a.h - brow * 16));
    __syncthreads();  // the previous step's readers are done with smv
    for (uint32_t fi = t; fi < nst && b < nblk; fi += 96) {
      int2 v = make_int2(INT_MIN, 0);
      if (fi != a.center) {
        const BlockMv m = a.mv[((size_t)fi * a.brows + brow) * a.bcols + bcol];
        if (m.sad < 13u * area) v = make_int2(m.mvx, m.mvy);
      }
      smv[g][fi] = v;
    }
    __syncthreads();
    if (b >= nblk) continue;
    int plane, x, y, pw, ph;
    if (t < 64) {
      plane = 0;
      x = bcol * 16 + 4 * (t & 3);
      y = brow * 16 + (t >> 2);
      pw = a.w;
      ph = a.h;
    } else {
      const int k = t - 64;
      plane = 1 + (k >> 4);
      x = bcol * 8 + 4 * (k & 1);
      y = brow * 8 + ((k >> 1) & 7);
      pw = a.cw;
      ph = a.ch;
    }
    if (x >= pw || y >= ph) continue;
    const int nvalid = min(4, pw - x);
    const uint8_t* cp = plane == 0 ? c.y : (plane == 1 ? c.u : c.v);
    const uint64_t cs = plane == 0 ? c.y_stride : c.uv_stride;
    const uint32_t ctr = row4(cp + (uint64_t)y * cs, x, pw, a.aligned_in);
    uint32_t acc[4], ws[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      acc[j] = 16u * ((ctr >> (8 * j)) & 0xffu);
      ws[j] = 16u;
    }
#pragma unroll 2
    for (uint32_t fi = 0; fi < a.n; fi++) {
      int2 mv;
      if (fi < nst) {
        mv = smv[g][fi];
      } else {
        mv = make_int2(INT_MIN, 0);
        if (fi != a.center) {
          const BlockMv m = a.mv[((size_t)fi * a.brows + brow) * a.bcols + bcol];
          if (m.sad < 13u * area) mv = make_int2(m.mvx, m.mvy);
        }
      }
      if (mv.x == INT_MIN) continue;
      int mvx = mv.x, mvy = mv.y;
      if (plane) {
        mvx /= 2;  // toward zero (src/arnr.rs:622)
        mvy /= 2;
      }
      const ArnrFrame f = a.frames[fi];
      const uint8_t* fp = plane == 0 ? f.y : (plane == 1 ? f.u : f.v);
      const uint64_t fs = plane == 0 ? f.y_stride : f.uv_stride;
      const uint32_t ref = row4(fp + (uint64_t)clampi(y + mvy, 0, ph - 1) * fs, x + mvx, pw, a.aligned_in);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int rv = (int)((ref >> (8 * j)) & 0xffu), cv = (int)((ctr >> (8 * j)) & 0xffu);
        const uint32_t wgt = wt[rv > cv ? rv - cv : cv - rv];
        acc[j] += wgt * (uint32_t)rv;
        ws[j] += wgt;
      }
    }
    uint32_t o = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) o |= udiv_small(acc[j] + ws[j] / 2, ws[j]) << (8 * j);
    uint8_t* const base = plane == 0 ? a.y_out : (plane == 1 ? a.u_out : a.v_out);
    const uint64_t os = plane == 0 ? a.ys : a.cs;
    const int opw = plane == 0 ? a.ow : a.ocw, oph = plane == 0 ? a.oh : a.och;
    const uint8_t last = (uint8_t)(o >> (8 * (nvalid - 1)));
    // The visible pixels, then (MB-padded output) the edge replication of
    // the last column into the padding columns and of the last row into the
    // padding rows, as the MB-padded reference planes hold them.
    const int rows = y == ph - 1 ? oph - y : 1;
    for (int rr = 0; rr < rows; rr++) {
      uint8_t* op = base + (size_t)(y + rr) * os;
      if (nvalid == 4 && a.aligned_out) {
        *reinterpret_cast<uint32_t*>(op + x) = o;
      } else {
        for (int j = 0; j < nvalid; j++) op[x + j] = (uint8_t)(o >> (8 * j));
      }
      if (x + nvalid == pw)
        for (int c = pw; c < opw; c++) op[c] = last;
    }
  }
}

__global__ void __launch_bounds__(BLEND_THREADS) arnr_blend_kernel(BlendArgs a) {
  blend_body(a, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(BLEND_THREADS)
    arnr_blend_batch_kernel(const BlendArgs* __restrict__ jobs, const uint32_t* __restrict__ cta_start, int n_jobs) {
  __shared__ BlendArgs sa;
  __shared__ uint32_t first[2];
  find_job(jobs, cta_start, n_jobs, &sa, first);
  blend_body(sa, blockIdx.x - first[0], first[1]);
}

}  // namespace

namespace {

// One ARNR job prepared: inputs staged, the kernels' arguments, and their
// CTA counts (no search when the window does not filter).
struct ArnrPrepared {
  SearchArgs sa;
  BlendArgs ba;
  uint32_t search_ctas, blend_ctas;
};

// Where an anchor goes: packed visible planes (row pitch = width, the
// ArnrPicture layout), or MB-padded planes with their own pitches (the
// KeyframePlanes layout of a reference, padding edge-replicated).
struct ArnrOut {
  uint8_t* y;
  uint8_t* u;
  uint8_t* v;
  uint64_t ys, cs;        // 0: packed
  uint32_t mb_cols, mb_rows;  // MB-padded output grid (0: packed)
};

// `hf` is the host copy of the frame table (uploaded before this returns).
vp8a_status prepare_arnr(vp8a_ctx* ctx, vp8a::Stager& st, const vp8a_i420* frames, uint32_t n, uint32_t center,
                         uint32_t strength, const ArnrOut& out, std::vector<ArnrFrame>& hf, ArnrPrepared* P) {
  if (!frames || !out.y || !out.u || !out.v) {
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
  vp8a_status s;
  hf.assign(n, ArnrFrame{});
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
  if ((s = st.upload(hf.data(), sizeof(ArnrFrame) * n, &dframes)) != VP8A_OK) return s;
  const bool padded = out.mb_cols != 0;
  const int ow = padded ? (int)out.mb_cols * 16 : w, oh = padded ? (int)out.mb_rows * 16 : h;
  const int ocw = padded ? (int)out.mb_cols * 8 : cw, och = padded ? (int)out.mb_rows * 8 : ch;
  const uint64_t ys = padded ? out.ys : (uint64_t)w, cs = padded ? out.cs : (uint64_t)cw;
  if (padded && ((int)out.mb_cols != (w + 15) / 16 || (int)out.mb_rows != (h + 15) / 16)) {
    vp8a::set_error("output planes do not match the frames' MB grid");
    return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
  }
  if (padded && (ys < (uint64_t)ow || cs < (uint64_t)ocw)) {
    vp8a::set_error("output stride below the MB-padded width");
    return VP8A_E_INVALID_ARGUMENT;
  }
  void *dy, *du, *dv;
  // Padded host planes may have a pitch wider than their rows: staged
  // in and out, so the bytes between rows come back unchanged.
  auto stage_out = [&](void* p, size_t bytes, void** d) { return padded ? st.inout(p, bytes, d) : st.out(p, bytes, d); };
  if ((s = stage_out(out.y, ys * (size_t)(oh - 1) + ow, &dy)) != VP8A_OK) return s;
  if ((s = stage_out(out.u, cs * (size_t)(och - 1) + ocw, &du)) != VP8A_OK) return s;
  if ((s = stage_out(out.v, cs * (size_t)(och - 1) + ocw, &dv)) != VP8A_OK) return s;

  const int bcols = (w + 15) / 16, brows = (h + 15) / 16;
  const bool filter = strength != 0 && n >= 2;
  const uint32_t str = strength > 6 ? 6 : strength;
  void* dmv = nullptr;
  if ((s = st.scratch(sizeof(BlockMv) * (size_t)n * bcols * brows, &dmv)) != VP8A_OK) return s;
  int aligned = 1;
  for (uint32_t i = 0; i < n; i++) aligned &= (((uintptr_t)hf[i].y | hf[i].y_stride) & 3) == 0;
  P->sa = SearchArgs{(const ArnrFrame*)dframes, n, center, w, h, bcols, brows, aligned, (BlockMv*)dmv};
  P->search_ctas = filter ? (uint32_t)((bcols + STRIP - 1) / STRIP) * brows * (n - 1) : 0u;
  int aligned_in = 1;
  for (uint32_t i = 0; i < n; i++)
    aligned_in &= (((uintptr_t)hf[i].y | (uintptr_t)hf[i].u | (uintptr_t)hf[i].v | hf[i].y_stride |
                     hf[i].uv_stride) & 3) == 0;
  const int aligned_out = (((uintptr_t)dy | (uintptr_t)du | (uintptr_t)dv | (uintptr_t)ys | (uintptr_t)cs) & 3) == 0;
  P->ba = BlendArgs{(const ArnrFrame*)dframes, (const BlockMv*)dmv, filter ? n : 0u, filter ? center : 0u,
                    8u << str, w, h, cw, ch, bcols, brows, aligned_in, aligned_out,
                    (uint8_t*)dy, (uint8_t*)du, (uint8_t*)dv, ys, cs, ow, oh, ocw, och};
  if (!filter) {
    // Pass-through (src/arnr.rs:527-529): the blend with no window frames
    // reproduces the centre exactly. The centre is frames[0] of a
    // one-entry view.
    P->ba.frames = (const ArnrFrame*)dframes + center;
    P->ba.n = 1;
    P->ba.center = 0;
  }
  const size_t nblk = (size_t)bcols * brows;
  P->blend_ctas = (uint32_t)std::min<size_t>(vp8a::grid_for(nblk, BLEND_BLOCKS), (size_t)ctx->sm_count * 16);
  return VP8A_OK;
}

}  // namespace

namespace {

vp8a_status build_one(vp8a_ctx* ctx, const vp8a_i420* frames, uint32_t n, uint32_t center, uint32_t strength,
                      const ArnrOut& out) {
  if (!ctx) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  ArnrPrepared P;
  std::vector<ArnrFrame> hf;
  vp8a_status s = prepare_arnr(ctx, st, frames, n, center, strength, out, hf, &P);
  if (s != VP8A_OK) return s;
  if (P.search_ctas) {
    arnr_search_kernel<<<P.search_ctas, STRIP * 32, 0, ctx->stream>>>(P.sa);
    VP8A_CUDA(cudaGetLastError());
    ctx->launches++;
  }
  arnr_blend_kernel<<<P.blend_ctas, BLEND_THREADS, 0, ctx->stream>>>(P.ba);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return st.finish();
}

ArnrOut planes_out(const vp8a_planes* p) {
  return ArnrOut{(uint8_t*)p->y, (uint8_t*)p->u, (uint8_t*)p->v, p->y_stride, p->uv_stride, p->mb_cols, p->mb_rows};
}

}  // namespace

extern "C" vp8a_status vp8a_build_arnr_altref(vp8a_ctx* ctx, const vp8a_i420* frames, uint32_t n,
                                              uint32_t center, uint32_t strength, uint8_t* y_out,
                                              uint8_t* u_out, uint8_t* v_out) {
  return build_one(ctx, frames, n, center, strength, ArnrOut{y_out, u_out, v_out, 0, 0, 0, 0});
}

extern "C" vp8a_status vp8a_build_arnr_altref_planes(vp8a_ctx* ctx, const vp8a_i420* frames, uint32_t n,
                                                     uint32_t center, uint32_t strength, const vp8a_planes* out) {
  if (!out || out->mb_cols == 0 || out->mb_rows == 0) {
    vp8a::set_error("null or empty output planes");
    return VP8A_E_INVALID_ARGUMENT;
  }
  return build_one(ctx, frames, n, center, strength, planes_out(out));
}

namespace {

// Every job's search in one launch and every job's blend in another; `job`
// gives job j's (frames, n, center, strength) and output.
template <class Job, class OutOf>
vp8a_status build_batch(vp8a_ctx* ctx, const Job* jobs, uint32_t n_jobs, OutOf out_of) {
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
  vp8a_status s;
  std::vector<SearchArgs> sj;
  std::vector<BlendArgs> bj;
  std::vector<uint32_t> s_start{0}, b_start{0};
  std::vector<std::vector<ArnrFrame>> hf(n_jobs);
  for (uint32_t j = 0; j < n_jobs; j++) {
    const Job& J = jobs[j];
    ArnrPrepared P;
    if ((s = prepare_arnr(ctx, st, J.frames, J.n, J.center, J.strength, out_of(J), hf[j], &P)) != VP8A_OK) return s;
    if (P.search_ctas) {
      sj.push_back(P.sa);
      s_start.push_back(s_start.back() + P.search_ctas);
    }
    bj.push_back(P.ba);
    b_start.push_back(b_start.back() + P.blend_ctas);
  }
  // Job tables: search args, search CTA offsets, blend args, blend CTA offsets.
  const size_t o_ss = sizeof(SearchArgs) * sj.size(), o_ba = (o_ss + sizeof(uint32_t) * s_start.size() + 15) & ~15,
               o_bs = o_ba + sizeof(BlendArgs) * bj.size(), total = o_bs + sizeof(uint32_t) * b_start.size();
  std::vector<uint8_t> blob(total, 0);
  if (!sj.empty()) memcpy(blob.data(), sj.data(), o_ss);
  memcpy(blob.data() + o_ss, s_start.data(), sizeof(uint32_t) * s_start.size());
  memcpy(blob.data() + o_ba, bj.data(), sizeof(BlendArgs) * bj.size());
  memcpy(blob.data() + o_bs, b_start.data(), sizeof(uint32_t) * b_start.size());
  void* d;
  if ((s = st.upload(blob.data(), total, &d)) != VP8A_OK) return s;
  const uint8_t* db = (const uint8_t*)d;
  if (!sj.empty()) {
    arnr_search_batch_kernel<<<s_start.back(), STRIP * 32, 0, ctx->stream>>>(
        (const SearchArgs*)db, (const uint32_t*)(db + o_ss), (int)sj.size());
    VP8A_CUDA(cudaGetLastError());
    ctx->launches++;
  }
  arnr_blend_batch_kernel<<<b_start.back(), BLEND_THREADS, 0, ctx->stream>>>(
      (const BlendArgs*)(db + o_ba), (const uint32_t*)(db + o_bs), (int)bj.size());
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return st.finish();
}

}  // namespace

extern "C" vp8a_status vp8a_build_arnr_altrefs(vp8a_ctx* ctx, const vp8a_arnr_job* jobs, uint32_t n_jobs) {
  return build_batch(ctx, jobs, n_jobs,
                     [](const vp8a_arnr_job& J) { return ArnrOut{J.y_out, J.u_out, J.v_out, 0, 0, 0, 0}; });
}

extern "C" vp8a_status vp8a_build_arnr_altrefs_planes(vp8a_ctx* ctx, const vp8a_arnr_planes_job* jobs,
                                                      uint32_t n_jobs) {
  for (uint32_t j = 0; jobs && j < n_jobs; j++)
    if (jobs[j].out.mb_cols == 0 || jobs[j].out.mb_rows == 0) {
      vp8a::set_error("empty output planes");
      return VP8A_E_INVALID_ARGUMENT;
    }
  return build_batch(ctx, jobs, n_jobs, [](const vp8a_arnr_planes_job& J) { return planes_out(&J.out); });
}
