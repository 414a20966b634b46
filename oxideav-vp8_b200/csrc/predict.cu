// predict.cu — §18 inter prediction (motion compensation) on the GPU:
//   vp8a_predict_inter_mb    (predict_inter_mb, src/motion_comp.rs:1986)
//   vp8a_predict_split_mv    (predict_split_mv, src/motion_comp.rs:2228)
//   vp8a_predict_inter_frame (the prediction pick_mb_for_ref builds for its
//                             chosen mode, src/encoder.rs:8704-8735)
//
// Work decomposition. The reference interpolates a whole-MB vector as one
// 16x16 luma and two 8x8 chroma blocks and a SPLITMV MB as 4x4 blocks; the
// §18.3 dot product of an output sample does not depend on the tiling, so
// every MB is cut into the same 48 tasks here: 32 luma (16 4x4 blocks x 2
// row pairs) and 16 chroma (4 blocks of U and of V x 2 row pairs). A CTA of
// 128 threads takes 8 MBs per step, 384 tasks = 3 per thread.
//
// Step: (1) 16 threads per MB derive the eighth-pel vectors of its 16 luma
// and 4 chroma blocks (stored_luma_mv, chroma_mv or split_chroma_mvs,
// apply_full_pixel); (2) the CTA copies the edge-clamped source of its MBs
// into shared memory as 32-bit words — one 21x21 luma and two 13x13 chroma
// regions for a whole-MB vector, 24 9x9 block halos for SPLITMV; (3) each task reads a
// 12-byte-wide, 7-row window as 32-bit words and runs the horizontal pass
// (4 outputs per row, dp4a with the tap row pre-shifted per output column),
// packs the 8-bit intermediate with saturation, transposes it with byte
// permutes and runs the vertical pass the same way. A zero fraction is the
// identity filter, taken as a byte select.
#include <algorithm>

#include "vp8a_internal.cuh"

namespace {

constexpr int PR_THREADS = 128;
constexpr int PR_MBS = 8;           // MBs per CTA step
constexpr int PR_TASKS = 48;        // tasks per MB
constexpr int SLOT_BYTES = 2592;    // 24 block halos of 9 rows x 12 bytes
constexpr int WY_STRIDE = 24, WC_STRIDE = 16, WU_OFF = 504, WV_OFF = 712;  // whole-MB layout
constexpr int HALO_STRIDE = 12, HALO_BYTES = 108;                          // SPLITMV layout
constexpr int MAX_PRED_REFS = 3;
constexpr int WHOLE_ROWS = 21 + 2 * 13, SPLIT_ROWS = 24 * 9;

// §18.3 tap tables (SIXTAP_FILTERS / BILINEAR_FILTERS, src/motion_comp.rs:294-334).
__constant__ int c_taps[2][8][6] = {
    {{0, 0, 128, 0, 0, 0},
     {0, -6, 123, 12, -1, 0},
     {2, -11, 108, 36, -8, 1},
     {0, -9, 93, 50, -6, 0},
     {3, -16, 77, 77, -16, 3},
     {0, -6, 50, 93, -9, 0},
     {1, -8, 36, 108, -11, 2},
     {0, -1, 12, 123, -6, 0}},
    {{0, 0, 128, 0, 0, 0},
     {0, 0, 112, 16, 0, 0},
     {0, 0, 96, 32, 0, 0},
     {0, 0, 80, 48, 0, 0},
     {0, 0, 64, 64, 0, 0},
     {0, 0, 48, 80, 0, 0},
     {0, 0, 32, 96, 0, 0},
     {0, 0, 16, 112, 0, 0}},
};

enum PredMode { PRED_WHOLE = 0, PRED_SPLIT = 1, PRED_FRAME = 2 };

struct PredPlanes {
  const uint8_t* y;
  const uint8_t* u;
  const uint8_t* v;
  uint64_t ys, uvs;
};

struct PredArgs {
  PredPlanes refs[MAX_PRED_REFS];
  uint8_t ref_ids[MAX_PRED_REFS];
  int n_refs;
  int lw, lh, cw, ch;  // MB-padded plane sizes of the references
  int mb_cols;         // frame mode: raster order of decisions
  uint32_t n;          // MBs
  const uint32_t* mb_xy;
  const vp8a_mv* mvs;  // whole: 1 per MB, split: 16 per MB
  const vp8a_mb_decision* dec;
  int full_pixel;
  int filter_set;
  // Output: batched -> out + 384 i; frame -> planes at the MB position.
  uint8_t* out;
  uint8_t *oy, *ou, *ov;
  uint64_t oys, ouvs;
  int aligned_out;  // every output row start is 4-byte aligned
  int aligned_src;  // every reference plane base and row pitch is 4-byte aligned
};

struct Job {
  const uint8_t* y;
  const uint8_t* u;
  const uint8_t* v;
  uint64_t ys, uvs;
  uint8_t *oy, *ou, *ov;
  uint64_t oys, ouvs;
  int x16, y16;  // MB luma origin (clamped so every offset fits int)
  int split;
  int skip;
  short2 lmv[16];  // eighth-pel (row, col) per luma block
  short2 cmv[4];   // eighth-pel per chroma block
};

__device__ __forceinline__ int dp4a_us(uint32_t a, uint32_t b, int c) {
  int d;
  asm("dp4a.u32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

// (c << 16) | (sat_u8(hi) << 8) | sat_u8(lo)
__device__ __forceinline__ uint32_t pack2_sat(int lo, int hi, uint32_t rest) {
  uint32_t d;
  asm("cvt.pack.sat.u8.s32.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(hi), "r"(lo), "r"(rest));
  return d;
}

__device__ __forceinline__ uint32_t pack4_sat(int v0, int v1, int v2, int v3) {
  return pack2_sat(v0, v1, pack2_sat(v2, v3, 0u));
}

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t s) { return __byte_perm(a, b, s); }

// stored_luma_mv (src/motion_comp.rs:187): i16 wrapping doubling.
__device__ __forceinline__ int dbl16(int v) { return (int)(short)(unsigned short)((unsigned)v * 2u); }
// avg (src/motion_comp.rs:209).
__device__ __forceinline__ int avg_sum(int s) { return s >= 0 ? (s + 4) >> 3 : -((-s + 4) >> 3); }

// One 4-column output row pair of a 4x4 block: rows 0..6 of `win` (stride
// ws) are the block's halo rows 2h .. 2h+6 starting at halo column 0.
__device__ __forceinline__ void predict_pair(const uint8_t* win, int ws, int mx, int my, const uint32_t (*tw)[4][3],
                                             uint32_t& o0, uint32_t& o1) {
  uint32_t R[7];
  if (mx == 0) {
#pragma unroll
    for (int i = 0; i < 7; i++) {
      const uint32_t* w = reinterpret_cast<const uint32_t*>(win + i * ws);
      R[i] = prmt(w[0], w[1], 0x5432);
    }
  } else {
    const uint32_t(*T)[3] = tw[mx];
    const uint32_t t00 = T[0][0], t01 = T[0][1], t10 = T[1][0], t11 = T[1][1];
    const uint32_t t20 = T[2][0], t21 = T[2][1], t30 = T[3][0], t31 = T[3][1], t32 = T[3][2];
#pragma unroll
    for (int i = 0; i < 7; i++) {
      const uint32_t* w = reinterpret_cast<const uint32_t*>(win + i * ws);
      const uint32_t A = w[0], B = w[1], C = w[2];
      const int a0 = dp4a_us(A, t00, dp4a_us(B, t01, 64));
      const int a1 = dp4a_us(A, t10, dp4a_us(B, t11, 64));
      const int a2 = dp4a_us(A, t20, dp4a_us(B, t21, 64));
      const int a3 = dp4a_us(A, t30, dp4a_us(B, t31, dp4a_us(C, t32, 64)));
      R[i] = pack4_sat(a0 >> 7, a1 >> 7, a2 >> 7, a3 >> 7);
    }
  }
  if (my == 0) {
    o0 = R[2];
    o1 = R[3];
    return;
  }
  // Column words: L[j] = column j of rows 0..3, H[j] = rows 4..6 (+ 0).
  const uint32_t x01l = prmt(R[0], R[1], 0x5140), x01h = prmt(R[0], R[1], 0x7362);
  const uint32_t x23l = prmt(R[2], R[3], 0x5140), x23h = prmt(R[2], R[3], 0x7362);
  const uint32_t x45l = prmt(R[4], R[5], 0x5140), x45h = prmt(R[4], R[5], 0x7362);
  const uint32_t x67l = prmt(R[6], 0u, 0x5140), x67h = prmt(R[6], 0u, 0x7362);
  const uint32_t L0 = prmt(x01l, x23l, 0x5410), L1 = prmt(x01l, x23l, 0x7632);
  const uint32_t L2 = prmt(x01h, x23h, 0x5410), L3 = prmt(x01h, x23h, 0x7632);
  const uint32_t H0 = prmt(x45l, x67l, 0x5410), H1 = prmt(x45l, x67l, 0x7632);
  const uint32_t H2 = prmt(x45h, x67h, 0x5410), H3 = prmt(x45h, x67h, 0x7632);
  const uint32_t(*V)[3] = tw[my];
  const uint32_t v00 = V[0][0], v01 = V[0][1], v10 = V[1][0], v11 = V[1][1];
  o0 = pack4_sat(dp4a_us(L0, v00, dp4a_us(H0, v01, 64)) >> 7, dp4a_us(L1, v00, dp4a_us(H1, v01, 64)) >> 7,
                 dp4a_us(L2, v00, dp4a_us(H2, v01, 64)) >> 7, dp4a_us(L3, v00, dp4a_us(H3, v01, 64)) >> 7);
  o1 = pack4_sat(dp4a_us(L0, v10, dp4a_us(H0, v11, 64)) >> 7, dp4a_us(L1, v10, dp4a_us(H1, v11, 64)) >> 7,
                 dp4a_us(L2, v10, dp4a_us(H2, v11, 64)) >> 7, dp4a_us(L3, v10, dp4a_us(H3, v11, 64)) >> 7);
}

__device__ __forceinline__ void store_row(uint8_t* p, uint32_t v, int aligned) {
  if (aligned) {
    *reinterpret_cast<uint32_t*>(p) = v;
  } else {
    p[0] = (uint8_t)v;
    p[1] = (uint8_t)(v >> 8);
    p[2] = (uint8_t)(v >> 16);
    p[3] = (uint8_t)(v >> 24);
  }
}

// Row i of MB slot S's staging list: one row of one region, copied to
// shared memory so that smem byte c of the row is source column x0 + c of
// source row y0 + r (edge-clamped; bytes past the region's `ncols` are
// don't-care). A whole-MB vector has 21 luma rows of 21 bytes and 2 x 13
// chroma rows of 13; SPLITMV has 24 x 9 block-halo rows of 9. Rows inside
// the plane horizontally are read as aligned 32-bit words and realigned with
// funnel shifts — the plane width is a multiple of 4, so a word that starts
// inside it ends inside it; rows that straddle an edge take clamped bytes.
__device__ __forceinline__ void stage_row(const Job& J, uint8_t* S, int i, const PredArgs& a) {
  const uint8_t* plane;
  uint64_t stride;
  int w, h, x0, y0, r, ncols, off;
  if (!J.split) {
    if (i < 21) {
      r = i;
      plane = J.y;
      stride = J.ys;
      w = a.lw;
      h = a.lh;
      x0 = J.x16 + (J.lmv[0].y >> 3) - 2;
      y0 = J.y16 + (J.lmv[0].x >> 3) - 2;
      ncols = 21;
      off = r * WY_STRIDE;
    } else {
      const int p = i >= 34;
      r = i - 21 - 13 * p;
      plane = p ? J.v : J.u;
      stride = J.uvs;
      w = a.cw;
      h = a.ch;
      x0 = (J.x16 >> 1) + (J.cmv[0].y >> 3) - 2;
      y0 = (J.y16 >> 1) + (J.cmv[0].x >> 3) - 2;
      ncols = 13;
      off = (p ? WV_OFF : WU_OFF) + r * WC_STRIDE;
    }
  } else {
    const int blk = i / 9;
    r = i - 9 * blk;
    ncols = 9;
    off = blk * HALO_BYTES + r * HALO_STRIDE;
    if (blk < 16) {
      const short2 m = J.lmv[blk];
      plane = J.y;
      stride = J.ys;
      w = a.lw;
      h = a.lh;
      x0 = J.x16 + 4 * (blk & 3) + (m.y >> 3) - 2;
      y0 = J.y16 + 4 * (blk >> 2) + (m.x >> 3) - 2;
    } else {
      const int cb = (blk - 16) & 3;
      const short2 m = J.cmv[cb];
      plane = blk < 20 ? J.u : J.v;
      stride = J.uvs;
      w = a.cw;
      h = a.ch;
      x0 = (J.x16 >> 1) + 4 * (cb & 1) + (m.y >> 3) - 2;
      y0 = (J.y16 >> 1) + 4 * (cb >> 1) + (m.x >> 3) - 2;
    }
  }
  uint32_t* dst = reinterpret_cast<uint32_t*>(S + off);
  const int sy = y0 + r < 0 ? 0 : (y0 + r >= h ? h - 1 : y0 + r);
  const uint8_t* row = plane + (uint64_t)sy * stride;
  const int nw = (ncols + 3) >> 2;  // words stored: 6, 4 or 3
  if (a.aligned_src && x0 >= 0 && x0 + ncols <= w) {
    const int j0 = x0 & ~3, sh = 8 * (x0 & 3);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(row + j0);
    const int avail = (w - j0) >> 2;  // words from j0 to the row's end
    uint32_t wd[7];
#pragma unroll
    for (int k = 0; k < 7; k++) wd[k] = (k <= nw && k < avail) ? __ldg(src + k) : 0u;
#pragma unroll
    for (int k = 0; k < 6; k++)
      if (k < nw) dst[k] = __funnelshift_r(wd[k], wd[k + 1], sh);
    return;
  }
#pragma unroll 1
  for (int k = 0; k < nw; k++) {
    uint32_t v = 0;
    for (int c = 0; c < 4 && 4 * k + c < ncols; c++) {
      const int x = x0 + 4 * k + c;
      v |= (uint32_t)__ldg(row + (x < 0 ? 0 : (x >= w ? w - 1 : x))) << (8 * c);
    }
    dst[k] = v;
  }
}

// CTA `cta` of the `ncta` working on `a` (grid-stride over 8-MB groups).
template <int MODE>
__device__ __forceinline__ void predict_body(const PredArgs& a, uint32_t cta, uint32_t ncta) {
  __shared__ __align__(16) uint8_t slots[PR_MBS][SLOT_BYTES];
  __shared__ Job jobs[PR_MBS];
  __shared__ uint32_t tw[8][4][3];  // tap words: [fraction][output shift][window word]
  const int tid = threadIdx.x;

  // Tap words for dp4a: byte m of word q for output column j holds tap
  // 4q + m - j (0 outside 0..5). The identity fraction never uses them.
  if (tid < 96) {
    const int f = tid / 12, j = (tid / 3) & 3, q = tid % 3;
    uint32_t w = 0;
    if (f != 0)
      for (int m = 0; m < 4; m++) {
        const int k = 4 * q + m - j;
        if (k >= 0 && k < 6) w |= (uint32_t)(uint8_t)(int8_t)c_taps[a.filter_set][f][k] << (8 * m);
      }
    tw[f][j][q] = w;
  }

  for (uint32_t g = cta; (size_t)g * PR_MBS < a.n; g += ncta) {
    // ---- (1) per-MB vectors: 16 threads per MB, thread b = luma block b.
    {
      const int s = tid >> 4, b = tid & 15;
      const uint32_t item = g * PR_MBS + s;
      Job& J = jobs[s];
      int skip = item >= a.n, split = 0, col = 0, row = 0, ridx = 0;
      vp8a_mv mv = {0, 0};
      if (!skip) {
        if (MODE == PRED_FRAME) {
          const vp8a_mb_decision& d = a.dec[item];
          ridx = -1;
          for (int k = 0; k < a.n_refs; k++)
            if (d.ref_frame != VP8A_REF_INTRA && a.ref_ids[k] == d.ref_frame) ridx = k;
          skip = ridx < 0;
          split = d.mode == VP8A_MODE_SPLIT;
          mv = split ? d.split_mvs[b] : d.mv;
          col = (int)(item % (uint32_t)a.mb_cols);
          row = (int)(item / (uint32_t)a.mb_cols);
        } else {
          split = MODE == PRED_SPLIT;
          mv = a.mvs[split ? (size_t)item * 16 + b : item];
          col = (int)min(a.mb_xy[2 * item], 0x40000u);
          row = (int)min(a.mb_xy[2 * item + 1], 0x40000u);
        }
      }
      // Luma block vector.
      int er = dbl16(mv.row), ec = dbl16(mv.col);
      // Chroma: the SPLITMV four-block average of the i32-doubled vectors
      // (blocks b, b^1, b^4, b^5 share a chroma block), or the whole-MB
      // chroma_mv of the doubled vector. The sums run in every lane so the
      // shuffles stay converged.
      int sr = 2 * (int)mv.row, sc = 2 * (int)mv.col;
      sr += __shfl_xor_sync(0xffffffffu, sr, 1);
      sc += __shfl_xor_sync(0xffffffffu, sc, 1);
      sr += __shfl_xor_sync(0xffffffffu, sr, 4);
      sc += __shfl_xor_sync(0xffffffffu, sc, 4);
      int cr = (short)avg_sum(split ? sr : 4 * er);
      int cc = (short)avg_sum(split ? sc : 4 * ec);
      if (a.full_pixel) {
        er &= ~7;
        ec &= ~7;
        cr &= ~7;
        cc &= ~7;
      }
      J.lmv[b] = make_short2((short)er, (short)ec);
      const int cidx = ((b >> 1) & 1) + ((b >> 2) & 2);
      if ((b & 5) == 0) J.cmv[cidx] = make_short2((short)cr, (short)cc);
      if (b == 0) {
        J.skip = skip;
        J.split = split;
        // Vector offsets reach 4096 pixels in luma and in chroma, so an MB
        // origin more than 16448 luma pixels past the plane fetches only
        // edge pixels in both; clamping it there keeps every offset an int.
        J.x16 = min(col * 16, a.lw + 16448);
        J.y16 = min(row * 16, a.lh + 16448);
        if (!skip) {
          const PredPlanes& P = a.refs[ridx];
          J.y = P.y;
          J.u = P.u;
          J.v = P.v;
          J.ys = P.ys;
          J.uvs = P.uvs;
          if (MODE == PRED_FRAME) {
            J.oy = a.oy + (uint64_t)row * 16 * a.oys + (uint64_t)col * 16;
            J.ou = a.ou + (uint64_t)row * 8 * a.ouvs + (uint64_t)col * 8;
            J.ov = a.ov + (uint64_t)row * 8 * a.ouvs + (uint64_t)col * 8;
            J.oys = a.oys;
            J.ouvs = a.ouvs;
          } else {
            J.oy = a.out + (size_t)item * 384;
            J.ou = J.oy + 256;
            J.ov = J.oy + 320;
            J.oys = 16;
            J.ouvs = 8;
          }
        }
      }
    }
    __syncthreads();

    // ---- (2) edge-clamped source regions into shared memory, one region
    // row per thread and step over the 8 MBs' rows.
    {
      int start[PR_MBS + 1];
      start[0] = 0;
#pragma unroll
      for (int q = 0; q < PR_MBS; q++)
        start[q + 1] = start[q] + (jobs[q].skip ? 0 : (jobs[q].split ? SPLIT_ROWS : WHOLE_ROWS));
      const int total = start[PR_MBS];
#pragma unroll 1
      for (int i = tid; i < total; i += PR_THREADS) {
        int s = 0, first = 0;
#pragma unroll
        for (int q = 1; q < PR_MBS; q++)
          if (i >= start[q]) {
            s = q;
            first = start[q];
          }
        stage_row(jobs[s], slots[s], i - first, a);
      }
    }
    __syncthreads();

    // ---- (3) tasks: 48 per MB.
#pragma unroll 1
    for (int t = tid; t < PR_MBS * PR_TASKS; t += PR_THREADS) {
      const int s = t / PR_TASKS, k = t - PR_TASKS * s;
      const Job& J = jobs[s];
      if (J.skip) continue;
      const uint8_t* S = slots[s];
      const uint8_t* win;
      int ws, sb, sc, h;
      short2 m;
      uint8_t* dst;
      uint64_t ds;
      if (k < 32) {
        const int b = k >> 1;
        h = k & 1;
        sb = b >> 2;
        sc = b & 3;
        m = J.lmv[b];
        if (J.split) {
          win = S + b * HALO_BYTES + 2 * h * HALO_STRIDE;
          ws = HALO_STRIDE;
        } else {
          win = S + (4 * sb + 2 * h) * WY_STRIDE + 4 * sc;
          ws = WY_STRIDE;
        }
        dst = J.oy;
        ds = J.oys;
      } else {
        const int kk = k - 32, p = kk >> 3, cb = (kk >> 1) & 3;
        h = kk & 1;
        sb = cb >> 1;
        sc = cb & 1;
        m = J.cmv[cb];
        if (J.split) {
          win = S + (16 + 4 * p + cb) * HALO_BYTES + 2 * h * HALO_STRIDE;
          ws = HALO_STRIDE;
        } else {
          win = S + (p ? WV_OFF : WU_OFF) + (4 * sb + 2 * h) * WC_STRIDE + 4 * sc;
          ws = WC_STRIDE;
        }
        dst = p ? J.ov : J.ou;
        ds = J.ouvs;
      }
      uint32_t o0, o1;
      predict_pair(win, ws, m.y & 7, m.x & 7, tw, o0, o1);
      uint8_t* d0 = dst + (uint64_t)(4 * sb + 2 * h) * ds + 4 * sc;
      store_row(d0, o0, a.aligned_out);
      store_row(d0 + ds, o1, a.aligned_out);
    }
    __syncthreads();
  }
}

template <int MODE>
__global__ void __launch_bounds__(PR_THREADS) predict_kernel(PredArgs a) {
  predict_body<MODE>(a, blockIdx.x, gridDim.x);
}

// Frame prediction over a job table (one job per frame).
__global__ void __launch_bounds__(PR_THREADS)
    predict_frames_kernel(const PredArgs* __restrict__ jobs, const uint32_t* __restrict__ cta_start, int n_jobs) {
  __shared__ PredArgs sa;
  __shared__ uint32_t first[2];
  vp8a_dev::find_job(jobs, cta_start, n_jobs, &sa, first);
  predict_body<PRED_FRAME>(sa, blockIdx.x - first[0], first[1]);
}

int g_pred_blocks_per_sm[3] = {0, 0, 0};

template <int MODE>
vp8a_status launch(vp8a_ctx* ctx, const PredArgs& a) {
  if (a.n == 0) return VP8A_OK;
  if (!g_pred_blocks_per_sm[MODE]) {
    int b = 0;
    VP8A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, predict_kernel<MODE>, PR_THREADS, 0));
    g_pred_blocks_per_sm[MODE] = std::max(b, 1);
  }
  const size_t groups = (a.n + PR_MBS - 1) / PR_MBS;
  const unsigned grid = (unsigned)std::min<size_t>(groups, (size_t)ctx->sm_count * g_pred_blocks_per_sm[MODE]);
  predict_kernel<MODE><<<grid, PR_THREADS, 0, ctx->stream>>>(a);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

vp8a_status check_planes(const vp8a_planes* p, const char* what) {
  if (!p || !p->y || !p->u || !p->v) {
    vp8a::set_error(std::string(what) + ": null plane");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (p->mb_cols == 0 || p->mb_rows == 0 || p->mb_cols > 1024 || p->mb_rows > 1024) {
    vp8a::set_error(std::string(what) + ": MB grid must be 1..1024 x 1..1024");
    return VP8A_E_INVALID_DIMENSIONS;
  }
  if (p->y_stride < (uint64_t)p->mb_cols * 16 || p->uv_stride < (uint64_t)p->mb_cols * 8) {
    vp8a::set_error(std::string(what) + ": stride below the MB-padded width");
    return VP8A_E_INVALID_ARGUMENT;
  }
  return VP8A_OK;
}

size_t luma_bytes(const vp8a_planes* p) { return p->y_stride * ((size_t)p->mb_rows * 16 - 1) + (size_t)p->mb_cols * 16; }
size_t chroma_bytes(const vp8a_planes* p) { return p->uv_stride * ((size_t)p->mb_rows * 8 - 1) + (size_t)p->mb_cols * 8; }

// Stages one reference's planes (read-only) into a.refs[k].
vp8a_status stage_ref(vp8a::Stager& st, const vp8a_planes* p, PredPlanes* out) {
  vp8a_status s;
  const void* d;
  if ((s = st.in(p->y, luma_bytes(p), &d)) != VP8A_OK) return s;
  out->y = (const uint8_t*)d;
  if ((s = st.in(p->u, chroma_bytes(p), &d)) != VP8A_OK) return s;
  out->u = (const uint8_t*)d;
  if ((s = st.in(p->v, chroma_bytes(p), &d)) != VP8A_OK) return s;
  out->v = (const uint8_t*)d;
  out->ys = p->y_stride;
  out->uvs = p->uv_stride;
  return VP8A_OK;
}

int src_aligned(const PredPlanes& p) {
  return (((uintptr_t)p.y | (uintptr_t)p.u | (uintptr_t)p.v | p.ys | p.uvs) & 3) == 0;
}

void set_dims(PredArgs& a, const vp8a_planes* p) {
  a.lw = (int)p->mb_cols * 16;
  a.lh = (int)p->mb_rows * 16;
  a.cw = (int)p->mb_cols * 8;
  a.ch = (int)p->mb_rows * 8;
}

vp8a_status predict_batch(vp8a_ctx* ctx, const vp8a_planes* ref, const uint32_t* mb_xy, const vp8a_mv* mvs,
                          uint32_t n, uint32_t full_pixel, uint32_t filter_set, uint8_t* out, bool split) {
  if (!ctx) {
    vp8a::set_error("null context");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (filter_set > VP8A_FILTER_BILINEAR) {
    vp8a::set_error("filter_set must be VP8A_FILTER_SIXTAP or VP8A_FILTER_BILINEAR");
    return VP8A_E_INVALID_ARGUMENT;
  }
  vp8a_status s;
  if ((s = check_planes(ref, "reference")) != VP8A_OK) return s;
  if (n == 0) return VP8A_OK;
  if (!mb_xy || !mvs || !out) {
    vp8a::set_error("null batch argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  PredArgs a{};
  if ((s = stage_ref(st, ref, &a.refs[0])) != VP8A_OK) return s;
  a.ref_ids[0] = VP8A_REF_LAST;
  a.n_refs = 1;
  a.aligned_src = src_aligned(a.refs[0]);
  set_dims(a, ref);
  const void* d;
  if ((s = st.in(mb_xy, (size_t)n * 8, &d)) != VP8A_OK) return s;
  a.mb_xy = (const uint32_t*)d;
  if ((s = st.in(mvs, (size_t)n * (split ? 16 : 1) * sizeof(vp8a_mv), &d)) != VP8A_OK) return s;
  a.mvs = (const vp8a_mv*)d;
  void* o;
  if ((s = st.out(out, (size_t)n * 384, &o)) != VP8A_OK) return s;
  a.out = (uint8_t*)o;
  a.aligned_out = ((uintptr_t)o & 3) == 0;
  a.n = n;
  a.full_pixel = full_pixel != 0;
  a.filter_set = (int)filter_set;
  if ((s = split ? launch<PRED_SPLIT>(ctx, a) : launch<PRED_WHOLE>(ctx, a)) != VP8A_OK) return s;
  return st.finish();
}

}  // namespace

namespace vp8a {

vp8a_status predict_frame(vp8a_ctx* ctx, Stager& st, const vp8a_planes* refs, const uint8_t* ref_ids,
                          uint32_t n_refs, const vp8a_mb_decision* decisions, uint32_t full_pixel,
                          uint32_t filter_set, const vp8a_planes* out, FramePrediction* fp, bool defer) {
  if (!refs || !ref_ids || !decisions) {
    set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (n_refs == 0 || n_refs > (uint32_t)MAX_PRED_REFS) {
    set_error("n_refs must be 1..3");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (filter_set > VP8A_FILTER_BILINEAR) {
    set_error("filter_set must be VP8A_FILTER_SIXTAP or VP8A_FILTER_BILINEAR");
    return VP8A_E_INVALID_ARGUMENT;
  }
  vp8a_status s;
  if ((s = check_planes(out, "output")) != VP8A_OK) return s;
  for (uint32_t k = 0; k < n_refs; k++) {
    if ((s = check_planes(&refs[k], "reference")) != VP8A_OK) return s;
    if (refs[k].mb_cols != out->mb_cols || refs[k].mb_rows != out->mb_rows) {
      set_error("reference planes do not match the output MB grid");
      return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
    }
  }
  PredArgs a{};
  if ((s = st.read_to_host(ref_ids, n_refs, fp->ref_ids)) != VP8A_OK) return s;
  for (uint32_t k = 0; k < n_refs; k++) {
    if (fp->ref_ids[k] < VP8A_REF_LAST || fp->ref_ids[k] > VP8A_REF_ALTREF) {
      set_error("reference ids must be VP8A_REF_LAST, _GOLDEN or _ALTREF");
      return VP8A_E_INVALID_ARGUMENT;
    }
    if ((s = stage_ref(st, &refs[k], &a.refs[k])) != VP8A_OK) return s;
    a.ref_ids[k] = fp->ref_ids[k];
  }
  fp->n_refs = n_refs;
  a.n_refs = (int)n_refs;
  a.aligned_src = 1;
  for (uint32_t k = 0; k < n_refs; k++) a.aligned_src &= src_aligned(a.refs[k]);
  set_dims(a, out);
  a.mb_cols = (int)out->mb_cols;
  const uint32_t n = out->mb_cols * out->mb_rows;
  const void* d;
  if ((s = st.in(decisions, (size_t)n * sizeof(vp8a_mb_decision), &d)) != VP8A_OK) return s;
  a.dec = (const vp8a_mb_decision*)d;
  // In/out: MBs without an inter reference keep the caller's pixels.
  void* o;
  if ((s = st.inout(out->y, luma_bytes(out), &o)) != VP8A_OK) return s;
  a.oy = (uint8_t*)o;
  if ((s = st.inout(out->u, chroma_bytes(out), &o)) != VP8A_OK) return s;
  a.ou = (uint8_t*)o;
  if ((s = st.inout(out->v, chroma_bytes(out), &o)) != VP8A_OK) return s;
  a.ov = (uint8_t*)o;
  a.oys = out->y_stride;
  a.ouvs = out->uv_stride;
  a.aligned_out = (((uintptr_t)a.oy | (uintptr_t)a.ou | (uintptr_t)a.ov | a.oys | a.ouvs) & 3) == 0;
  a.n = n;
  a.full_pixel = full_pixel != 0;
  a.filter_set = (int)filter_set;
  static_assert(sizeof(PredArgs) <= sizeof(fp->args), "FramePrediction holds the launch arguments");
  memcpy(fp->args, &a, sizeof a);
  if (!defer && (s = launch<PRED_FRAME>(ctx, a)) != VP8A_OK) return s;
  fp->dec = a.dec;
  fp->planes = *out;
  fp->planes.y = a.oy;
  fp->planes.u = a.ou;
  fp->planes.v = a.ov;
  return VP8A_OK;
}

vp8a_status predict_frames(vp8a_ctx* ctx, Stager& st, const FramePrediction* fps, uint32_t n) {
  std::vector<PredArgs> table;
  std::vector<uint32_t> start{0};
  if (!g_pred_blocks_per_sm[PRED_FRAME]) {
    int b = 0;
    VP8A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, predict_kernel<PRED_FRAME>, PR_THREADS, 0));
    g_pred_blocks_per_sm[PRED_FRAME] = std::max(b, 1);
  }
  for (uint32_t j = 0; j < n; j++) {
    PredArgs a;
    memcpy(&a, fps[j].args, sizeof a);
    if (a.n == 0) continue;
    const size_t groups = (a.n + PR_MBS - 1) / PR_MBS;
    table.push_back(a);
    start.push_back(start.back() +
                    (uint32_t)std::min<size_t>(groups, (size_t)ctx->sm_count * g_pred_blocks_per_sm[PRED_FRAME]));
  }
  if (table.empty()) return VP8A_OK;
  const size_t o_start = sizeof(PredArgs) * table.size(), total = o_start + sizeof(uint32_t) * start.size();
  std::vector<uint8_t> blob(total);
  memcpy(blob.data(), table.data(), o_start);
  memcpy(blob.data() + o_start, start.data(), sizeof(uint32_t) * start.size());
  void* d;
  vp8a_status s;
  if ((s = st.upload(blob.data(), total, &d)) != VP8A_OK) return s;
  predict_frames_kernel<<<start.back(), PR_THREADS, 0, ctx->stream>>>(
      (const PredArgs*)d, (const uint32_t*)((const uint8_t*)d + o_start), (int)table.size());
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

}  // namespace vp8a

extern "C" {

vp8a_status vp8a_predict_inter_mb(vp8a_ctx* ctx, const vp8a_planes* ref, const uint32_t* mb_xy, const vp8a_mv* mvs,
                                  uint32_t n, uint32_t full_pixel, uint32_t filter_set, uint8_t* out) {
  return predict_batch(ctx, ref, mb_xy, mvs, n, full_pixel, filter_set, out, false);
}

vp8a_status vp8a_predict_split_mv(vp8a_ctx* ctx, const vp8a_planes* ref, const uint32_t* mb_xy,
                                  const vp8a_mv* split_mvs, uint32_t n, uint32_t full_pixel, uint32_t filter_set,
                                  uint8_t* out) {
  return predict_batch(ctx, ref, mb_xy, split_mvs, n, full_pixel, filter_set, out, true);
}

vp8a_status vp8a_predict_inter_frame(vp8a_ctx* ctx, const vp8a_planes* refs, const uint8_t* ref_ids, uint32_t n_refs,
                                     const vp8a_mb_decision* decisions, uint32_t full_pixel, uint32_t filter_set,
                                     vp8a_planes* out) {
  if (!ctx) {
    vp8a::set_error("null context");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  vp8a::FramePrediction fp;
  vp8a_status s = vp8a::predict_frame(ctx, st, refs, ref_ids, n_refs, decisions, full_pixel, filter_set, out, &fp);
  if (s != VP8A_OK) return s;
  return st.finish();
}

}  // extern "C"
