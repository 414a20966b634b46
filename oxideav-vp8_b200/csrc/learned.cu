// learned.cu — the learned motion proposal: a 4-layer 3x3 conv net (BF16
// weights and activations, FP32 accumulation) that scores a 32x32 grid of
// whole-pel vectors (2 px apart, -32 .. +30 px) for an MB from a coarse
// cost volume: at each grid vector, the half-resolution SAD of the MB
// against the reference and the reference's texture there. Its top four
// cells seed an exact local search (the plain search's SAD kernels), so
// the net only proposes; every returned vector and SAD is exact.
//
// Kernels (all hand-written; the GEMM-shaped ones on the tensor cores, the
// training layers with mma.sync m16n8k16 BF16 -> FP32, inference and the
// 32 -> 32 forward layers with tcgen05 and TMEM accumulators):
//   lp_windows_kernel       coarse cost volumes -> NHWC [n, 32, 32, 2] BF16
//   lp_net_kernel           the whole net and the top-k cells per map in one
//                           launch (inference), activations on chip
//   lp_seeded_search_kernel every whole-pel vector near the seed cells,
//                           first smallest SAD
//   lp_conv_fwd_smem_kernel implicit-GEMM conv (+ bias, ReLU), one CTA per
//                           image staged with its halo in shared memory
//   lp_conv_bwd_data_kernel dX = conv^T(dY, W), masked by the ReLU of X
//   lp_conv_fwd_tc_kernel   the 32 -> 32 forward layers on tcgen05 tensor
//                           cores (TMEM accumulators)
//   lp_conv_bwd_w_smem_kernel dW = sum over pixels of dY x shifted X (16
//                           staged chunks per CTA, one atomic per weight), db
//   lp_softmax_ce_kernel    softmax over the 1024 cells, cross-entropy,
//                           d(logits) = (p - onehot) / n
//   lp_adam_kernel          Adam on FP32 master weights, BF16 copies
// Layout: activations NHWC, 32x32 pixels per MB, channel count 2 or 32
// (the last layer 1); weights [cout][tap][cin], tap = (dy + 1) * 3 + dx + 1.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>

#include "vp8a_internal.cuh"

namespace {

constexpr int LP_S = 32;          // image side
constexpr int LP_P = LP_S * LP_S; // pixels per image

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ uint32_t pack_raw(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Element (pixel q of image img shifted by (dy, dx), channel c) of an NHWC
// BF16 tensor with C channels, 0 outside the image or past C.
__device__ __forceinline__ uint16_t act(const uint16_t* X, int C, int img, int y, int x, int c) {
  if (y < 0 || y >= LP_S || x < 0 || x >= LP_S || c >= C) return 0;
  return X[((size_t)img * LP_P + y * LP_S + x) * C + c];
}

// ---------------------------------------------------------------- windows

// Item i: the MB at (xy[2i], xy[2i+1]). Both pictures are averaged over
// 2x2 (rounded) and edge-clamped: the MB to 8x8, the reference around it
// (80x80 pixels, the MB at [32, 48)) to 40x40. Cell (i, j) is the vector
// (2 (i - 16), 2 (j - 16)) px: channel 0 = (32 - mean |MB - reference block
// at that vector|) / 32, channel 1 = (reference at the block's centre - 128)
// / 64.
__global__ void __launch_bounds__(256) lp_windows_kernel(const uint8_t* src, uint64_t ss, const uint8_t* ref,
                                                         uint64_t rs, int w, int h, const uint32_t* xy, int n,
                                                         uint16_t* out) {
  __shared__ uint32_t rw32[40 * 40 / 4];  // the reference window at half resolution, rows of 10 words
  __shared__ uint32_t mb32[16];           // the MB at half resolution, rows of 2 words
  uint8_t* rw = reinterpret_cast<uint8_t*>(rw32);
  uint8_t* mb = reinterpret_cast<uint8_t*>(mb32);
  const int i = blockIdx.x, t = threadIdx.x;
  if (i >= n) return;
  const int mx = (int)xy[2 * i] * 16, my = (int)xy[2 * i + 1] * 16;
  auto avg2 = [&](const uint8_t* p, uint64_t st, int y, int x) -> int {
    int s = 0;
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++) s += p[(size_t)min(max(y + a, 0), h - 1) * st + min(max(x + b, 0), w - 1)];
    return (s + 2) >> 2;
  };
  for (int q = t; q < 40 * 40; q += blockDim.x)
    rw[q] = (uint8_t)avg2(ref, rs, my - 32 + 2 * (q / 40), mx - 32 + 2 * (q % 40));
  if (t < 64) mb[t] = (uint8_t)avg2(src, ss, my + 2 * (t >> 3), mx + 2 * (t & 7));
  __syncthreads();
  // Thread t: cells (oy, 4 j .. 4 j + 3) with oy = t / 8, j = t % 8. Per
  // window row three words hold the 11 bytes the four 8-byte rows need; the
  // byte-shifted rows come from byte permutes and four-byte SADs.
  const int oy = t >> 3, ox0 = (t & 7) * 4;
  uint32_t sad[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const uint32_t* row = rw32 + (oy + r) * 10 + (ox0 >> 2);
    const uint32_t w0 = row[0], w1 = row[1], w2 = row[2];
    const uint32_t m0 = mb32[2 * r], m1 = mb32[2 * r + 1];
    sad[0] = __vsadu4(w0, m0) + __vsadu4(w1, m1) + sad[0];
    sad[1] = __vsadu4(__byte_perm(w0, w1, 0x4321), m0) + __vsadu4(__byte_perm(w1, w2, 0x4321), m1) + sad[1];
    sad[2] = __vsadu4(__byte_perm(w0, w1, 0x5432), m0) + __vsadu4(__byte_perm(w1, w2, 0x5432), m1) + sad[2];
    sad[3] = __vsadu4(__byte_perm(w0, w1, 0x6543), m0) + __vsadu4(__byte_perm(w1, w2, 0x6543), m1) + sad[3];
  }
  uint32_t o[4];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const float c0 = (32.0f - (float)sad[c] * (1.0f / 64.0f)) * (1.0f / 32.0f);
    const float c1 = ((float)rw[(oy + 4) * 40 + ox0 + c + 4] - 128.0f) * (1.0f / 64.0f);
    o[c] = pack_bf16(c0, c1);
  }
  *reinterpret_cast<uint4*>(out + ((size_t)i * LP_P + oy * 32 + ox0) * 2) = make_uint4(o[0], o[1], o[2], o[3]);
}

// ------------------------------------------------------- seeded search

// The exact search around the net's seeds: one CTA per MB, thread t takes
// candidate t = (seed s, row offset dr, column offset dc) in seed, row,
// column order. The source MB and each seed's (16 + 2 radius)-pixel square
// window of the reference (edge-clamped, as every whole-pel SAD reads it)
// sit in shared memory; the first smallest (SAD, order) wins.
constexpr int LP_SEED_MAXC = 128;  // k * (2 radius + 1)^2
constexpr int LP_SEED_MAXW = 16 + 2 * 4;  // window side for radius <= 4
constexpr int LP_SEED_PITCH = 28;         // window row pitch: 7 words, so a row's five words stay in it
__global__ void __launch_bounds__(LP_SEED_MAXC) lp_seeded_search_kernel(const uint8_t* ref, uint64_t rs, int rw,
                                                                        int rh, const uint8_t* src_mbs,
                                                                        const uint32_t* xy, const int32_t* seeds,
                                                                        int k, int radius, vp8a_search_result* out) {
  __shared__ uint32_t win32[4][LP_SEED_MAXW * LP_SEED_PITCH / 4];
  __shared__ uint32_t sm32[64];
  uint8_t* sm = reinterpret_cast<uint8_t*>(sm32);
  __shared__ uint32_t best_w[LP_SEED_MAXC / 32];
  const int i = blockIdx.x, t = threadIdx.x;
  const int mx = (int)xy[2 * i] * 16, my = (int)xy[2 * i + 1] * 16;
  const int side = 16 + 2 * radius, per = (2 * radius + 1) * (2 * radius + 1);
  for (int q = t; q < 256; q += blockDim.x) sm[q] = src_mbs[(size_t)i * 256 + q];
  for (int s = 0; s < k; s++) {
    const int c = seeds[(size_t)i * k + s];
    const int x0 = mx + (c % 32 - 16) * 2 - radius, y0 = my + (c / 32 - 16) * 2 - radius;
    uint8_t* win = reinterpret_cast<uint8_t*>(win32[s]);
    for (int q = t; q < side * side; q += blockDim.x) {
      const int y = min(max(y0 + q / side, 0), rh - 1), x = min(max(x0 + q % side, 0), rw - 1);
      win[(q / side) * LP_SEED_PITCH + q % side] = ref[(size_t)y * rs + x];
    }
  }
  __syncthreads();
  uint32_t key = 0xffffffffu;
  if (t < k * per) {
    const int s = t / per, o = t - s * per, dr = o / (2 * radius + 1), dc = o - dr * (2 * radius + 1);
    // Row r of the candidate: bytes dc .. dc + 15 of window row dr + r, cut
    // from five words by byte permutes, against the MB row's four words.
    const uint32_t* w = win32[s] + dr * (LP_SEED_PITCH / 4) + (dc >> 2);
    const uint32_t sel = 0x3210u + (uint32_t)(dc & 3) * 0x1111u;
    uint32_t sad = 0;
#pragma unroll 4
    for (int r = 0; r < 16; r++) {
      const uint32_t* wr = w + r * (LP_SEED_PITCH / 4);
      const uint32_t w0 = wr[0], w1 = wr[1], w2 = wr[2], w3 = wr[3], w4 = wr[4];
      sad += __vsadu4(__byte_perm(w0, w1, sel), sm32[4 * r]) + __vsadu4(__byte_perm(w1, w2, sel), sm32[4 * r + 1]) +
             __vsadu4(__byte_perm(w2, w3, sel), sm32[4 * r + 2]) + __vsadu4(__byte_perm(w3, w4, sel), sm32[4 * r + 3]);
    }
    key = (sad << 7) | (uint32_t)t;
  }
  key = __reduce_min_sync(0xffffffffu, key);
  if ((t & 31) == 0) best_w[t >> 5] = key;
  __syncthreads();
  if (t == 0) {
    uint32_t b = best_w[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) b = min(b, best_w[w]);
    const int o = (int)(b & 127u), s = o / per, r = o - s * per;
    const int c = seeds[(size_t)i * k + s];
    vp8a_search_result res;
    res.mv.row = (int16_t)((c / 32 - 16) * 8 + 4 * (r / (2 * radius + 1) - radius));
    res.mv.col = (int16_t)((c % 32 - 16) * 8 + 4 * (r % (2 * radius + 1) - radius));
    res.sad = b >> 7;
    out[i] = res;
  }
}

// ------------------------------------------------------------ conv fwd

// Implicit GEMM: A[p][k] = X[p + off(tap)][ci], k = tap * CP + ci (CP = CIN
// rounded up to 16); B[k][n] = W[n][tap][ci].
// Forward pass with the image staged: one CTA (8 warps) per image. The
// 32x32 input gets a zero halo (34x34) in shared memory, one pixel every PS
// halves (channels padded to CP, then 8 spare: a 16-byte-aligned row whose
// 32-bit words fall on distinct banks for the 8 pixels x 4 channel pairs a
// fragment reads); the weights sit beside it ([n][tap][ci], n stride
// 9 CIN + 8). Warp w takes the 16-pixel tiles w, w + 8, ... of the image.
template <int CIN, int NT>
__global__ void __launch_bounds__(256) lp_conv_fwd_smem_kernel(const uint16_t* X, const uint16_t* W, const float* bias,
                                                               int cout, int relu, uint16_t* Y, float* Yf) {
  constexpr int CP = (CIN + 15) / 16 * 16, PS = CP + 8, WS = 9 * CIN + 8, COUTP = NT * 8;
  extern __shared__ __align__(16) uint16_t sm[];
  uint16_t* img_s = sm;                 // 34 * 34 * PS
  uint16_t* w_s = sm + 34 * 34 * PS;    // COUTP * WS
  const int img = blockIdx.x, tid = threadIdx.x;
  // Zero the halo and the channel padding, then copy the image.
  for (int q = tid; q < 34 * 34 * PS / 2; q += blockDim.x) reinterpret_cast<uint32_t*>(img_s)[q] = 0u;
  for (int q = tid; q < COUTP * WS / 2; q += blockDim.x) reinterpret_cast<uint32_t*>(w_s)[q] = 0u;
  __syncthreads();
  const uint16_t* Xi = X + (size_t)img * LP_P * CIN;
  if (CIN % 2 == 0) {
    for (int q = tid; q < LP_P * CIN / 2; q += blockDim.x) {
      const int p = q / (CIN / 2), c = (q % (CIN / 2)) * 2;
      const int sy = (p >> 5) + 1, sx = (p & 31) + 1;
      *reinterpret_cast<uint32_t*>(img_s + (sy * 34 + sx) * PS + c) = reinterpret_cast<const uint32_t*>(Xi)[q];
    }
  }
  for (int q = tid; q < cout * 9 * CIN; q += blockDim.x) w_s[(q / (9 * CIN)) * WS + q % (9 * CIN)] = W[q];
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  // Warp w takes tiles w, w + 8, ..., four at a time, so each weight
  // fragment loaded from shared memory feeds four MMAs.
  constexpr int TG = 4;
  for (int t0 = warp; t0 < LP_P / 16; t0 += 8 * TG) {
    float d[TG][NT][4];
#pragma unroll
    for (int u = 0; u < TG; u++)
#pragma unroll
      for (int j = 0; j < NT; j++) d[u][j][0] = d[u][j][1] = d[u][j][2] = d[u][j][3] = 0.f;
#pragma unroll
    for (int tap = 0; tap < 9; tap++) {
      const int dy = tap / 3 - 1, dx = tap % 3 - 1;
#pragma unroll
      for (int c0 = 0; c0 < CP; c0 += 16) {
        uint32_t a[TG][4];
#pragma unroll
        for (int u = 0; u < TG; u++) {
          const int tile = t0 + 8 * u, y = tile >> 1, xb = (tile & 1) * 16;
          const uint16_t* r0 = img_s + ((y + dy + 1) * 34 + (xb + g + dx + 1)) * PS;
          const uint16_t* r1 = r0 + 8 * PS;
          a[u][0] = *reinterpret_cast<const uint32_t*>(r0 + c0 + 2 * t);
          a[u][1] = *reinterpret_cast<const uint32_t*>(r1 + c0 + 2 * t);
          a[u][2] = *reinterpret_cast<const uint32_t*>(r0 + c0 + 2 * t + 8);
          a[u][3] = *reinterpret_cast<const uint32_t*>(r1 + c0 + 2 * t + 8);
        }
#pragma unroll
        for (int j = 0; j < NT; j++) {
          const uint16_t* wr = w_s + (j * 8 + g) * WS + tap * CIN + c0 + 2 * t;
          uint32_t b[2];
          if (CIN >= 16) {
            b[0] = *reinterpret_cast<const uint32_t*>(wr);
            b[1] = *reinterpret_cast<const uint32_t*>(wr + 8);
          } else {  // CIN = 2: channels past CIN are zero
            b[0] = (c0 + 2 * t < CIN) ? *reinterpret_cast<const uint32_t*>(wr) : 0u;
            b[1] = 0u;
          }
#pragma unroll
          for (int u = 0; u < TG; u++) mma_bf16(d[u][j], a[u], b);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < TG; u++) {
      const int tile = t0 + 8 * u, y = tile >> 1, xb = (tile & 1) * 16;
#pragma unroll
      for (int j = 0; j < NT; j++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int p = y * LP_S + xb + g + 8 * h, n = j * 8 + 2 * t;
          const size_t o = ((size_t)img * LP_P + p) * cout + n;
          float v0 = d[u][j][2 * h] + (n < cout ? bias[n] : 0.f);
          float v1 = d[u][j][2 * h + 1] + (n + 1 < cout ? bias[n + 1] : 0.f);
          if (relu) {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
          }
          if (Yf) {
            if (n < cout) Yf[o] = v0;
            if (n + 1 < cout) Yf[o + 1] = v1;
          } else if (n + 1 < cout) {
            *reinterpret_cast<uint32_t*>(Y + o) = pack_bf16(v0, v1);
          } else if (n < cout) {
            Y[o] = __bfloat16_as_ushort(__float2bfloat16_rn(v0));
          }
        }
    }
  }
}

// --------------------------------------------------------- conv bwd data

// dX[p][ci] = sum over taps and co of dY[p - off(tap)][co] W[co][tap][ci],
// times (Xa[p][ci] > 0) when `mask` (the ReLU of the layer that produced X).
template <int COUT, int NT>
__global__ void __launch_bounds__(128) lp_conv_bwd_data_kernel(const uint16_t* dY, const uint16_t* W, int cin,
                                                               int n_img, const uint16_t* Xa, uint16_t* dX) {
  constexpr int KP = (COUT + 15) / 16 * 16;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int tile = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (tile >= n_img * (LP_P / 16)) return;
  const int img = tile / (LP_P / 16), rem = tile % (LP_P / 16), y = rem >> 1, xb = (rem & 1) * 16;
  float d[NT][4];
#pragma unroll
  for (int j = 0; j < NT; j++) d[j][0] = d[j][1] = d[j][2] = d[j][3] = 0.f;
  for (int tap = 0; tap < 9; tap++) {
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
#pragma unroll
    for (int c0 = 0; c0 < KP; c0 += 16) {
      uint32_t a[4];
      const int ca = c0 + 2 * t, cb = c0 + 2 * t + 8;
      // dY at p - off: the output pixel whose tap `tap` reads p.
      a[0] = pack_raw(act(dY, COUT, img, y - dy, xb + g - dx, ca), act(dY, COUT, img, y - dy, xb + g - dx, ca + 1));
      a[1] = pack_raw(act(dY, COUT, img, y - dy, xb + g + 8 - dx, ca),
                      act(dY, COUT, img, y - dy, xb + g + 8 - dx, ca + 1));
      a[2] = pack_raw(act(dY, COUT, img, y - dy, xb + g - dx, cb), act(dY, COUT, img, y - dy, xb + g - dx, cb + 1));
      a[3] = pack_raw(act(dY, COUT, img, y - dy, xb + g + 8 - dx, cb),
                      act(dY, COUT, img, y - dy, xb + g + 8 - dx, cb + 1));
#pragma unroll
      for (int j = 0; j < NT; j++) {
        const int n = j * 8 + g;  // ci
        auto wv = [&](int co) -> uint16_t {
          return (n < cin && co < COUT) ? W[((size_t)co * 9 + tap) * cin + n] : (uint16_t)0;
        };
        const uint32_t b[2] = {pack_raw(wv(ca), wv(ca + 1)), pack_raw(wv(cb), wv(cb + 1))};
        mma_bf16(d[j], a, b);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NT; j++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int p = y * LP_S + xb + g + 8 * h;
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int n = j * 8 + 2 * t + e;
        if (n >= cin) continue;
        const size_t o = ((size_t)img * LP_P + p) * cin + n;
        float v = d[j][2 * h + e];
        if (Xa && !(__bfloat162float(__ushort_as_bfloat16(Xa[o])) > 0.f)) v = 0.f;
        dX[o] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
      }
    }
}

// ------------------------------------------------------- conv bwd weights

// dW[co][tap][ci] += sum over a chunk of pixels of dY[p][co] X[p + off][ci]:
// M = co (16-row tiles), N = tap * CIN + ci (8-column tiles), K = pixels.
constexpr int LP_WCHUNK = 512;  // pixels per staged chunk (half an image)


// ------------------------------------------------------------- loss

// One block per item: softmax over its 1024 logits, the cross-entropy of
// the label cell (added to *loss), and d(logits) = (softmax - onehot) / n
// as BF16. Labels < 0 contribute nothing (zero gradient).
__global__ void __launch_bounds__(256) lp_softmax_ce_kernel(const float* logits, const int32_t* labels, int n,
                                                            uint16_t* dlogits, float* loss, float* top_prob) {
  const int i = blockIdx.x, t = threadIdx.x;
  __shared__ float red[8];
  const float* z = logits + (size_t)i * LP_P;
  float m = -INFINITY;
  for (int q = t; q < LP_P; q += 256) m = fmaxf(m, z[q]);
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((t & 31) == 0) red[t >> 5] = m;
  __syncthreads();
  m = red[0];
  for (int k = 1; k < 8; k++) m = fmaxf(m, red[k]);
  __syncthreads();
  float s = 0.f;
  for (int q = t; q < LP_P; q += 256) s += __expf(z[q] - m);
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((t & 31) == 0) red[t >> 5] = s;
  __syncthreads();
  s = 0.f;
  for (int k = 0; k < 8; k++) s += red[k];
  const int lab = labels ? labels[i] : -1;
  for (int q = t; q < LP_P; q += 256) {
    const float p = __expf(z[q] - m) / s;
    if (dlogits) {
      const float gr = lab < 0 ? 0.f : (p - (q == lab ? 1.f : 0.f)) / (float)n;
      dlogits[(size_t)i * LP_P + q] = __bfloat16_as_ushort(__float2bfloat16_rn(gr));
    }
    if (top_prob && q == lab) top_prob[i] = p;
  }
  if (t == 0 && loss && lab >= 0) atomicAdd(loss, -(z[lab] - m - __logf(s)));
}

// ------------------------------------------------------------- Adam

__global__ void lp_adam_kernel(float* w, const float* grad, float* m, float* v, int n, float lr, float b1, float b2,
                               float eps, float c1, float c2, uint16_t* w_bf16) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gr = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * gr, vi = b2 * v[i] + (1.f - b2) * gr * gr;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  w_bf16[i] = __bfloat16_as_ushort(__float2bfloat16_rn(wi));
}

// ------------------------------------------------- loop-filter window

// Channel sums of n images' activations ([n][32][32][C] BF16) into
// out[C] (FP32, accumulated): one CTA per image.
__global__ void __launch_bounds__(256) lp_pool_kernel(const uint16_t* X, int C, float* out) {
  __shared__ float part[64];
  const int img = blockIdx.x, t = threadIdx.x;
  if (t < 64) part[t] = 0.f;
  __syncthreads();
  const uint16_t* Xi = X + (size_t)img * LP_P * C;
  // Thread t sums channel t % C over pixels t / C, t / C + 256 / C, ...
  const int c = t % C, step = 256 / C;
  float s = 0.f;
  if (t < step * C)
    for (int p = t / C; p < LP_P; p += step) s += __bfloat162float(__ushort_as_bfloat16(Xi[(size_t)p * C + c]));
  atomicAdd(&part[c], s);
  __syncthreads();
  if (t < C) atomicAdd(&out[t], part[t]);
}

// The head: f = sums / count (C features), z = W f + b (L levels), softmax;
// with a label: loss += CE, dW += (p - onehot) f^T, db += p - onehot. One
// CTA of L threads.
__global__ void lp_lf_head_kernel(const float* sums, float count, int C, const float* W, const float* b, int L,
                                  int label, float* logits, float* dW, float* db, float* loss) {
  __shared__ float f[64], z[128];
  const int t = threadIdx.x;
  if (t < C) f[t] = sums[t] / count;
  __syncthreads();
  float zi = 0.f;
  if (t < L) {
    zi = b[t];
    for (int c = 0; c < C; c++) zi += W[t * C + c] * f[c];
    z[t] = zi;
    if (logits) logits[t] = zi;
  }
  __syncthreads();
  if (label < 0 || t >= L) return;
  float m = -INFINITY;
  for (int k = 0; k < L; k++) m = fmaxf(m, z[k]);
  float s = 0.f;
  for (int k = 0; k < L; k++) s += __expf(z[k] - m);
  const float p = __expf(zi - m) / s, gz = p - (t == label ? 1.f : 0.f);
  for (int c = 0; c < C; c++) dW[t * C + c] += gz * f[c];
  db[t] += gz;
  if (t == label && loss) *loss += -(zi - m - __logf(s));
}

// ------------------------------------------- tcgen05 forward, 32 -> 32
// The 32 -> 32 layers on the 5th-generation tensor cores: one CTA per
// image, the 3x3 convolution as an implicit GEMM D[pixel][n] = sum over
// (tap, ci) of A[pixel + tap offset][ci] * W[n][tap][ci]. The image sits in
// shared memory with a zero halo on a 34-pixel row pitch, channel-group
// major (group g of 8 channels: 16 bytes per halo pixel). Four TMA tile
// loads bring it in: the activations as a 4-D tensor (channel, x, y,
// image), a box of 8 channels x 34 x 34 pixels x 1 image per channel
// group, started at (8 g, -1, -1, image), so the box lands in exactly that
// layout and the halo ring is the loads' out-of-bounds zero fill. So that 8
// consecutive "virtual" output pixels v = y * 34 + x form one 8 x 16-byte
// core matrix of the K-major, unswizzled canonical layout and a tap
// (dy, dx) is only a base-address shift of (dy + 1) * 34 + dx + 1 pixels.
// The virtual grid computes 2 discarded columns per row (x = 32, 33) and
// is covered by 9 M = 128 tiles; each tile takes 18 MMAs of K = 16 (9 taps
// x 2 channel halves) into a 32-column FP32 accumulator in tensor memory.
// The weights sit as [k-group of 8][n][8] (k = tap * 32 + ci). One thread
// issues the MMAs of up to four tiles, one commit signals an mbarrier, and
// the 8 warps read the accumulators back (warp w: lanes 32 (w % 4) .. +31,
// columns 16 (w / 4) .. +15 of each tile), add the bias, apply the ReLU and
// store BF16.
namespace lptc {
constexpr int NV = 1224;                    // halo pixels per channel group (>= 1151 + 70 + 1)
constexpr int REGION = NV * 16;             // bytes per channel group
constexpr int IMG_BYTES = 4 * REGION;
constexpr int W_BYTES = 36 * 32 * 16;       // 36 k-groups x 32 n x 16 bytes
constexpr int SMEM = IMG_BYTES + W_BYTES + 32;
constexpr uint32_t BOX_BYTES = 8 * 34 * 34 * 2;  // one channel group's TMA box
static_assert(REGION % 128 == 0, "TMA destinations are 128-byte aligned");
constexpr int TILES = 9;                    // ceil(32 * 34 / 128)
constexpr uint32_t TMEM_COLS = 128;         // four 32-column accumulators
// Instruction descriptor (kind::f16): D FP32, A and B BF16, both K-major,
// N = 32, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
constexpr int WAIT_LIMIT = 1 << 22;

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  // Unswizzled K-major shared-memory matrix descriptor: start address,
  // leading (K) and stride (M/N) byte offsets in 16-byte units, version 1.
  return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
}  // namespace lptc

// Bounded wait for phase `phase` of the mbarrier at shared address `bar`;
// true when it completed.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, int limit) {
  uint32_t done = 0;
  for (int it = 0; it < limit && !done; it++) {
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
  }
  return done != 0;
}

__global__ void __launch_bounds__(256, 2) lp_conv_fwd_tc_kernel(const __grid_constant__ CUtensorMap tmx,
                                                                 const uint16_t* W, const float* bias, int relu,
                                                                 uint16_t* Y, uint32_t* status) {
  using namespace lptc;
  extern __shared__ __align__(128) uint8_t smt[];
  uint8_t* img_s = smt;
  uint8_t* w_s = smt + IMG_BYTES;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smt + IMG_BYTES + W_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smt + IMG_BYTES + W_BYTES + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t im = blockIdx.x;
  const uint32_t img_a = (uint32_t)__cvta_generic_to_shared(img_s);
  const uint32_t w_a = (uint32_t)__cvta_generic_to_shared(w_s);
  const uint32_t bar_a = (uint32_t)__cvta_generic_to_shared(mbar);
  const uint32_t bar_t = bar_a + 8;  // the image loads' mbarrier

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_a), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_t), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;");
    // The image: four TMA tile loads (one per channel group, the halo ring
    // from their out-of-bounds fill) completing on bar_t.
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_t), "r"(4 * BOX_BYTES)
                 : "memory");
    const uint64_t tm = reinterpret_cast<uint64_t>(&tmx);
    for (int g = 0; g < 4; g++)
      asm volatile(
          "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
          "[%6];" ::"r"(img_a + (uint32_t)(g * REGION)),
          "l"(tm), "r"(8 * g), "r"(-1), "r"(-1), "r"((int)im), "r"(bar_t)
          : "memory");
  }
  // The weights by 16-byte asynchronous copies, and zeros into each
  // channel group's tail past the 34 x 34 box, which no load touches.
  for (int q = tid; q < 32 * 36; q += 256) {
    const int n = q / 36, kg = q % 36;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(w_a + (uint32_t)((kg * 32 + n) * 16)),
                 "l"(W + n * 288 + kg * 8)
                 : "memory");
  }
  constexpr int TAIL = NV - 34 * 34;
  for (int q = tid; q < 4 * TAIL; q += 256)
    reinterpret_cast<uint4*>(img_s + (q / TAIL) * REGION)[34 * 34 + q % TAIL] = make_uint4(0, 0, 0, 0);
  asm volatile("cp.async.wait_all;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();  // the mbarrier inits are visible from here on
  // Bounded wait for the image; a load that never lands is reported, and
  // the CTA waits once more (bounded) for it before leaving.
  bool failed = __syncthreads_or(!mbar_wait(bar_t, 0, WAIT_LIMIT));
  if (failed) {
    if (tid == 0) atomicExch(status, 1u);  // DEV_TIMEOUT
    mbar_wait(bar_t, 0, WAIT_LIMIT);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  uint32_t phase = 0;
  for (int t0 = 0; t0 < TILES && !failed; t0 += 4) {
    const int nt = TILES - t0 < 4 ? TILES - t0 : 4;
    if (tid == 0) {
      for (int u = 0; u < nt; u++) {
        const int v0 = (t0 + u) * 128;
        const uint32_t d = tmem + (uint32_t)(u * 32);
        for (int ks = 0; ks < 18; ks++) {
          const int tap = ks >> 1, hh = ks & 1;
          const int off = (tap / 3) * 34 + tap % 3;
          const uint64_t ad = smem_desc(img_a + (uint32_t)(2 * hh * REGION + (v0 + off) * 16), REGION, 128);
          const uint64_t bd = smem_desc(w_a + (uint32_t)((tap * 4 + 2 * hh) * 32 * 16), 512, 128);
          const uint32_t acc = ks > 0 ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
              "l"(ad), "l"(bd), "r"(IDESC), "r"(acc));
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_a)
                   : "memory");
    }
    // Bounded wait for the commit; a timeout is reported, not waited out.
    const bool done = mbar_wait(bar_a, phase, WAIT_LIMIT);
    phase ^= 1u;
    failed = __syncthreads_or(!done);
    if (failed) {
      if (tid == 0) atomicExch(status, 1u);  // DEV_TIMEOUT
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int lq = warp & 3, half = warp >> 2;
    for (int u = 0; u < nt; u++) {
      uint32_t r[16];
      const uint32_t ta = tmem + ((uint32_t)(32 * lq) << 16) + (uint32_t)(u * 32 + half * 16);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(ta));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const int v = (t0 + u) * 128 + 32 * lq + lane, y = v / 34, x = v % 34;
      if (y < 32 && x < 32) {
        uint32_t o[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const int n = half * 16 + 2 * j;
          float a = __uint_as_float(r[2 * j]) + __ldg(bias + n);
          float b = __uint_as_float(r[2 * j + 1]) + __ldg(bias + n + 1);
          if (relu) {
            a = fmaxf(a, 0.f);
            b = fmaxf(b, 0.f);
          }
          o[j] = pack_bf16(a, b);
        }
        uint4* dst = reinterpret_cast<uint4*>(Y + (im * LP_P + y * 32 + x) * 32 + half * 16);
        dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
        dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// ------------------------------------------ fused net inference (tcgen05)
// The whole proposal net, one image at a time per persistent CTA (one per
// SM, the weights staged once), warp-specialised: the MMA warps (8 on)
// issue the tcgen05.mma of the tiles in turn (lane 0 of each) into a ring
// of 16 TMEM accumulators of 32 columns; warps 0-7 read each one back as soon
// as its MMAs commit, add the bias, apply the ReLU, store BF16 into the
// next layer's activation buffer and mark the (layer, tile) written. A tile
// u of the next layer reads the halo rows of tiles u - 1 .. u + 1, so its
// MMAs start once those three are written, while the epilogue of the later
// tiles runs. Two activation buffers alternate: B holds the input and layer
// 2's output, A layers 1 and 3. Layouts are the 32 -> 32 kernel's: a
// 34-pixel halo pitch, channel-group major (8 channels = 16 bytes per
// pixel), each 3x3 tap a descriptor offset, 9 M = 128 tiles of virtual
// pixels.
//
// One thread issuing tcgen05.mma (M = 128, K = 16) sustains one per ~63
// cycles whatever N up to 128, and between a tile's commit and its next
// tile it waits on the queue for several hundred more; the operands stream
// from shared memory at ~128 B per cycle (4 KB of A and 1 KB of B at N =
// 32: ~40 cycles an MMA). Several issuing warps keep the tensor pipe fed.
// The shapes follow from that:
//  - Layer 1 (2 -> 32): each pixel of B's first group holds the input pairs
//    of (x - 1, x, x + 1) and two zeros, so a kernel row is one K = 8 core
//    matrix; rows dy = -1 and 0 share one K = 16 MMA (leading byte offset
//    34 pixels), dy = +1 shares one with a zero-weight half: 2 MMAs a tile.
//  - Layers 2 and 3 (32 -> 32): 18 MMAs a tile (9 taps x 2 K halves), the
//    taps as row offsets of the A descriptor, so the epilogue only adds the
//    bias (putting taps into N instead makes the epilogue shift rows across
//    lanes, which costs more than the MMAs it saves).
//  - Layer 4 (32 -> 1): a 1 x 1 contraction with the 9 taps as N (= 16),
//    z[h][t] = act[h] . w4[t], 2 MMAs a tile, stored into B's channel
//    groups 1-3 (free once layer 3's MMAs are done; their halo rings and
//    tails are zeroed again after); after the last tile the epilogue forms
//    logit[o] = b4 + sum_t z[o + off_t][t] in one pass.
// The next image's 4 KB input arrives by one bulk copy while this image
// runs and is repacked into B's first group at layer 4's first tile. The
// one epilogue group consumes the tiles in order, waiting on each commit,
// so whenever it writes a buffer every MMA issued before that reads it has
// completed, whichever warp issued it. The top k cells of the logits
// (first index on ties) are written per image, and the logits themselves
// when asked.
//
// Every slot's tiles come from one issuer (16 is a multiple of the issuer
// count) and go to the one
// epilogue group in order, and each (layer, tile) barrier completes once
// an image, so no parity wait can run a phase ahead of its barrier. Every
// wait is bounded; a wait that runs out sets the context's status word,
// the other warps leave at their next wait, and the CTA drains its MMAs
// and copy before freeing TMEM.
namespace lpnet {
constexpr int REGION = lptc::REGION;           // one channel group's halo plane (1224 pixels x 16 B)
constexpr int BUF = 4 * REGION;                // 32 channels
constexpr int OFF_A = 0;
constexpr int OFF_B = OFF_A + BUF;
constexpr int OFF_W1 = OFF_B + BUF;            // 4 k-groups x 32 n x 16 B: dy = -1, 0, +1, zeros
constexpr int OFF_W2 = OFF_W1 + 4 * 32 * 16;   // 36 k-groups (tap, channel group) x 32 n x 16 B
constexpr int OFF_W3 = OFF_W2 + 36 * 32 * 16;
constexpr int OFF_W4 = OFF_W3 + 36 * 32 * 16;  // 4 k-groups x 16 n (taps 0-8, zeros) x 16 B
constexpr int OFF_STAGE = OFF_W4 + 4 * 16 * 16;  // the next image's input, 32 x 32 x 2 BF16
constexpr int OFF_Z = OFF_B + REGION;          // layer 4's z, [9 taps][1152 rows] FP32, in B's groups 1-3
constexpr int OFF_LOG = OFF_STAGE + 4096;      // 1024 FP32 logits
constexpr int OFF_RED = OFF_LOG + 1024 * 4;    // 2 x 8 u64 per-warp maxima (by round parity)
constexpr int OFF_BAR = OFF_RED + 2 * 8 * 8;
constexpr int TILES = 9;                       // ceil(32 * 34 / 128)
constexpr int NSLOT = 16;                      // TMEM accumulators of 32 columns
constexpr int ISSUERS = 4;
constexpr int BAR_FULL = 0;                    // [16] MMAs of a slot committed
constexpr int BAR_EMPTY = BAR_FULL + NSLOT;    // [16] a slot read back (8 warp arrivals)
constexpr int BAR_WRITTEN = BAR_EMPTY + NSLOT; // [3][9] layer l's tile u stored (8 warp arrivals)
constexpr int BAR_INPUT = BAR_WRITTEN + 3 * TILES;  // the image's input repacked (8 warp arrivals)
constexpr int BAR_STAGE = BAR_INPUT + 1;       // the bulk copy landed
constexpr int BAR_FIN = BAR_STAGE + 1;         // [4] an issuer's MMAs all completed
constexpr int NBAR = BAR_FIN + ISSUERS;
constexpr int OFF_TMEM = OFF_BAR + NBAR * 8;
constexpr int OFF_ABORT = OFF_TMEM + 4;
constexpr int SMEM = OFF_ABORT + 12;
constexpr int EPI = 256;                       // 8 epilogue warps
constexpr int THREADS = EPI + 32 * ISSUERS;
constexpr uint32_t TMEM_COLS = 512;
constexpr int LIMIT = 1 << 22;
constexpr uint32_t IDESC32 = lptc::IDESC;
constexpr uint32_t IDESC16 = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
static_assert(SMEM <= 227 * 1024, "fits one CTA per SM");
static_assert(OFF_STAGE % 128 == 0 && OFF_BAR % 8 == 0, "copy and barrier alignment");
static_assert(NSLOT * 32 <= (int)TMEM_COLS && NSLOT % ISSUERS == 0, "TMEM ring; a slot's tiles from one issuer");
static_assert((TILES - 1) * 128 + 127 + 70 < REGION / 16, "tile reads stay in a channel group");
static_assert(9 * TILES * 128 * 4 <= 3 * REGION, "z fits B's groups 1-3");

// A float's order as an unsigned key (finite values).
__device__ __forceinline__ uint32_t fkey(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ bool try_wait(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for the phase of parity `parity`; gives up early once another
// warp has set the abort word.
__device__ __forceinline__ bool wait(uint32_t bar, uint32_t parity, const volatile uint32_t* abort) {
  for (int it = 0; it < LIMIT; it++) {
    if (try_wait(bar, parity)) return true;
    if ((it & 255) == 255 && *abort) return false;
  }
  return false;
}

__device__ __forceinline__ void arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Named barrier 1 over the 256 epilogue threads; the OR of `p` over them.
__device__ __forceinline__ bool epi_or(bool p) {
  uint32_t r;
  __syncwarp();
  asm volatile(
      "{\n\t.reg .pred q, r;\n\t"
      "setp.ne.b32 q, %1, 0;\n\t"
      "bar.red.or.pred r, 1, 256, q;\n\t"
      "selp.b32 %0, 1, 0, r;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)p)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void epi_sync() {
  __syncwarp();
  asm volatile("bar.sync 1, 256;" ::: "memory");
}

// 16 consecutive 32-bit TMEM columns of this warp's 32 lanes.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}

// The 4 KB input of one image into `stage` by one bulk copy completing on `bar`.
__device__ __forceinline__ void fetch_input(uint32_t stage, const uint16_t* src, uint32_t bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(4096) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 4096, [%2];" ::"r"(stage),
      "l"(src), "r"(bar)
      : "memory");
}
}  // namespace lpnet

__global__ void __launch_bounds__(lpnet::THREADS, 1) lp_net_kernel(const uint16_t* X, int n, const uint16_t* W1,
                                                                 const float* b1, const uint16_t* W2, const float* b2,
                                                                 const uint16_t* W3, const float* b3,
                                                                 const uint16_t* W4, const float* b4, int k,
                                                                 int32_t* cells, float* logits, uint32_t* status) {
  using namespace lpnet;
  extern __shared__ __align__(128) uint8_t sm_[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t base = (uint32_t)__cvta_generic_to_shared(sm_);
  const uint32_t a_a = base + OFF_A, b_a = base + OFF_B;
  const uint32_t w1_a = base + OFF_W1, w2_a = base + OFF_W2, w3_a = base + OFF_W3, w4_a = base + OFF_W4;
  const uint32_t stage_a = base + OFF_STAGE;
  auto bar = [&](int i) { return base + (uint32_t)(OFF_BAR + 8 * i); };
  volatile uint32_t* abort_w = reinterpret_cast<volatile uint32_t*>(sm_ + OFF_ABORT);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm_ + OFF_TMEM);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + OFF_TMEM),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < NBAR; i++) {
      const bool one = (i >= BAR_FULL && i < BAR_FULL + NSLOT) || i == BAR_STAGE || i >= BAR_FIN;
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar(i)), "r"(one ? 1 : 8));
    }
    *abort_w = 0;
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  // Zero both activation buffers once (halo rings and tails stay zero: only
  // interior pixels are ever written), and stage the weights as
  // [k-group][n][8] K-major matrices.
  for (int q = tid; q < 2 * BUF / 16; q += THREADS) reinterpret_cast<uint4*>(sm_ + OFF_A)[q] = make_uint4(0, 0, 0, 0);
  uint16_t* w1s = reinterpret_cast<uint16_t*>(sm_ + OFF_W1);
  for (int q = tid; q < 4 * 32 * 8; q += THREADS) {
    // k-group kg = dy + 1 holds the row's taps dx = -1, 0, +1 for both input
    // channels (e = 2 (dx + 1) + c); k-group 3 and e = 6, 7 are zero.
    const int e = q & 7, nn = (q >> 3) & 31, kg = q >> 8;
    w1s[q] = (kg < 3 && e < 6) ? W1[nn * 18 + (kg * 3 + (e >> 1)) * 2 + (e & 1)] : (uint16_t)0;
  }
  uint16_t* w2s = reinterpret_cast<uint16_t*>(sm_ + OFF_W2);
  uint16_t* w3s = reinterpret_cast<uint16_t*>(sm_ + OFF_W3);
  for (int q = tid; q < 36 * 32 * 8; q += THREADS) {
    // k-group kg = 4 tap + channel group.
    const int e = q & 7, nn = (q >> 3) & 31, kg = q >> 8;
    w2s[q] = W2[nn * 288 + kg * 8 + e];
    w3s[q] = W3[nn * 288 + kg * 8 + e];
  }
  uint16_t* w4s = reinterpret_cast<uint16_t*>(sm_ + OFF_W4);
  for (int q = tid; q < 4 * 16 * 8; q += THREADS) {
    // n = tap t (rows 9-15 zero), k = channel.
    const int e = q & 7, t = (q >> 3) & 15, kg = q >> 7;
    w4s[q] = t < 9 ? W4[t * 32 + kg * 8 + e] : (uint16_t)0;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int first = blockIdx.x, stride = gridDim.x;

  if (warp >= EPI / 32) {
    // ---- the MMA warps: issuer i takes the tiles t = i, i + ISSUERS, ... of
    // the 36 an image (layers 1-4 x 9); lane 0 issues, the whole warp waits.
    const int iss = warp - EPI / 32;
    bool ok = true;
    int copies = 0;  // bulk copies issued (issuer 0)
    if (iss == 0) {
      if (lane == 0) fetch_input(stage_a, X + (size_t)first * 2048, bar(BAR_STAGE));
      copies = 1;
    }
    int j = 0;
    for (int img = first; img < n && ok; img += stride, j++) {
      ok = __all_sync(0xffffffffu, wait(bar(BAR_INPUT), (uint32_t)j & 1u, abort_w));
      if (!ok) break;
      // The stage is free again (its contents repacked): the next image's copy.
      if (iss == 0 && img + stride < n) {
        if (lane == 0) fetch_input(stage_a, X + (size_t)(img + stride) * 2048, bar(BAR_STAGE));
        copies++;
      }
      for (int t = iss; t < 4 * TILES; t += ISSUERS) {
        const int layer = t / TILES, u = t % TILES;
        bool w_ok = true;
        if (layer > 0) {
          // The previous layer's tiles u - 1 .. u + 1 stored.
          for (int w = u - 1; w <= u + 1 && w_ok; w++)
            if (w >= 0 && w < TILES) w_ok = wait(bar(BAR_WRITTEN + (layer - 1) * TILES + w), (uint32_t)j & 1u, abort_w);
        }
        const uint32_t seq = (uint32_t)j * (4u * TILES) + (uint32_t)t, s = seq % NSLOT, use = seq / NSLOT;
        if (w_ok && use > 0) w_ok = wait(bar(BAR_EMPTY + (int)s), (use - 1) & 1u, abort_w);
        ok = __all_sync(0xffffffffu, w_ok);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (lane == 0) {
          const uint32_t d = tmem + s * 32;
          const uint32_t v0 = (uint32_t)u * 128;
          if (layer == 0) {
            // Rows dy = -1 and 0 (34 pixels apart), then dy = +1 with a
            // zero-weight half one pixel on.
            mma(d, lptc::smem_desc(b_a + (v0 + 1) * 16, 34 * 16, 128), lptc::smem_desc(w1_a, 512, 128), IDESC32, 0u);
            mma(d, lptc::smem_desc(b_a + (v0 + 69) * 16, 16, 128), lptc::smem_desc(w1_a + 2 * 512, 512, 128), IDESC32,
                1u);
          } else if (layer < 3) {
            const uint32_t src = layer == 1 ? a_a : b_a, w_a = layer == 1 ? w2_a : w3_a;
#pragma unroll
            for (int ks = 0; ks < 18; ks++) {
              const int tap = ks >> 1, hh = ks & 1, off = (tap / 3) * 34 + tap % 3;
              mma(d, lptc::smem_desc(src + (uint32_t)(2 * hh * REGION) + (v0 + off) * 16, REGION, 128),
                  lptc::smem_desc(w_a + (uint32_t)((tap * 4 + 2 * hh) * 512), 512, 128), IDESC32, ks > 0 ? 1u : 0u);
            }
          } else {
            // Layer 4 over A: z for the tile's 128 halo pixels.
            mma(d, lptc::smem_desc(a_a + v0 * 16, REGION, 128), lptc::smem_desc(w4_a, 256, 128), IDESC16, 0u);
            mma(d, lptc::smem_desc(a_a + 2 * REGION + v0 * 16, REGION, 128), lptc::smem_desc(w4_a + 512, 256, 128),
                IDESC16, 1u);
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           bar(BAR_FULL + (int)s))
                       : "memory");
        }
        __syncwarp();
      }
    }
    if (!ok && lane == 0) {
      atomicExch(status, 1u);  // DEV_TIMEOUT
      *abort_w = 1;
    }
    // Drain: every MMA this warp issued, and the last bulk copy, complete
    // before the CTA frees TMEM and leaves.
    if (lane == 0)
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       bar(BAR_FIN + iss))
                   : "memory");
    __syncwarp();
    mbar_wait(bar(BAR_FIN + iss), 0, LIMIT);
    if (iss == 0) mbar_wait(bar(BAR_STAGE), (uint32_t)(copies - 1) & 1u, LIMIT);
    __syncwarp();
  } else {
    // ---- the epilogue warps: warp w reads TMEM lanes 32 (w % 4) .. +31,
    // columns 16 (w / 4) .. +15 of each accumulator.
    const int lq = warp & 3, half = warp >> 2;
    float* z = reinterpret_cast<float*>(sm_ + OFF_Z);
    float* log_s = reinterpret_cast<float*>(sm_ + OFF_LOG);
    unsigned long long* red = reinterpret_cast<unsigned long long*>(sm_ + OFF_RED);
    const float bias4 = __ldg(b4);
    bool ok = true;
    // One image's input from the stage into B's first group: pixel (y, x)
    // holds the pairs of (x - 1, x, x + 1) (zero outside the image) and two
    // zeros; then the hand-over to the MMA warps.
    auto repack = [&]() {
      const uint32_t* st = reinterpret_cast<const uint32_t*>(sm_ + OFF_STAGE);
      for (int p = tid; p < 1024; p += EPI) {
        const int y = p >> 5, x = p & 31;
        const uint32_t l = x > 0 ? st[p - 1] : 0u, c = st[p], r = x < 31 ? st[p + 1] : 0u;
        *reinterpret_cast<uint4*>(sm_ + OFF_B + ((y + 1) * 34 + x + 1) * 16) = make_uint4(l, c, r, 0u);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) arrive(bar(BAR_INPUT));
    };
    // The logits from z (halo rows past the last tile are zero).
    auto outputs = [&]() {
      for (int o = tid; o < 32 * 34; o += EPI) {
        const int y = o / 34, x = o % 34;
        if (x < 32) {
          float acc = 0.f;
#pragma unroll
          for (int tap = 0; tap < 9; tap++) {
            const int h = o + (tap / 3) * 34 + tap % 3;
            acc += h < TILES * 128 ? z[tap * (TILES * 128) + h] : 0.f;
          }
          log_s[y * 32 + x] = acc + bias4;
        }
      }
    };
    ok = !epi_or(!wait(bar(BAR_STAGE), 0u, abort_w));
    if (ok) repack();
    int j = 0;
    for (int img = first; img < n && ok; img += stride, j++) {
      for (int layer = 0; layer < 3 && ok; layer++) {
        const uint32_t dst = layer == 1 ? OFF_B : OFF_A;
        const float* bias = layer == 0 ? b1 : layer == 1 ? b2 : b3;
        float bb[16];
#pragma unroll
        for (int q = 0; q < 16; q++) bb[q] = __ldg(bias + half * 16 + q);
        for (int u = 0; u < TILES; u++) {
          const uint32_t seq = (uint32_t)j * (4u * TILES) + (uint32_t)(layer * TILES + u);
          const uint32_t s = seq % NSLOT, use = seq / NSLOT;
          ok = !epi_or(!wait(bar(BAR_FULL + (int)s), use & 1u, abort_w));
          if (!ok) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          uint32_t r[16];
          tmem_ld16(tmem + ((uint32_t)(32 * lq) << 16) + s * 32 + (uint32_t)(half * 16), r);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) arrive(bar(BAR_EMPTY + (int)s));
          const int v = u * 128 + 32 * lq + lane, y = v / 34, x = v % 34;
          if (y < 32 && x < 32) {
            uint32_t o[8];
#pragma unroll
            for (int q = 0; q < 8; q++)
              o[q] = pack_bf16(fmaxf(__uint_as_float(r[2 * q]) + bb[2 * q], 0.f),
                               fmaxf(__uint_as_float(r[2 * q + 1]) + bb[2 * q + 1], 0.f));
            uint8_t* px = sm_ + dst + ((y + 1) * 34 + x + 1) * 16;
            *reinterpret_cast<uint4*>(px + (2 * half) * REGION) = make_uint4(o[0], o[1], o[2], o[3]);
            *reinterpret_cast<uint4*>(px + (2 * half + 1) * REGION) = make_uint4(o[4], o[5], o[6], o[7]);
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) arrive(bar(BAR_WRITTEN + layer * TILES + u));
        }
      }
      if (!ok) break;
      // Layer 4: z into B's groups 1-3, then the logits in one pass.
      for (int u = 0; u < TILES; u++) {
        const uint32_t seq = (uint32_t)j * (4u * TILES) + (uint32_t)(3 * TILES + u);
        const uint32_t s = seq % NSLOT, use = seq / NSLOT;
        ok = !epi_or(!wait(bar(BAR_FULL + (int)s), use & 1u, abort_w));
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (half == 0) {
          uint32_t r[16];
          tmem_ld16(tmem + ((uint32_t)(32 * lq) << 16) + s * 32, r);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          float* zs = z + u * 128 + 32 * lq + lane;
#pragma unroll
          for (int t = 0; t < 9; t++) zs[t * (TILES * 128)] = __uint_as_float(r[t]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) arrive(bar(BAR_EMPTY + (int)s));
        if (u == 0 && img + stride < n) {
          // Every layer-3 tile's MMAs are done: B's first group takes the next input.
          ok = !epi_or(!wait(bar(BAR_STAGE), (uint32_t)(j + 1) & 1u, abort_w));
          if (!ok) break;
          repack();
        }
      }
      if (!ok) break;
      epi_sync();  // z complete
      outputs();
      epi_sync();  // z read: B's groups 1-3 get their zero halo rings and tails back
      for (int q = tid; q < 3 * (34 * 34 - 32 * 32 + lptc::NV - 34 * 34); q += EPI) {
        const int g = 1 + q / (lptc::NV - 32 * 32), r = q % (lptc::NV - 32 * 32);
        // r-th non-interior pixel of the group: the ring (34 x 34 minus the
        // 32 x 32 interior), then the tail past 34 x 34.
        int h;
        if (r < 34) h = r;                                    // top row
        else if (r < 68) h = 33 * 34 + (r - 34);              // bottom row
        else if (r < 68 + 64) { const int rr = r - 68; h = (1 + (rr >> 1)) * 34 + ((rr & 1) ? 33 : 0); }
        else h = 34 * 34 + (r - 132);                          // tail
        *reinterpret_cast<uint4*>(sm_ + OFF_B + g * REGION + h * 16) = make_uint4(0, 0, 0, 0);
      }
      if (logits)
        for (int q = tid; q < 1024; q += EPI) logits[(size_t)img * 1024 + q] = log_s[q];
      // The top k cells, best first, the first index among equal scores:
      // each thread keeps its four scores in registers; a round publishes
      // the warp maxima (one barrier, the array alternating by round),
      // every thread reduces them alike and the owner drops the chosen cell.
      float mine[4];
#pragma unroll
      for (int i = 0; i < 4; i++) mine[i] = log_s[tid + EPI * i];
      for (int round = 0; round < k; round++) {
        unsigned long long best = 0;
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const unsigned long long key =
              ((unsigned long long)fkey(mine[i]) << 32) | (uint32_t)(1023 - (tid + EPI * i));
          best = key > best ? key : best;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
          best = other > best ? other : best;
        }
        unsigned long long* rr = red + (round & 1) * 8;
        if (lane == 0) rr[warp] = best;
        epi_sync();
        unsigned long long b = rr[0];
#pragma unroll
        for (int w = 1; w < 8; w++) b = rr[w] > b ? rr[w] : b;
        const int cell = 1023 - (int)(b & 0x3ffu);
        if (tid == 0) cells[(size_t)img * k + round] = cell;
#pragma unroll
        for (int i = 0; i < 4; i++)
          if (cell == tid + EPI * i) mine[i] = -INFINITY;
      }
    }
    if (!ok && tid == 0) {
      atomicExch(status, 1u);  // DEV_TIMEOUT
      *abort_w = 1;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// cuTensorMapEncodeTiled, taken from the driver once.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

// The TMA map of n NHWC [32][32][32] BF16 images for the tcgen05 conv: a
// 4-D tensor (channel, x, y, image) with boxes of 8 channels x 34 x 34 x 1.
vp8a_status conv_image_map(const uint16_t* x, uint32_t n, CUtensorMap* tm) {
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) {
    vp8a::set_error("the driver does not provide cuTensorMapEncodeTiled");
    return VP8A_E_CUDA;
  }
  const cuuint64_t gdim[4] = {32, 32, 32, (cuuint64_t)n};
  const cuuint64_t gstride[3] = {32 * 2, 32 * 32 * 2, 32 * 32 * 32 * 2};  // bytes, dims 1..3
  const cuuint32_t box[4] = {8, 34, 34, 1}, estride[4] = {1, 1, 1, 1};
  const CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<uint16_t*>(x), gdim, gstride, box, estride,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    vp8a::set_error("cuTensorMapEncodeTiled rejected the activation map (error " + std::to_string((int)r) + ")");
    return VP8A_E_CUDA;
  }
  return VP8A_OK;
}

template <int CIN, int NT>
vp8a_status conv_fwd(vp8a_ctx* ctx, const uint16_t* X, const uint16_t* W, const float* b, int cout, int n, int relu,
                     uint16_t* Y, float* Yf) {
  if (n == 0) return VP8A_OK;
  constexpr int CP = (CIN + 15) / 16 * 16, PS = CP + 8, WS = 9 * CIN + 8;
  const size_t smem = sizeof(uint16_t) * (34 * 34 * PS + NT * 8 * WS);
  VP8A_CUDA(cudaFuncSetAttribute(lp_conv_fwd_smem_kernel<CIN, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  lp_conv_fwd_smem_kernel<CIN, NT><<<n, 256, smem, ctx->stream>>>(X, W, b, cout, relu, Y, Yf);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

template <int COUT, int NT>
vp8a_status conv_bwd_data(vp8a_ctx* ctx, const uint16_t* dY, const uint16_t* W, int cin, int n, const uint16_t* Xa,
                          uint16_t* dX) {
  const int tiles = n * (LP_P / 16);
  lp_conv_bwd_data_kernel<COUT, NT><<<(tiles + 3) / 4, 128, 0, ctx->stream>>>(dY, W, cin, n, Xa, dX);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

// Weight gradient with staged chunks: each CTA walks LP_WCPB chunks of 512
// pixels (half an image each), staging the chunk's dY ([pixel][co], co
// padded to 16 * MT) and its 18 input rows with a zero halo ([row][col][ci])
// in shared memory; warp w accumulates the n-tiles w, w + 4, ... of
// dW = dY^T x im2col(X) in registers across all its chunks, and the CTA
// adds its partial sums with one atomic per weight at the end.
constexpr int LP_WCPB = 16;
template <int CIN, int MT>
__global__ void __launch_bounds__(128) lp_conv_bwd_w_smem_kernel(const uint16_t* dY, const uint16_t* X, int cout,
                                                                 long n_chunks, float* dW, float* db) {
  constexpr int NTOT = (9 * CIN + 7) / 8, NPW = (NTOT + 3) / 4;
  constexpr int DS = 16 * MT + 8, PS = CIN + (CIN >= 16 ? 8 : 0) + (CIN < 16 ? 2 : 0);
  extern __shared__ __align__(16) uint16_t smw[];
  uint16_t* dy_s = smw;                        // 512 * DS
  uint16_t* x_s = smw + LP_WCHUNK * DS;        // 18 * 34 * PS
  const int tid = threadIdx.x, lane = tid & 31, g = lane >> 2, t = lane & 3, warp = tid >> 5;
  float d[NPW][MT][4];
#pragma unroll
  for (int a = 0; a < NPW; a++)
#pragma unroll
    for (int m = 0; m < MT; m++) d[a][m][0] = d[a][m][1] = d[a][m][2] = d[a][m][3] = 0.f;
  float bsum = 0.f;
  for (long ch = (long)blockIdx.x * LP_WCPB; ch < n_chunks && ch < (long)(blockIdx.x + 1) * LP_WCPB; ch++) {
    const long p0 = ch * LP_WCHUNK;
    const int img = (int)(p0 / LP_P), row0 = (int)(p0 % LP_P) / 32;
    __syncthreads();  // the previous chunk's fragments are read
    for (int q = tid; q < LP_WCHUNK * DS; q += 128) {
      const int pp = q / DS, co = q % DS;
      dy_s[q] = co < cout ? dY[(p0 + pp) * cout + co] : (uint16_t)0;
    }
    for (int q = tid; q < 18 * 34 * PS; q += 128) {
      const int ci = q % PS, c = (q / PS) % 34, r = q / (PS * 34);
      const int y = row0 + r - 1, x = c - 1;
      x_s[q] = (ci < CIN && y >= 0 && y < 32 && x >= 0 && x < 32)
                   ? X[((size_t)img * LP_P + y * 32 + x) * CIN + ci]
                   : (uint16_t)0;
    }
    __syncthreads();
    if (tid < cout)
      for (int pp = 0; pp < LP_WCHUNK; pp++) bsum += __bfloat162float(__ushort_as_bfloat16(dy_s[pp * DS + tid]));
#pragma unroll
    for (int a = 0; a < NPW; a++) {
      const int nt = warp + 4 * a;
      if (nt >= NTOT) break;
      const int n = nt * 8 + g;
      const bool nv = n < 9 * CIN;
      const int tap = nv ? n / CIN : 0, ci = nv ? n % CIN : 0, oy = tap / 3, ox = tap % 3;
      for (int k0 = 0; k0 < LP_WCHUNK; k0 += 16) {
        auto xv = [&](int pp) -> uint32_t {
          return nv ? x_s[(((pp >> 5) + oy) * 34 + (pp & 31) + ox) * PS + ci] : 0u;
        };
        const uint32_t b[2] = {xv(k0 + 2 * t) | (xv(k0 + 2 * t + 1) << 16),
                               xv(k0 + 2 * t + 8) | (xv(k0 + 2 * t + 9) << 16)};
#pragma unroll
        for (int m = 0; m < MT; m++) {
          const int m0 = m * 16 + g, m1 = m0 + 8;
          auto dv = [&](int co, int pp) -> uint32_t { return dy_s[pp * DS + co]; };
          const uint32_t av[4] = {dv(m0, k0 + 2 * t) | (dv(m0, k0 + 2 * t + 1) << 16),
                                  dv(m1, k0 + 2 * t) | (dv(m1, k0 + 2 * t + 1) << 16),
                                  dv(m0, k0 + 2 * t + 8) | (dv(m0, k0 + 2 * t + 9) << 16),
                                  dv(m1, k0 + 2 * t + 8) | (dv(m1, k0 + 2 * t + 9) << 16)};
          mma_bf16(d[a][m], av, b);
        }
      }
    }
  }
#pragma unroll
  for (int a = 0; a < NPW; a++) {
    const int nt = warp + 4 * a;
    if (nt >= NTOT) break;
#pragma unroll
    for (int m = 0; m < MT; m++)
#pragma unroll
      for (int h = 0; h < 2; h++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int co = m * 16 + g + 8 * h, n = nt * 8 + 2 * t + e;
          if (co < cout && n < 9 * CIN) atomicAdd(&dW[(size_t)co * 9 * CIN + n], d[a][m][2 * h + e]);
        }
  }
  if (tid < cout) atomicAdd(&db[tid], bsum);
}

template <int CIN>
vp8a_status conv_bwd_w(vp8a_ctx* ctx, const uint16_t* dY, const uint16_t* X, int cout, int n, float* dW, float* db) {
  const long n_chunks = (long)n * LP_P / LP_WCHUNK;
  const unsigned grid = (unsigned)((n_chunks + LP_WCPB - 1) / LP_WCPB);
  if (grid == 0) return VP8A_OK;
  constexpr int PS = CIN + (CIN >= 16 ? 8 : 0) + (CIN < 16 ? 2 : 0);
  if (cout > 16) {
    const size_t smem = sizeof(uint16_t) * (LP_WCHUNK * (32 + 8) + 18 * 34 * PS);
    VP8A_CUDA(cudaFuncSetAttribute(lp_conv_bwd_w_smem_kernel<CIN, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    lp_conv_bwd_w_smem_kernel<CIN, 2><<<grid, 128, smem, ctx->stream>>>(dY, X, cout, n_chunks, dW, db);
  } else {
    const size_t smem = sizeof(uint16_t) * (LP_WCHUNK * (16 + 8) + 18 * 34 * PS);
    VP8A_CUDA(cudaFuncSetAttribute(lp_conv_bwd_w_smem_kernel<CIN, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    lp_conv_bwd_w_smem_kernel<CIN, 1><<<grid, 128, smem, ctx->stream>>>(dY, X, cout, n_chunks, dW, db);
  }
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

}  // namespace

extern "C" {

vp8a_status vp8a_lp_windows(vp8a_ctx* ctx, const vp8a_luma_ref* src, const vp8a_luma_ref* ref, const uint32_t* mb_xy,
                            uint32_t n, uint16_t* out) {
  if (!ctx || !src || !ref || (n && (!mb_xy || !out))) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (src->width != ref->width || src->height != ref->height || !src->width || !src->height) {
    vp8a::set_error("source and reference planes differ in size");
    return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
  }
  if (n == 0) return VP8A_OK;
  if ((uintptr_t)out & 15) {
    vp8a::set_error("out must be 16-byte aligned");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  lp_windows_kernel<<<n, 256, 0, ctx->stream>>>(src->plane, src->stride, ref->plane, ref->stride, (int)src->width,
                                                 (int)src->height, mb_xy, (int)n, out);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

vp8a_status vp8a_lp_seeded_search(vp8a_ctx* ctx, const vp8a_luma_ref* ref, const uint8_t* src_mbs,
                                  const uint32_t* mb_xy, const int32_t* seeds, uint32_t k, uint32_t radius, uint32_t n,
                                  vp8a_search_result* out) {
  if (!ctx || !ref || (n && (!src_mbs || !mb_xy || !seeds || !out))) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (k < 1 || k > 4 || radius > 4 || k * (2 * radius + 1) * (2 * radius + 1) > (uint32_t)LP_SEED_MAXC) {
    vp8a::set_error("seeded search: 1 <= k <= 4, radius <= 4 and k * (2 radius + 1)^2 <= 128");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (!ref->plane || ref->width < 16 || ref->height < 16 || ref->stride < ref->width) {
    vp8a::set_error("bad reference plane");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (n == 0) return VP8A_OK;
  VP8A_CUDA(cudaSetDevice(ctx->device));
  lp_seeded_search_kernel<<<n, LP_SEED_MAXC, 0, ctx->stream>>>(ref->plane, ref->stride, (int)ref->width,
                                                                (int)ref->height, src_mbs, mb_xy, seeds, (int)k,
                                                                (int)radius, out);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

vp8a_status vp8a_lp_net_propose(vp8a_ctx* ctx, const uint16_t* x, uint32_t n, const uint16_t* w1, const float* b1,
                                const uint16_t* w2, const float* b2, const uint16_t* w3, const float* b3,
                                const uint16_t* w4, const float* b4, uint32_t k, int32_t* cells, float* logits) {
  if (!ctx || (n && (!x || !w1 || !b1 || !w2 || !b2 || !w3 || !b3 || !w4 || !b4 || !cells))) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (k < 1 || k > 16) {
    vp8a::set_error("k must be 1..16");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if ((((uintptr_t)x) & 15) || (((uintptr_t)w1 | (uintptr_t)w2 | (uintptr_t)w3 | (uintptr_t)w4) & 1)) {
    vp8a::set_error("the input must be 16-byte aligned, the weights 2-byte aligned");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (n == 0) return VP8A_OK;
  VP8A_CUDA(cudaSetDevice(ctx->device));
  VP8A_CUDA(cudaFuncSetAttribute(lp_net_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lpnet::SMEM));
  const unsigned grid = (unsigned)std::min<uint32_t>(n, (uint32_t)ctx->sm_count);
  lp_net_kernel<<<grid, lpnet::THREADS, lpnet::SMEM, ctx->stream>>>(x, (int)n, w1, b1, w2, b2, w3, b3, w4, b4, (int)k, cells,
                                                          logits, ctx->d_status);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

vp8a_status vp8a_lp_conv_forward(vp8a_ctx* ctx, const uint16_t* x, uint32_t cin, const uint16_t* w, const float* bias,
                                 uint32_t cout, uint32_t n, uint32_t relu, uint16_t* y, float* y_f32) {
  if (!ctx || !x || !w || !bias || (!y && !y_f32)) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  if (cin == 2 && cout == 32) return conv_fwd<2, 4>(ctx, x, w, bias, 32, (int)n, relu, y, y_f32);
  if (cin == 32 && cout == 32 && y && !y_f32 && n > 0) {
    // The tensor-core path: 16-byte aligned activations and weights.
    if (((uintptr_t)x | (uintptr_t)w | (uintptr_t)y) & 15) {
      vp8a::set_error("tensor-core conv needs 16-byte aligned buffers");
      return VP8A_E_INVALID_ARGUMENT;
    }
    CUtensorMap tm;
    const vp8a_status s = conv_image_map(x, n, &tm);
    if (s != VP8A_OK) return s;
    VP8A_CUDA(cudaFuncSetAttribute(lp_conv_fwd_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lptc::SMEM));
    lp_conv_fwd_tc_kernel<<<n, 256, lptc::SMEM, ctx->stream>>>(tm, w, bias, (int)relu, y, ctx->d_status);
    VP8A_CUDA(cudaGetLastError());
    ctx->launches++;
    return VP8A_OK;
  }
  if (cin == 32 && cout == 32) return conv_fwd<32, 4>(ctx, x, w, bias, 32, (int)n, relu, y, y_f32);
  if (cin == 32 && cout == 1) return conv_fwd<32, 1>(ctx, x, w, bias, 1, (int)n, relu, y, y_f32);
  vp8a::set_error("conv shape must be 2->32, 32->32 or 32->1");
  return VP8A_E_INVALID_ARGUMENT;
}

vp8a_status vp8a_lp_conv_backward(vp8a_ctx* ctx, const uint16_t* x, uint32_t cin, const uint16_t* w, uint32_t cout,
                                  uint32_t n, const uint16_t* dy, uint32_t x_relu, uint16_t* dx, float* dw,
                                  float* db) {
  if (!ctx || !x || !w || !dy || !dw || !db) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a_status s;
  const uint16_t* mask = x_relu ? x : nullptr;
  if (cin == 2 && cout == 32) {
    if ((s = conv_bwd_w<2>(ctx, dy, x, 32, (int)n, dw, db)) != VP8A_OK) return s;
    if (dx) return conv_bwd_data<32, 1>(ctx, dy, w, 2, (int)n, mask, dx);
    return VP8A_OK;
  }
  if (cin == 32 && cout == 32) {
    if ((s = conv_bwd_w<32>(ctx, dy, x, 32, (int)n, dw, db)) != VP8A_OK) return s;
    if (dx) return conv_bwd_data<32, 4>(ctx, dy, w, 32, (int)n, mask, dx);
    return VP8A_OK;
  }
  if (cin == 32 && cout == 1) {
    if ((s = conv_bwd_w<32>(ctx, dy, x, 1, (int)n, dw, db)) != VP8A_OK) return s;
    if (dx) return conv_bwd_data<1, 4>(ctx, dy, w, 32, (int)n, mask, dx);
    return VP8A_OK;
  }
  vp8a::set_error("conv shape must be 2->32, 32->32 or 32->1");
  return VP8A_E_INVALID_ARGUMENT;
}

vp8a_status vp8a_lp_softmax_ce(vp8a_ctx* ctx, const float* logits, const int32_t* labels, uint32_t n,
                               uint16_t* dlogits, float* loss, float* label_prob) {
  if (!ctx || !logits) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (n == 0) return VP8A_OK;
  VP8A_CUDA(cudaSetDevice(ctx->device));
  lp_softmax_ce_kernel<<<n, 256, 0, ctx->stream>>>(logits, labels, (int)n, dlogits, loss, label_prob);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

vp8a_status vp8a_lp_adam(vp8a_ctx* ctx, float* w, const float* grad, float* m, float* v, uint32_t n, float lr,
                         float beta1, float beta2, float eps, uint32_t step, uint16_t* w_bf16) {
  if (!ctx || !w || !grad || !m || !v || !w_bf16 || step == 0) {
    vp8a::set_error("null argument or step 0");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (n == 0) return VP8A_OK;
  VP8A_CUDA(cudaSetDevice(ctx->device));
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  lp_adam_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(w, grad, m, v, (int)n, lr, beta1, beta2, eps, c1, c2,
                                                            w_bf16);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

vp8a_status vp8a_lp_pool(vp8a_ctx* ctx, const uint16_t* x, uint32_t c, uint32_t n, float* sums) {
  if (!ctx || !sums || (n && !x) || c == 0 || c > 64 || 256 % c != 0) {
    vp8a::set_error("null argument or channel count not a divisor of 256 up to 64");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (n == 0) return VP8A_OK;
  VP8A_CUDA(cudaSetDevice(ctx->device));
  lp_pool_kernel<<<n, 256, 0, ctx->stream>>>(x, (int)c, sums);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

vp8a_status vp8a_lp_lf_head(vp8a_ctx* ctx, const float* sums, float count, uint32_t c, const float* w,
                            const float* b, uint32_t levels, int32_t label, float* logits, float* dw, float* db,
                            float* loss) {
  if (!ctx || !sums || !w || !b || c == 0 || c > 64 || levels == 0 || levels > 128 || !(count > 0.f) ||
      (label >= 0 && (!dw || !db || label >= (int32_t)levels))) {
    vp8a::set_error("bad loop-filter head arguments");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  lp_lf_head_kernel<<<1, 128, 0, ctx->stream>>>(sums, count, (int)c, w, b, (int)levels, label, logits, dw, db, loss);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

}  // extern "C"
