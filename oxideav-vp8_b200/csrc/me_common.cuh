// me_common.cuh — warp-level motion-search building blocks shared by the
// batched search kernels (me.cu) and the wavefront analysis (analysis.cu).
//
// A warp owns one (MB, reference) item. The reference luma around the
// search centre is staged once in shared memory as an edge-clamped window
// (the §20.14 edge replication of fetch_luma_mb_whole_pixel /
// fetch_luma_mb_halo, src/motion_comp.rs:837,1513, is applied while the
// window is filled), so every later SAD or six-tap read is an unchecked
// shared-memory access. Candidates that leave the window fall back to
// clamped global loads with identical results.
#pragma once

#include "vp8a_internal.cuh"

namespace vp8a_dev {

constexpr unsigned FULL = 0xffffffffu;
constexpr int WS = 40;              // window extent and stride (bytes)
constexpr int WIN_BYTES = WS * WS + 16;
constexpr int WIN_R = 8;            // diamond radius the window is sized for
constexpr int WIN_LEAD = WIN_R + 3; // window origin = centre - WIN_LEAD

struct MePlane {
  const uint8_t* plane;
  uint64_t stride;
  int width;
  int height;
};

// Every member is a multiple of 16 bytes and the struct is 16-byte aligned,
// so arrays of it (and structs embedding it) keep word access aligned.
struct __align__(16) WarpScratch {
  uint8_t win[WIN_BYTES];        // 1616
  uint8_t temp[21 * 16 + 16];    // 352
  uint8_t halo[21 * 24 + 24];    // 528
  // Half-pel planes around a whole-pel centre: H 22x17, V 17x16, D 17x17.
  uint8_t hp[22 * 17 + 10];      // 384
  uint8_t vp[17 * 16 + 16];      // 288
  uint8_t dp[17 * 17 + 15];      // 304
};
static_assert(sizeof(WarpScratch) % 16 == 0, "WarpScratch must keep 16-byte multiples");

__device__ __forceinline__ int16_t clamp_component(int v) { return (int16_t)clampi(v, -1023, 1023); }
__device__ __forceinline__ int16_t snap_whole(int v) { return (int16_t)((v / 4) * 4); }
// stored_luma_mv (src/motion_comp.rs:187): wrapping doubling.
__device__ __forceinline__ int eighth(int16_t v) { return (int)(int16_t)(uint16_t)((uint16_t)v * 2u); }

// 8 unaligned bytes from shared memory as two little-endian words.
__device__ __forceinline__ void load8u(const uint8_t* p, uint32_t& o0, uint32_t& o1) {
  uintptr_t a = (uintptr_t)p;
  const uint32_t* w = (const uint32_t*)(a & ~(uintptr_t)3);
  unsigned sh = (unsigned)(a & 3) * 8u;
  uint32_t w0 = w[0], w1 = w[1], w2 = w[2];
  o0 = __funnelshift_r(w0, w1, sh);
  o1 = __funnelshift_r(w1, w2, sh);
}

// Fill a WS x WS window whose top-left is plane pixel (x0, y0), clamping
// every coordinate into the plane.
__device__ __forceinline__ void load_window(const MePlane& P, uint8_t* win, int x0, int y0, int lane) {
  for (int r = 0; r < WS; r++) {
    int y = clampi(y0 + r, 0, P.height - 1);
    const uint8_t* row = P.plane + (size_t)y * P.stride;
    for (int c = lane; c < WS; c += 32) win[r * WS + c] = row[clampi(x0 + c, 0, P.width - 1)];
  }
  __syncwarp();
}

// Source MB in shared memory (16x16, stride 16); each lane's 8-byte slice
// is lane>>1 = row, (lane&1)*8 = column.
__device__ __forceinline__ uint32_t sad_win16(const uint8_t* win, int lx, int ly, const uint8_t* src, int lane) {
  int row = lane >> 1, c0 = (lane & 1) * 8;
  uint32_t r0, r1;
  load8u(win + (ly + row) * WS + lx + c0, r0, r1);
  const uint32_t* sp = (const uint32_t*)(src + row * 16 + c0);
  uint32_t s = __vsadu4(r0, sp[0]) + __vsadu4(r1, sp[1]);
  return __reduce_add_sync(FULL, s);
}

// Whole-pel SAD of the 16x16 block at plane pixel (x0, y0), clamped loads.
__device__ __forceinline__ uint32_t sad_global16(const MePlane& P, int x0, int y0, const uint8_t* src, int lane) {
  int row = lane >> 1, c0 = (lane & 1) * 8;
  int y = clampi(y0 + row, 0, P.height - 1);
  const uint8_t* pr = P.plane + (size_t)y * P.stride;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int d = (int)pr[clampi(x0 + c0 + k, 0, P.width - 1)] - (int)src[row * 16 + c0 + k];
    s += (uint32_t)(d < 0 ? -d : d);
  }
  return __reduce_add_sync(FULL, s);
}

// Whole-pel SAD at plane pixel (x0, y0): window when it covers the block.
__device__ __forceinline__ uint32_t sad_whole_at(const MePlane& P, const uint8_t* win, int wx0, int wy0,
                                                 int x0, int y0, const uint8_t* src, int lane) {
  int lx = x0 - wx0, ly = y0 - wy0;
  if (lx >= 0 && ly >= 0 && lx <= WS - 16 && ly <= WS - 16) return sad_win16(win, lx, ly, src, lane);
  return sad_global16(P, x0, y0, src, lane);
}

// §18.3 two-pass six-tap prediction SAD (sixtap_mb_luma,
// src/motion_comp.rs:902-1057) from a 21x21 halo at `h` (stride hs; block
// origin at (2, 2)). The horizontal pass keeps its 8-bit clamp; a pass
// whose fraction is 0 is the identity and is skipped (the reference's own
// identity elision, src/motion_comp.rs:960-1007).
__device__ __forceinline__ uint32_t subpel_sad(const uint8_t* h, int hs, int mx, int my, const uint8_t* src,
                                               uint8_t* temp, int lane) {
  const int c = lane & 15;
  if (mx) {
    const int* fh = c_sixtap[mx];
    for (int r = lane >> 4; r < 21; r += 2) {
      const uint8_t* p = h + r * hs + c;
      temp[r * 16 + c] = (uint8_t)interp6(fh, p[0], p[1], p[2], p[3], p[4], p[5]);
    }
    __syncwarp();
  }
  const int* fv = c_sixtap[my];
  const int r0 = (lane >> 4) * 8;
  uint32_t s = 0;
#pragma unroll 2
  for (int r = r0; r < r0 + 8; r++) {
    int v;
    if (mx) {
      const uint8_t* t = temp + r * 16 + c;
      v = my ? interp6(fv, t[0], t[16], t[32], t[48], t[64], t[80]) : t[32];
    } else {
      const uint8_t* p = h + r * hs + c + 2;
      v = my ? interp6(fv, p[0], p[hs], p[2 * hs], p[3 * hs], p[4 * hs], p[5 * hs]) : p[2 * hs];
    }
    int d = v - (int)src[r * 16 + c];
    s += (uint32_t)(d < 0 ? -d : d);
  }
  __syncwarp();
  return __reduce_add_sync(FULL, s);
}

// mb_luma_sad_at_mv (src/motion_search.rs:470-529) for the MB at plane
// pixel (mbx, mby), served from the window when it covers the candidate.
// `temp` (21 x 16 bytes) and `halo` (21 x 24) are the warp's own scratch.
__device__ __forceinline__ uint32_t sad_at_mv(const MePlane& P, const uint8_t* win, uint8_t* temp, uint8_t* halo,
                                              int wx0, int wy0, int mbx, int mby, int16_t mv_row, int16_t mv_col,
                                              const uint8_t* src, int lane) {
  int er = eighth(mv_row), ec = eighth(mv_col);
  int mx = ec & 7, my = er & 7;
  int bx = mbx + (ec >> 3), by = mby + (er >> 3);
  if (mx == 0 && my == 0) return sad_whole_at(P, win, wx0, wy0, bx, by, src, lane);
  int hx = bx - 2, hy = by - 2;
  int lx = hx - wx0, ly = hy - wy0;
  if (lx >= 0 && ly >= 0 && lx <= WS - 21 && ly <= WS - 21)
    return subpel_sad(win + ly * WS + lx, WS, mx, my, src, temp, lane);
  // Out-of-window halo: clamped fetch into scratch (fetch_luma_mb_halo).
  for (int r = 0; r < 21; r++) {
    int y = clampi(hy + r, 0, P.height - 1);
    const uint8_t* row = P.plane + (size_t)y * P.stride;
    if (lane < 21) halo[r * 24 + lane] = row[clampi(hx + lane, 0, P.width - 1)];
  }
  __syncwarp();
  uint32_t s = subpel_sad(halo, 24, mx, my, src, temp, lane);
  return s;
}

__device__ __forceinline__ uint32_t sad_at_mv(const MePlane& P, WarpScratch& S, int wx0, int wy0, int mbx,
                                              int mby, int16_t mv_row, int16_t mv_col, const uint8_t* src,
                                              int lane) {
  return sad_at_mv(P, S.win, S.temp, S.halo, wx0, wy0, mbx, mby, mv_row, mv_col, src, lane);
}

// small_diamond_search_luma (src/motion_search.rs:381-442). Each round
// scores the eight whole-pel neighbours of the round's starting best in
// parallel (four lanes per neighbour), then replays the reference's
// sequential N, S, W, E walk — whose candidates all lie in that 3x3
// neighbourhood — with its strict '<' and collapse skips.
__device__ __forceinline__ vp8a_search_result diamond(const MePlane& P, WarpScratch& S, int wx0, int wy0,
                                                      int mbx, int mby, vp8a_mv center, uint32_t max_iters,
                                                      const uint8_t* src, int lane) {
  vp8a_mv best;
  best.row = snap_whole(clamp_component(center.row));
  best.col = snap_whole(clamp_component(center.col));
  uint32_t best_sad = sad_whole_at(P, S.win, wx0, wy0, mbx + best.col / 4, mby + best.row / 4, src, lane);
  const int k = lane >> 2, q = lane & 3;
  // Neighbour k of the 3x3 ring (row, col) in pixels; index 4 is skipped.
  const int kr = (k < 3) ? -1 : (k < 5 ? 0 : 1);
  const int kc = (k == 0 || k == 3 || k == 5) ? -1 : ((k == 1 || k == 6) ? 0 : 1);
  for (uint32_t it = 0; it < max_iters; it++) {
    const int bx = mbx + best.col / 4, by = mby + best.row / 4;
    const int lx = bx - 1 - wx0, ly = by - 1 - wy0;
    uint32_t tab[8];
    if (lx >= 0 && ly >= 0 && lx + 18 <= WS && ly + 18 <= WS) {
      uint32_t s = 0;
      const uint8_t* base = S.win + (ly + 1 + kr + q * 4) * WS + (lx + 1 + kc);
#pragma unroll
      for (int r = 0; r < 4; r++) {
        uint32_t a0, a1, a2, a3;
        load8u(base + r * WS, a0, a1);
        load8u(base + r * WS + 8, a2, a3);
        const uint32_t* sp = (const uint32_t*)(src + (q * 4 + r) * 16);
        s += __vsadu4(a0, sp[0]) + __vsadu4(a1, sp[1]) + __vsadu4(a2, sp[2]) + __vsadu4(a3, sp[3]);
      }
      s += __shfl_xor_sync(FULL, s, 1);
      s += __shfl_xor_sync(FULL, s, 2);
#pragma unroll
      for (int j = 0; j < 8; j++) tab[j] = __shfl_sync(FULL, s, j * 4);
    } else {
#pragma unroll 1
      for (int j = 0; j < 8; j++) {
        int jr = (j < 3) ? -1 : (j < 5 ? 0 : 1);
        int jc = (j == 0 || j == 3 || j == 5) ? -1 : ((j == 1 || j == 6) ? 0 : 1);
        tab[j] = sad_whole_at(P, S.win, wx0, wy0, bx + jc, by + jr, src, lane);
      }
    }
    // Replay the reference's walk over the 3x3 table.
    vp8a_mv b = best;
    uint32_t bs = best_sad;
    bool improved = false;
    const int dr[4] = {-4, 4, 0, 0}, dc[4] = {0, 0, -4, 4};
#pragma unroll
    for (int d = 0; d < 4; d++) {
      vp8a_mv cand;
      cand.row = snap_whole(clamp_component(b.row + dr[d]));
      cand.col = snap_whole(clamp_component(b.col + dc[d]));
      if (cand.row == b.row && cand.col == b.col) continue;
      int rr = (cand.row - best.row) / 4, rc = (cand.col - best.col) / 4;
      uint32_t s;
      if (rr == 0 && rc == 0) s = best_sad;
      else {
        int idx = (rr + 1) * 3 + (rc + 1);
        s = tab[idx < 4 ? idx : idx - 1];
      }
      if (s < bs) {
        bs = s;
        b = cand;
        improved = true;
      }
    }
    best = b;
    best_sad = bs;
    if (!improved) break;
  }
  vp8a_search_result res;
  res.mv = best;
  res.sad = best_sad;
  return res;
}

// half_pixel_refine_luma / quarter_pixel_refine_luma
// (src/motion_search.rs:564-728): centre plus 8 offsets of `step`
// quarter-pels in the fixed order, strict '<', collapse skips.
// `center_sad` is the SAD at `center` when the caller already has it (the
// previous refinement's result), else ~0u.
__device__ __forceinline__ vp8a_search_result refine(const MePlane& P, WarpScratch& S, int wx0, int wy0, int mbx,
                                                     int mby, vp8a_mv center, int step, const uint8_t* src,
                                                     int lane, uint32_t center_sad = ~0u) {
  vp8a_mv best = center;
  uint32_t best_sad = center_sad != ~0u ? center_sad
                                        : sad_at_mv(P, S, wx0, wy0, mbx, mby, center.row, center.col, src, lane);
#pragma unroll 1
  for (int k = 0; k < 8; k++) {
    // Offsets (-1,-1) (-1,0) (-1,1) (0,-1) (0,1) (1,-1) (1,0) (1,1).
    const int orow = (k < 3) ? -1 : (k < 5 ? 0 : 1);
    const int ocol = (k == 0 || k == 3 || k == 5) ? -1 : ((k == 1 || k == 6) ? 0 : 1);
    vp8a_mv cand;
    cand.row = clamp_component(center.row + orow * step);
    cand.col = clamp_component(center.col + ocol * step);
    if (cand.row == best.row && cand.col == best.col) continue;
    uint32_t s = sad_at_mv(P, S, wx0, wy0, mbx, mby, cand.row, cand.col, src, lane);
    if (s < best_sad) {
      best_sad = s;
      best = cand;
    }
  }
  vp8a_search_result res;
  res.mv = best;
  res.sad = best_sad;
  return res;
}

// The eight half-pel candidates around a whole-pel centre share three
// planes — horizontal (H), vertical (V) and horizontal-then-vertical (D)
// half-pel samples — so each six-tap output is computed once per MB instead
// of once per candidate; every candidate's prediction is a 16x16 sub-block
// of one plane, byte-identical to its own two-pass synthesis (same taps,
// same 8-bit intermediate, same edge-clamped source). half_plane_sads fills
// sads[k] for the offsets (row, col) = (-1,-1) (-1,0) (-1,1) (0,-1) (0,1)
// (1,-1) (1,0) (1,1) half-pels, in that order (the order of
// half_pixel_refine_luma, src/motion_search.rs:589-598, and of
// sub_pixel_refine, src/encoder/inter_search.rs:520-535), and returns false
// when the window does not cover the planes.
__device__ __forceinline__ bool half_plane_sads(WarpScratch& S, int wx0, int wy0, int mbx, int mby, vp8a_mv center,
                                                const uint8_t* src, int lane, uint32_t* sads) {
  if ((center.row & 3) || (center.col & 3)) return false;
  const int bx = mbx + center.col / 4 - wx0, by = mby + center.row / 4 - wy0;  // block origin in window
  if (bx < 3 || by < 3 || bx + 19 > WS || by + 19 > WS) return false;
  // H: 22 rows (window rows by-3 .. by+18), 17 outputs at x = bx + i - 0.5.
  for (int o = lane; o < 22 * 17; o += 32) {
    const int r = o / 17, i = o - r * 17;
    const uint8_t* p = S.win + (by - 3 + r) * WS + bx + i - 3;
    S.hp[o] = (uint8_t)interp6_half(p[0], p[1], p[2], p[3], p[4], p[5]);
  }
  // V: 17 rows at y = by + r - 0.5, 16 columns.
  for (int o = lane; o < 17 * 16; o += 32) {
    const int r = o >> 4, c = o & 15;
    const uint8_t* p = S.win + (by + r - 3) * WS + bx + c;
    S.vp[o] = (uint8_t)interp6_half(p[0], p[WS], p[2 * WS], p[3 * WS], p[4 * WS], p[5 * WS]);
  }
  __syncwarp();
  // D: vertical half-pel over H (rows r..r+5 of H), 17 x 17.
  for (int o = lane; o < 17 * 17; o += 32) {
    const int r = o / 17, i = o - r * 17;
    const uint8_t* p = S.hp + r * 17 + i;
    S.dp[o] = (uint8_t)interp6_half(p[0], p[17], p[34], p[51], p[68], p[85]);
  }
  __syncwarp();
  const int c = lane & 15, r0 = (lane >> 4) * 8;
#pragma unroll 1
  for (int k = 0; k < 8; k++) {
    const int dy = (k < 3) ? -1 : (k < 5 ? 0 : 1);
    const int dx = (k == 0 || k == 3 || k == 5) ? -1 : ((k == 1 || k == 6) ? 0 : 1);
    const int cx = dx > 0, cy = dy > 0;
    const uint8_t* pl;
    int st;
    if (dy == 0) {
      pl = S.hp + 3 * 17 + cx;
      st = 17;
    } else if (dx == 0) {
      pl = S.vp + cy * 16;
      st = 16;
    } else {
      pl = S.dp + cy * 17 + cx;
      st = 17;
    }
    uint32_t s = 0;
#pragma unroll
    for (int r = r0; r < r0 + 8; r++) {
      const int d = (int)pl[r * st + c] - (int)src[r * 16 + c];
      s += (uint32_t)(d < 0 ? -d : d);
    }
    sads[k] = __reduce_add_sync(FULL, s);
  }
  return true;
}

// half_pixel_refine_luma (src/motion_search.rs:564-627) over the shared
// planes; for a whole-pel centre inside [-1020, 1020] no candidate is
// clamped or collapses, so the reference walk is the first strict minimum.
__device__ __forceinline__ bool half_refine_planes(WarpScratch& S, int wx0, int wy0, int mbx, int mby,
                                                   vp8a_mv center, const uint8_t* src, int lane,
                                                   vp8a_search_result* out) {
  if (center.row < -1020 || center.row > 1020 || center.col < -1020 || center.col > 1020) return false;
  uint32_t sads[8];
  if (!half_plane_sads(S, wx0, wy0, mbx, mby, center, src, lane, sads)) return false;
  const int bx = mbx + center.col / 4 - wx0, by = mby + center.row / 4 - wy0;
  vp8a_mv best = center;
  uint32_t best_sad = sad_win16(S.win, bx, by, src, lane);
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int dy = (k < 3) ? -1 : (k < 5 ? 0 : 1);
    const int dx = (k == 0 || k == 3 || k == 5) ? -1 : ((k == 1 || k == 6) ? 0 : 1);
    if (sads[k] < best_sad) {
      best_sad = sads[k];
      best.row = (int16_t)(center.row + 2 * dy);
      best.col = (int16_t)(center.col + 2 * dx);
    }
  }
  out->mv = best;
  out->sad = best_sad;
  return true;
}

}  // namespace vp8a_dev
