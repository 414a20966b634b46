// lf.cu — §15 loop filter and the §9.4 (level, sharpness) search.
//
// Entry points:
//   vp8a_filter_frame                  filter_inter_frame_flags / filter_frame_flags
//                                      (src/loop_filter.rs:1364, :2506), in place
//   vp8a_reconstruction_ssd            (src/loop_filter.rs:1965)
//   vp8a_filter_sweep                  score_filter_candidate (:2062) for all 64 x 8
//   vp8a_select_filter_params          select_filter_params_threaded (:2133)
//   vp8a_select_filter_params_sampled  select_filter_params_sampled (:2288)
//
// Kernel design. One CTA filters the whole picture for one (level,
// sharpness) candidate and returns its visible-window SSD against the
// source. The §15 raster order makes MB (r, c) depend on (r, c-1) and
// (r-1, c+1) (the filter never writes right of or below the MB it
// processes), so MB (r, c) runs at wavefront step t = t0(r) + c with
// t0(r) = 2r. Warps own MB rows; at each step every active row filters one
// MB, and one __syncthreads separates steps. A row keeps its last four MBs
// in a ring of shared-memory slots (Y 16x16 + U 8x8 + V 8x8 = 384 B): an MB
// is loaded from the unfiltered reconstruction when its step comes and is
// final — no later MB writes it — two steps later, when it is scored
// against the source (or written back) and its slot reused. The picture
// therefore crosses HBM once per candidate (all CTAs read the same
// reconstruction, which stays L2-resident), and no candidate copy of the
// planes is ever materialised. Within an MB a lane owns one pixel row for
// the four vertical edges, then one pixel column for the four horizontal
// edges (luma lanes 0-15, U 16-23, V 24-31), matching the reference's
// step order (left MB edge, inner vertical, top MB edge, inner horizontal).
// The sampled search's two-row bands are rows whose t0 restarts at 0 and
// whose first row has no top edge.
#include <algorithm>
#include <mutex>

#include "vp8a_internal.cuh"

namespace {
using namespace vp8a_dev;
constexpr unsigned FULL = 0xffffffffu;
// An MB slot holds Y 16x16 + U 8x8 + V 8x8 = 384 bytes, padded to 400 so
// that the slots of neighbouring rows start on different banks.
constexpr int SLOT_STRIDE = 400;
// Slots per MB row: MB (r, c) takes slot c % 3 once MB (r, c - 3) is final
// (its last writer, MB (r + 1, c - 3), ran the step before) and scored.
// While MB (r, c) runs, row r - 1 runs (r - 1, c + 2) and row r + 1 runs
// (r + 1, c - 2): the slots they touch are never the one being refilled.
constexpr int RING = 3;

struct LfArgs {
  const uint8_t* y;
  const uint8_t* u;
  const uint8_t* v;
  uint64_t ys, cs;
  int mb_cols, mb_rows;
  const vp8a_mb_lf_info* mbs;
  vp8a_filter_config base;
  const uint8_t* sy;
  const uint8_t* su;
  const uint8_t* sv;
  uint64_t sys, scs;
  int width, height;
  const uint8_t* cands;    // [n][2] (level, sharpness)
  // [n] or null: the sharpness values whose table entries candidate i's
  // SSD fills (bit s = level * 8 + s), null = its own sharpness only.
  const uint8_t* cand_mask;
  const int16_t* row_t0;   // per MB row: first step, -1 = row not scored
  const uint8_t* row_top;  // per MB row: has a top MB edge
  int steps;
  const int32_t* sched_off;  // [steps + 1]: rows active at step t are
  const uint16_t* sched_row; //   sched_row[sched_off[t] .. sched_off[t + 1])
  int max_active;            // most rows active at one step
  // Ring sets: row r keeps its slots in set row_set[r] (rows whose slot
  // lifetimes do not overlap share a set; n_sets sets). Its last RING MBs
  // are scored at the step where they are final: the rows listed in
  // fin_row[fin_off[t] .. fin_off[t + 1]) at step t. Null row_set: set r
  // for row r, tails scored after the last step.
  const uint16_t* row_set;
  const int32_t* fin_off;
  const uint16_t* fin_row;
  int n_sets;
  int recon_words;           // planes and strides allow 4-byte accesses
  int source_words;
  int recon_vec;   // luma rows allow 16-byte and chroma rows 8-byte loads
  int source_vec;
  // Next-step prefetch: each half-warp copies its next MB's reconstruction,
  // source rows and MB record into its own staging area (dynamic shared
  // memory at byte stage_off) while the current step runs (cp.async).
  int prefetch;
  int stage_off;
  int n_cands;    // candidates in `cands`; a CTA takes NC consecutive ones
  int ring_bytes; // one candidate's slot rings
  uint64_t* ssd_out;  // [64 * 8], indexed level * 8 + sharpness
  uint8_t* oy;        // write-back planes (apply mode) or null
  uint8_t* ou;
  uint8_t* ov;
  uint8_t* gslots;  // global slot storage when shared memory is too small
  int smem_slots;
  // Sweep mode: a level-0 candidate scores the unfiltered planes
  // (score_filter_candidate's short cut, src/loop_filter.rs:2071). Apply
  // mode runs the pass with the base level as given, since per-MB
  // segment overrides and deltas can still filter MBs at base level 0.
  int level0_unfiltered;
};

__device__ __forceinline__ int c8(int v) { return min(max(v, -128), 127); }
__device__ __forceinline__ int iabs(int v) { return v < 0 ? -v : v; }

// LoopFilterParams::derive (src/loop_filter.rs:99-148).
struct Prm {
  int interior, hev, mbedge, subedge;
};
__device__ __forceinline__ Prm derive(int level, int sharp, bool key) {
  int interior = level;
  if (sharp != 0) {
    interior >>= (sharp > 4) ? 2 : 1;
    int cap = max(9 - sharp, 0);
    if (interior > cap) interior = cap;
  }
  if (interior == 0) interior = 1;
  int hev = key ? (level >= 40 ? 2 : (level >= 15 ? 1 : 0))
                : (level >= 40 ? 3 : (level >= 20 ? 2 : (level >= 15 ? 1 : 0)));
  Prm p;
  p.interior = interior;
  p.hev = hev;
  p.mbedge = min((level + 2) * 2 + interior, 255);
  p.subedge = min(level * 2 + interior, 255);
  return p;
}

__host__ __device__ __forceinline__ int clamp63(int v) { return v < 0 ? 0 : (v > 63 ? 63 : v); }

// calculate_mb_filter_level_inter (src/loop_filter.rs:1280-1331).
__host__ __device__ __forceinline__ int mb_level(const vp8a_filter_config& c, int level0, const vp8a_mb_lf_info& m) {
  int level = level0;
  if (c.segmentation_enabled) {
    int seg = m.segment_id < 0 ? 0 : (m.segment_id > 3 ? 3 : (int)m.segment_id);
    if (c.segment_abs) level = c.segment_lf_level[seg];
    else level += c.segment_lf_level[seg];
  }
  level = clamp63(level);
  if (c.delta_enabled) {
    int rd = m.ref_frame == VP8A_REF_LAST     ? c.ref_delta_last
             : m.ref_frame == VP8A_REF_GOLDEN ? c.ref_delta_golden
             : m.ref_frame == VP8A_REF_ALTREF ? c.ref_delta_altref
                                              : c.ref_delta_current;
    level += rd;
    if (m.ref_frame == VP8A_REF_INTRA) {
      if (m.y_mode_is_bpred) level += c.bpred_mode_delta;
    } else if (m.inter_mode == VP8A_MODE_ZERO) {
      level += c.zero_mv_mode_delta;
    } else if (m.inter_mode == VP8A_MODE_SPLIT) {
      level += c.split_mv_mode_delta;
    } else {
      level += c.other_mv_mode_delta;
    }
  }
  return clamp63(level);
}

// LoopFilterParams::derive's interior limit (src/loop_filter.rs:99-148):
// with the level, it fixes every parameter of the §15 filters.
__host__ __device__ __forceinline__ int interior_limit(int level, int sharp) {
  int interior = level;
  if (sharp != 0) {
    interior >>= (sharp > 4) ? 2 : 1;
    const int cap = 9 - sharp > 0 ? 9 - sharp : 0;
    if (interior > cap) interior = cap;
  }
  return interior == 0 ? 1 : interior;
}

// The filters below work on unsigned pixels (0..255): the reference's
// signed taps are pixel - 128, every difference is the same, and
// c8(x_signed + a) + 128 == u8c(x_unsigned + a). Both outcomes of each
// per-segment test are formed and selected, so lanes never diverge.
__device__ __forceinline__ int u8c(int v) { return min(max(v, 0), 255); }

// §15.3 MBfilter (src/loop_filter.rs:331-371) on taps p[O..O+8).
template <int O, int N>
__device__ __forceinline__ void mb_filter(int (&p)[N], const Prm& q) {
  const int p3 = p[O], p2 = p[O + 1], p1 = p[O + 2], p0 = p[O + 3];
  const int q0 = p[O + 4], q1 = p[O + 5], q2 = p[O + 6], q3 = p[O + 7];
  const int inner = max(iabs(p1 - p0), iabs(q1 - q0));
  const int flat = max(max(iabs(p3 - p2), iabs(p2 - p1)), max(max(iabs(q3 - q2), iabs(q2 - q1)), inner));
  const bool yes = (iabs(p0 - q0) * 2 + (iabs(p1 - q1) >> 1)) <= q.mbedge && flat <= q.interior;
  const bool hv = inner > q.hev;
  const int w = c8(c8(p1 - q1) + 3 * (q0 - p0));
  const int a27 = c8((27 * w + 63) >> 7), a18 = c8((18 * w + 63) >> 7), a9 = c8((9 * w + 63) >> 7);
  const int aq = hv ? c8(w + 4) >> 3 : a27, ap = hv ? c8(w + 3) >> 3 : a27;
  const bool wide = yes && !hv;
  p[O + 4] = yes ? u8c(q0 - aq) : q0;
  p[O + 3] = yes ? u8c(p0 + ap) : p0;
  p[O + 5] = wide ? u8c(q1 - a18) : q1;
  p[O + 2] = wide ? u8c(p1 + a18) : p1;
  p[O + 6] = wide ? u8c(q2 - a9) : q2;
  p[O + 1] = wide ? u8c(p2 + a9) : p2;
}

// §15.3 subblock_filter (src/loop_filter.rs:292-318).
template <int O, int N>
__device__ __forceinline__ void sb_filter(int (&p)[N], const Prm& q) {
  const int p3 = p[O], p2 = p[O + 1], p1 = p[O + 2], p0 = p[O + 3];
  const int q0 = p[O + 4], q1 = p[O + 5], q2 = p[O + 6], q3 = p[O + 7];
  const int inner = max(iabs(p1 - p0), iabs(q1 - q0));
  const int flat = max(max(iabs(p3 - p2), iabs(p2 - p1)), max(max(iabs(q3 - q2), iabs(q2 - q1)), inner));
  const bool yes = (iabs(p0 - q0) * 2 + (iabs(p1 - q1) >> 1)) <= q.subedge && flat <= q.interior;
  const bool hv = inner > q.hev;
  int a = c8((hv ? c8(p1 - q1) : 0) + 3 * (q0 - p0));
  const int b = c8(a + 3) >> 3;
  a = c8(a + 4) >> 3;
  const int a2 = (a + 1) >> 1;
  const bool wide = yes && !hv;
  p[O + 4] = yes ? u8c(q0 - a) : q0;
  p[O + 3] = yes ? u8c(p0 + b) : p0;
  p[O + 5] = wide ? u8c(q1 - a2) : q1;
  p[O + 2] = wide ? u8c(p1 + a2) : p1;
}

// §15.2 simple_segment (src/loop_filter.rs:235-247).
template <int O, int N>
__device__ __forceinline__ void simple_filter(int (&p)[N], int edge) {
  const int p1 = p[O], p0 = p[O + 1], q0 = p[O + 2], q1 = p[O + 3];
  const bool yes = iabs(p0 - q0) * 2 + (iabs(p1 - q1) >> 1) <= edge;
  int a = c8(c8(p1 - q1) + 3 * (q0 - p0));
  const int b = c8(a + 3) >> 3;
  a = c8(a + 4) >> 3;
  p[O + 2] = yes ? u8c(q0 - a) : q0;
  p[O + 1] = yes ? u8c(p0 + b) : p0;
}

__device__ __forceinline__ void unpack4(uint32_t w, int* o) {
#pragma unroll
  for (int k = 0; k < 4; k++) o[k] = (int)((w >> (8 * k)) & 0xffu);
}
__device__ __forceinline__ uint32_t pack4(const int* o) {
  return (uint32_t)o[0] | ((uint32_t)o[1] << 8) | ((uint32_t)o[2] << 16) | ((uint32_t)o[3] << 24);
}

// Slot of column c of the row using ring set `set`.
__device__ __forceinline__ uint8_t* slot_ptr(uint8_t* slots, int set, int c) {
  return slots + ((size_t)set * RING + c % RING) * SLOT_STRIDE;
}

// One half-warp handles one MB: lane l (0-15) owns luma row l and chroma
// row l & 7 of U (l < 8) or V (l >= 8) for the vertical edges, then the
// same-numbered columns for the horizontal edges, so luma and chroma run on
// the same instructions.
struct MbWords {
  uint32_t y[4], c[2];
};

// This lane's 24 bytes of MB (r, c) of the unfiltered reconstruction.
__device__ __forceinline__ MbWords fetch_recon(const LfArgs& a, int r, int c, int l) {
  MbWords w;
  const uint8_t* gy = a.y + (size_t)(r * 16 + l) * a.ys + (size_t)c * 16;
  const uint8_t* gc = (l < 8 ? a.u : a.v) + (size_t)(r * 8 + (l & 7)) * a.cs + (size_t)c * 8;
  if (a.recon_vec) {
    // Plain loads: apply mode writes final MBs back into these planes.
    const uint4 y4 = *(const uint4*)gy;
    const uint2 c2 = *(const uint2*)gc;
    w.y[0] = y4.x;
    w.y[1] = y4.y;
    w.y[2] = y4.z;
    w.y[3] = y4.w;
    w.c[0] = c2.x;
    w.c[1] = c2.y;
  } else if (a.recon_words) {
#pragma unroll
    for (int k = 0; k < 4; k++) w.y[k] = ((const uint32_t*)gy)[k];
    w.c[0] = ((const uint32_t*)gc)[0];
    w.c[1] = ((const uint32_t*)gc)[1];
  } else {
#pragma unroll
    for (int k = 0; k < 4; k++)
      w.y[k] = (uint32_t)gy[4 * k] | ((uint32_t)gy[4 * k + 1] << 8) | ((uint32_t)gy[4 * k + 2] << 16) |
               ((uint32_t)gy[4 * k + 3] << 24);
#pragma unroll
    for (int k = 0; k < 2; k++)
      w.c[k] = (uint32_t)gc[4 * k] | ((uint32_t)gc[4 * k + 1] << 8) | ((uint32_t)gc[4 * k + 2] << 16) |
               ((uint32_t)gc[4 * k + 3] << 24);
  }
  return w;
}

__device__ __forceinline__ void store_slot(uint8_t* s, const MbWords& w, int l) {
  uint32_t* sy = (uint32_t*)(s + l * 16);
#pragma unroll
  for (int k = 0; k < 4; k++) sy[k] = w.y[k];
  uint32_t* sc = (uint32_t*)(s + (l < 8 ? 256 : 320) + (l & 7) * 8);
  sc[0] = w.c[0];
  sc[1] = w.c[1];
}

// The source under this lane's rows of MB (r, c), restricted to the
// visible window: bytes outside it read as 0 and their mask bytes are 0.
struct SrcWords {
  uint32_t y[4], c[2], my[4], mc[2];
};

__device__ __forceinline__ uint32_t vis_mask(int n, int k) {
  const int v = n - 4 * k;
  return v >= 4 ? 0xffffffffu : (v <= 0 ? 0u : (1u << (8 * v)) - 1u);
}

__device__ __forceinline__ SrcWords fetch_source(const LfArgs& a, int r, int c, int l) {
  SrcWords w;
  const int yy = r * 16 + l, x0 = c * 16;
  const int ny = yy < a.height ? clampi(a.width - x0, 0, 16) : 0;
  const int cw = (a.width + 1) >> 1, ch = (a.height + 1) >> 1;
  const int cy = r * 8 + (l & 7), cx0 = c * 8;
  const int nc = cy < ch ? clampi(cw - cx0, 0, 8) : 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    w.my[k] = vis_mask(ny, k);
    w.y[k] = 0;
  }
#pragma unroll
  for (int k = 0; k < 2; k++) {
    w.mc[k] = vis_mask(nc, k);
    w.c[k] = 0;
  }
  if (ny > 0) {
    const uint8_t* p = a.sy + (size_t)yy * a.sys + x0;
    if (ny == 16 && a.source_vec) {
      const uint4 v = __ldg((const uint4*)p);
      w.y[0] = v.x;
      w.y[1] = v.y;
      w.y[2] = v.z;
      w.y[3] = v.w;
    } else if (ny == 16 && a.source_words) {
#pragma unroll
      for (int k = 0; k < 4; k++) w.y[k] = ((const uint32_t*)p)[k];
    } else {
#pragma unroll
      for (int i = 0; i < 16; i++)
        if (i < ny) w.y[i >> 2] |= (uint32_t)p[i] << (8 * (i & 3));
    }
  }
  if (nc > 0) {
    const uint8_t* p = (l < 8 ? a.su : a.sv) + (size_t)cy * a.scs + cx0;
    if (nc == 8 && a.source_vec) {
      const uint2 v = __ldg((const uint2*)p);
      w.c[0] = v.x;
      w.c[1] = v.y;
    } else if (nc == 8 && a.source_words) {
      w.c[0] = ((const uint32_t*)p)[0];
      w.c[1] = ((const uint32_t*)p)[1];
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++)
        if (i < nc) w.c[i >> 2] |= (uint32_t)p[i] << (8 * (i & 3));
    }
  }
  return w;
}

// Sum of squared differences of four byte pairs, masked bytes excluded.
__device__ __forceinline__ uint32_t ssd4(uint32_t x, uint32_t y, uint32_t m) {
  const uint32_t d = __vabsdiffu4(x, y) & m;
  return (uint32_t)__dp4a(d, d, 0u);
}

// Finish final MB (r, c): write it back (apply mode) and return this lane's
// share of its visible-window SSD.
__device__ __forceinline__ uint32_t finish_mb(const LfArgs& a, const uint8_t* slots, int set, int r, int c, int l,
                                              const SrcWords& sw) {
  const uint8_t* s = slot_ptr(const_cast<uint8_t*>(slots), set, c);
  const uint32_t* sy = (const uint32_t*)(s + l * 16);
  const uint32_t* sc = (const uint32_t*)(s + (l < 8 ? 256 : 320) + (l & 7) * 8);
  if (a.oy) {
    uint8_t* gy = a.oy + (size_t)(r * 16 + l) * a.ys + (size_t)c * 16;
    uint8_t* gc = (l < 8 ? a.ou : a.ov) + (size_t)(r * 8 + (l & 7)) * a.cs + (size_t)c * 8;
    if (a.recon_words) {
#pragma unroll
      for (int k = 0; k < 4; k++) ((uint32_t*)gy)[k] = sy[k];
      ((uint32_t*)gc)[0] = sc[0];
      ((uint32_t*)gc)[1] = sc[1];
    } else {
      for (int i = 0; i < 16; i++) gy[i] = s[l * 16 + i];
      for (int i = 0; i < 8; i++) gc[i] = s[(l < 8 ? 256 : 320) + (l & 7) * 8 + i];
    }
  }
  uint32_t acc = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) acc += ssd4(sy[k], sw.y[k], sw.my[k]);
  acc += ssd4(sc[0], sw.c[0], sw.mc[0]) + ssd4(sc[1], sw.c[1], sw.mc[1]);
  return acc;
}

// Filter MB (r, c) held in its slot; neighbours in their slots. The
// caller's half-warp (mask hm) runs this together.
__device__ __forceinline__ void filter_mb(const LfArgs& a, const Prm* prm, const vp8a_mb_lf_info m, uint8_t* slots,
                                          int level0, int set, int set_above, int c, bool has_top, int l,
                                          unsigned hm) {
  const int level = mb_level(a.base, level0, m);
  if (level == 0) return;
  const Prm q = prm[level];
  const bool sub = m.y_mode_is_bpred || m.has_coeffs;
  const bool has_left = c > 0;
  uint8_t* me = slot_ptr(slots, set, c);
  uint8_t* left = slot_ptr(slots, set, c - 1);
  uint8_t* above = has_top ? slot_ptr(slots, set_above, c) : nullptr;

  if (a.base.simple) {
    // §20.6 filter_row_simple: luma only.
    {
      uint32_t* rw = (uint32_t*)(me + l * 16);
      int p[20];
      unpack4(has_left ? *(const uint32_t*)(left + l * 16 + 12) : 0x80808080u, p);
#pragma unroll
      for (int k = 0; k < 4; k++) unpack4(rw[k], p + 4 + 4 * k);
      if (has_left) simple_filter<2>(p, q.mbedge);
      if (sub) {
        simple_filter<6>(p, q.subedge);
        simple_filter<10>(p, q.subedge);
        simple_filter<14>(p, q.subedge);
      }
      if (has_left) *(uint32_t*)(left + l * 16 + 12) = pack4(p);
#pragma unroll
      for (int k = 0; k < 4; k++) rw[k] = pack4(p + 4 + 4 * k);
    }
    __syncwarp(hm);
    {
      int p[20];
#pragma unroll
      for (int k = 0; k < 4; k++) p[k] = has_top ? (int)above[(12 + k) * 16 + l] : 0;
#pragma unroll
      for (int k = 0; k < 16; k++) p[4 + k] = (int)me[k * 16 + l];
      if (has_top) simple_filter<2>(p, q.mbedge);
      if (sub) {
        simple_filter<6>(p, q.subedge);
        simple_filter<10>(p, q.subedge);
        simple_filter<14>(p, q.subedge);
      }
      if (has_top)
#pragma unroll
        for (int k = 2; k < 4; k++) above[(12 + k) * 16 + l] = (uint8_t)(p[k]);
#pragma unroll
      for (int k = 0; k < 16; k++) me[k * 16 + l] = (uint8_t)(p[4 + k]);
    }
    __syncwarp(hm);
    return;
  }

  const int pl = l < 8 ? 256 : 320, cl = l & 7;  // this lane's chroma plane offset and row/column
  // MBs without inner edges (no coefficients, not B_PRED) filter only their
  // left and top MB edges: eight taps per lane and direction. When no MB of
  // the warp's converged lanes has inner edges, the warp takes that narrow
  // path (both half-warps run the same instructions); otherwise every MB
  // runs the full rows and columns below, filtering inner edges only where
  // it has them.
  if (__ballot_sync(__activemask(), sub) == 0u) {
    if (has_left) {
      int p[8];
      uint32_t* lw = (uint32_t*)(left + l * 16 + 12);
      uint32_t* rw = (uint32_t*)(me + l * 16);
      unpack4(*lw, p);
      unpack4(*rw, p + 4);
      mb_filter<0>(p, q);
      *lw = pack4(p);
      *rw = pack4(p + 4);
      uint32_t* lc = (uint32_t*)(left + pl + cl * 8 + 4);
      uint32_t* rc = (uint32_t*)(me + pl + cl * 8);
      unpack4(*lc, p);
      unpack4(*rc, p + 4);
      mb_filter<0>(p, q);
      *lc = pack4(p);
      *rc = pack4(p + 4);
    }
    __syncwarp(hm);
    if (has_top) {
      // The last four rows of the MB above and the first four here; the
      // filter changes the last three above and the first three here.
      int p[8];
#pragma unroll
      for (int k = 0; k < 4; k++) p[k] = (int)above[(12 + k) * 16 + l];
#pragma unroll
      for (int k = 0; k < 4; k++) p[4 + k] = (int)me[k * 16 + l];
      mb_filter<0>(p, q);
#pragma unroll
      for (int k = 1; k < 4; k++) above[(12 + k) * 16 + l] = (uint8_t)p[k];
#pragma unroll
      for (int k = 0; k < 3; k++) me[k * 16 + l] = (uint8_t)p[4 + k];
#pragma unroll
      for (int k = 0; k < 4; k++) p[k] = (int)above[pl + (4 + k) * 8 + cl];
#pragma unroll
      for (int k = 0; k < 4; k++) p[4 + k] = (int)me[pl + k * 8 + cl];
      mb_filter<0>(p, q);
#pragma unroll
      for (int k = 1; k < 4; k++) above[pl + (4 + k) * 8 + cl] = (uint8_t)p[k];
#pragma unroll
      for (int k = 0; k < 3; k++) me[pl + k * 8 + cl] = (uint8_t)p[4 + k];
    }
    __syncwarp(hm);
    return;
  }
  // ---- vertical edges (steps 1 and 2): luma row l, then chroma row cl ----
  {
    uint32_t* rw = (uint32_t*)(me + l * 16);
    int p[20];
    unpack4(has_left ? *(const uint32_t*)(left + l * 16 + 12) : 0x80808080u, p);
#pragma unroll
    for (int k = 0; k < 4; k++) unpack4(rw[k], p + 4 + 4 * k);
    if (has_left) mb_filter<0>(p, q);
    if (sub) {
      sb_filter<4>(p, q);
      sb_filter<8>(p, q);
      sb_filter<12>(p, q);
    }
    if (has_left) *(uint32_t*)(left + l * 16 + 12) = pack4(p);
#pragma unroll
    for (int k = 0; k < 4; k++) rw[k] = pack4(p + 4 + 4 * k);
  }
  {
    uint32_t* rw = (uint32_t*)(me + pl + cl * 8);
    int p[12];
    unpack4(has_left ? *(const uint32_t*)(left + pl + cl * 8 + 4) : 0x80808080u, p);
    unpack4(rw[0], p + 4);
    unpack4(rw[1], p + 8);
    if (has_left) mb_filter<0>(p, q);
    if (sub) sb_filter<4>(p, q);
    if (has_left) *(uint32_t*)(left + pl + cl * 8 + 4) = pack4(p);
    rw[0] = pack4(p + 4);
    rw[1] = pack4(p + 8);
  }
  __syncwarp(hm);
  // ---- horizontal edges (steps 3 and 4): luma column l, chroma column cl ----
  {
    int p[20];
#pragma unroll
    for (int k = 0; k < 4; k++) p[k] = has_top ? (int)above[(12 + k) * 16 + l] : 0;
#pragma unroll
    for (int k = 0; k < 16; k++) p[4 + k] = (int)me[k * 16 + l];
    if (has_top) mb_filter<0>(p, q);
    if (sub) {
      sb_filter<4>(p, q);
      sb_filter<8>(p, q);
      sb_filter<12>(p, q);
    }
    if (has_top)
#pragma unroll
      for (int k = 1; k < 4; k++) above[(12 + k) * 16 + l] = (uint8_t)(p[k]);
#pragma unroll
    for (int k = 0; k < 16; k++) me[k * 16 + l] = (uint8_t)(p[4 + k]);
  }
  {
    int p[12];
#pragma unroll
    for (int k = 0; k < 4; k++) p[k] = has_top ? (int)above[pl + (4 + k) * 8 + cl] : 0;
#pragma unroll
    for (int k = 0; k < 8; k++) p[4 + k] = (int)me[pl + k * 8 + cl];
    if (has_top) mb_filter<0>(p, q);
    if (sub) sb_filter<4>(p, q);
    if (has_top)
#pragma unroll
      for (int k = 1; k < 4; k++) above[pl + (4 + k) * 8 + cl] = (uint8_t)(p[k]);
#pragma unroll
    for (int k = 0; k < 8; k++) me[pl + k * 8 + cl] = (uint8_t)(p[4 + k]);
  }
  __syncwarp(hm);
}

// A half-warp's staged next MB.
struct __align__(16) Stage {
  uint8_t rec[384];  // Y rows 0-15, U rows 0-7, V rows 0-7 (slot layout)
  uint8_t src[384];  // the source under the MB the step finishes, same layout
  vp8a_mb_lf_info info;
  uint8_t pad[8];
};
static_assert(sizeof(Stage) % 16 == 0, "Stage keeps 16-byte copies aligned");

__device__ __forceinline__ void cp_async(void* smem, const void* g, int bytes, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes == 16)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(g), "r"(src_bytes) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(g), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Start copying MB (r, c)'s inputs into `g`: lane l copies luma row l and
// chroma row l & 7 of U (l < 8) or V of the reconstruction, the same rows of
// the source under MB (r, c - 3) when one is finished with it (bytes outside
// the visible window are filled with zeros, never read), and lane 0 the MB
// record.
__device__ __forceinline__ void prefetch_mb(const LfArgs& a, Stage* g, int r, int c, int l, bool score) {
  cp_async(g->rec + l * 16, a.y + (size_t)(r * 16 + l) * a.ys + (size_t)c * 16, 16, 16);
  const int pl = l < 8 ? 256 : 320, cr = l & 7;
  cp_async(g->rec + pl + cr * 8, (l < 8 ? a.u : a.v) + (size_t)(r * 8 + cr) * a.cs + (size_t)c * 8, 8, 8);
  if (score && c >= RING) {
    const int yy = r * 16 + l, x0 = (c - RING) * 16;
    const int ny = yy < a.height ? clampi(a.width - x0, 0, 16) : 0;
    cp_async(g->src + l * 16, ny > 0 ? (const void*)(a.sy + (size_t)yy * a.sys + x0) : (const void*)a.sy, 16, ny);
    const int cw = (a.width + 1) >> 1, ch = (a.height + 1) >> 1, cy = r * 8 + cr, cx0 = (c - RING) * 8;
    const int nc = cy < ch ? clampi(cw - cx0, 0, 8) : 0;
    const uint8_t* sp = l < 8 ? a.su : a.sv;
    cp_async(g->src + pl + cr * 8, nc > 0 ? (const void*)(sp + (size_t)cy * a.scs + cx0) : (const void*)sp, 8, nc);
  }
  if (l == 0) cp_async(&g->info, a.mbs + (size_t)r * a.mb_cols + c, 8, 8);
  cp_async_commit();
}


// One CTA per candidate. At step t the MBs of the rows listed in
// sched_row[sched_off[t] .. sched_off[t+1]) are independent; half-warp h
// takes the h-th, (h + H)-th, ... of them. Per MB the global fetches (its
// reconstruction and the source under the MB finished in its slot) are
// issued together before the slot is touched.
// SSD totals of the CTA's candidates into the table.
// A sweep-mode level-0 candidate's SSD is stored for every sharpness
// (level 0 scores the unfiltered planes whatever the sharpness).
template <int NC>
__device__ __forceinline__ void block_sums_store(const uint64_t (&v)[NC], const LfArgs& a, const int (&lv)[NC],
                                                 const int (&mk)[NC], int nc) {
  __shared__ unsigned long long red[NC][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NC; k++) {
    uint64_t x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
    if (lane == 0) red[k][warp] = x;
  }
  __syncthreads();
  const int nwarps = (int)(blockDim.x >> 5);
  for (int k = warp; k < nc; k += nwarps) {
    uint64_t x = lane < nwarps ? red[k][lane] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
    if (lane < 8 && ((mk[k] >> lane) & 1)) a.ssd_out[lv[k] * 8 + lane] = x;
  }
}

// NC candidates per CTA over one step schedule: the MB inputs are fetched
// (or prefetched) once and each candidate filters them in its own slot
// rings. A sweep-mode level-0 candidate is not filtered at all: it scores
// the unfiltered reconstruction (score_filter_candidate's short cut,
// src/loop_filter.rs:2071).
template <int NC>
__device__ __forceinline__ void sweep_body(const LfArgs& a, int cta) {
  extern __shared__ __align__(16) uint8_t smem_slots[];
  const int hw = threadIdx.x >> 4, nhw = blockDim.x >> 4, l = threadIdx.x & 15;
  const unsigned hm = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  const int first = cta * NC, nc = min(NC, a.n_cands - first);
  int lv[NC], sh[NC], mk[NC];
  bool filt[NC];
  uint64_t acc[NC];
  uint8_t* slots[NC];
  __shared__ Prm prm[NC][64];
#pragma unroll
  for (int k = 0; k < NC; k++) {
    const int q = first + min(k, nc - 1);
    lv[k] = a.cands[2 * q];
    sh[k] = a.cands[2 * q + 1];
    // A sweep-mode level-0 candidate scores the unfiltered planes, the same
    // for every sharpness.
    mk[k] = (lv[k] == 0 && a.level0_unfiltered) ? 0xff : (a.cand_mask ? a.cand_mask[q] : 1 << sh[k]);
    filt[k] = k < nc && !(lv[k] == 0 && a.level0_unfiltered);
    acc[k] = 0;
    slots[k] = (a.smem_slots ? smem_slots : a.gslots + (size_t)first * a.ring_bytes) + (size_t)k * a.ring_bytes;
    // LoopFilterParams::derive for every level at this candidate's sharpness.
    for (int i = threadIdx.x; i < 64; i += blockDim.x) prm[k][i] = derive(i, sh[k], a.base.key_frame != 0);
  }
  const bool score = a.ssd_out != nullptr;
  __syncthreads();
  Stage* stage = a.prefetch ? (Stage*)(smem_slots + a.stage_off) + hw : nullptr;
  // MB (r, c) of every candidate: its inputs come from the half-warp's
  // staging area (`from_stage`, then `next()` may refill it) or straight
  // from global memory; the MB three columns back leaves its slot scored,
  // MB (r, c) takes the slot and is filtered.
  auto set_of = [&](int r) -> int { return a.row_set ? (int)a.row_set[r] : r; };
  auto do_mb = [&](int r, int c, bool from_stage, auto&& next) {
    const int set = set_of(r), set_above = (a.row_top[r] != 0) ? set_of(r - 1) : 0;
    MbWords rec;
    SrcWords sw{};
    vp8a_mb_lf_info m;
    if (from_stage) {
      cp_async_wait_all();
      __syncwarp(hm);
      const uint32_t* ry = (const uint32_t*)(stage->rec + l * 16);
      const uint32_t* rc = (const uint32_t*)(stage->rec + (l < 8 ? 256 : 320) + (l & 7) * 8);
#pragma unroll
      for (int k = 0; k < 4; k++) rec.y[k] = ry[k];
      rec.c[0] = rc[0];
      rec.c[1] = rc[1];
      if (score && c >= RING) {
        const uint32_t* sy = (const uint32_t*)(stage->src + l * 16);
        const uint32_t* sc = (const uint32_t*)(stage->src + (l < 8 ? 256 : 320) + (l & 7) * 8);
        const int ny = r * 16 + l < a.height ? clampi(a.width - (c - RING) * 16, 0, 16) : 0;
        const int cw = (a.width + 1) >> 1, ch = (a.height + 1) >> 1;
        const int ncv = r * 8 + (l & 7) < ch ? clampi(cw - (c - RING) * 8, 0, 8) : 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
          sw.y[k] = sy[k];
          sw.my[k] = vis_mask(ny, k);
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
          sw.c[k] = sc[k];
          sw.mc[k] = vis_mask(ncv, k);
        }
      }
      m = stage->info;
      __syncwarp(hm);
      // The staging area is free again: start the next MB's copies.
      next();
    } else {
      rec = fetch_recon(a, r, c, l);
      if (score && c >= RING) sw = fetch_source(a, r, c - RING, l);
      m = a.mbs[(size_t)r * a.mb_cols + c];
    }
#pragma unroll
    for (int k = 0; k < NC; k++) {
      if (k >= nc) break;
      if (c >= RING) {
        acc[k] += finish_mb(a, slots[k], set, r, c - RING, l, sw);
        __syncwarp(hm);
      }
      store_slot(slot_ptr(slots[k], set, c), rec, l);
    }
    __syncwarp(hm);
#pragma unroll
    for (int k = 0; k < NC; k++)
      if (filt[k]) filter_mb(a, prm[k], m, slots[k], lv[k], set, set_above, c, a.row_top[r] != 0, l, hm);
  };
  // The half-warp's first MB of step t, or -1.
  auto first_mb = [&](int t) -> int {
    if (t >= a.steps) return -1;
    const int i = a.sched_off[t] + hw;
    return i < a.sched_off[t + 1] ? i : -1;
  };
  auto issue = [&](int t) -> bool {
    const int j = first_mb(t);
    if (j < 0) return false;
    const int r2 = a.sched_row[j];
    prefetch_mb(a, stage, r2, t - a.row_t0[r2], l, score);
    return true;
  };
  bool staged = a.prefetch ? issue(0) : false;
  for (int t = 0; t < a.steps; t++) {
    const int b = a.sched_off[t], e = a.sched_off[t + 1];
    bool next_issued = false;
    for (int i = b + hw; i < e; i += nhw) {
      const int r = a.sched_row[i], c = t - a.row_t0[r];
      const bool from_stage = staged && i == b + hw;
      do_mb(r, c, from_stage, [&] {
        staged = a.prefetch && issue(t + 1);
        next_issued = true;
      });
    }
    if (a.prefetch && !next_issued) staged = issue(t + 1);
    if (a.row_set) {
      // Rows whose last MBs became final with the previous step.
      const int fb = a.fin_off[t] * RING, fe = a.fin_off[t + 1] * RING;
      for (int j = fb + hw; j < fe; j += nhw) {
        const int r = a.fin_row[j / RING], c = a.mb_cols - RING + j % RING;
        if (c < 0) continue;
        const SrcWords sw = score ? fetch_source(a, r, c, l) : SrcWords{};
        const int set = set_of(r);
#pragma unroll
        for (int k = 0; k < NC; k++)
          if (k < nc) acc[k] += finish_mb(a, slots[k], set, r, c, l, sw);
      }
    }
    __syncthreads();
  }
  // Without a tail schedule: the last MBs of every scored row.
  for (int i = hw; !a.row_set && i < a.mb_rows * RING; i += nhw) {
    const int r = i / RING, c = a.mb_cols - RING + i % RING;
    if (c < 0 || a.row_t0[r] < 0) continue;
    const SrcWords sw = score ? fetch_source(a, r, c, l) : SrcWords{};
#pragma unroll
    for (int k = 0; k < NC; k++)
      if (k < nc) acc[k] += finish_mb(a, slots[k], r, r, c, l, sw);
  }
  if (score) block_sums_store<NC>(acc, a, lv, mk, nc);
}

template <int NC>
__global__ void __launch_bounds__(1024) lf_sweep_kernel(LfArgs a) {
  sweep_body<NC>(a, blockIdx.x);
}

// Many pictures' sweeps in one launch: CTA offsets per job as in find_job.
template <int NC>
__global__ void __launch_bounds__(1024)
    lf_sweep_batch_kernel(const LfArgs* __restrict__ jobs, const uint32_t* __restrict__ cta_start, int n_jobs) {
  __shared__ LfArgs sa;
  __shared__ uint32_t first[2];
  find_job(jobs, cta_start, n_jobs, &sa, first);
  sweep_body<NC>(sa, (int)(blockIdx.x - first[0]));
}

// Plain visible-window SSD of a reconstruction (reconstruction_ssd).
__global__ void __launch_bounds__(256) ssd_kernel(const uint8_t* rec, uint64_t rs, const uint8_t* src, uint64_t ss,
                                                  int w, int h, unsigned long long* out) {
  uint64_t acc = 0;
  const size_t n = (size_t)w * h;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    int y = (int)(i / w), x = (int)(i % w);
    int d = (int)rec[(size_t)y * rs + x] - (int)src[(size_t)y * ss + x];
    acc += (uint64_t)(d * d);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(FULL, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, (unsigned long long)acc);
}

// ------------------------------------------------------------------- host

struct LfInputs {
  LfArgs a{};
  int max_steps = 0;
};

vp8a_status validate_config(const vp8a_filter_config* c) {
  if (c->loop_filter_level > 63) {
    vp8a::set_error("loop_filter_level > 63");
    return VP8A_E_LOOP_FILTER_LEVEL_OUT_OF_RANGE;
  }
  if (c->sharpness_level > 7) {
    vp8a::set_error("sharpness_level > 7");
    return VP8A_E_SHARPNESS_LEVEL_OUT_OF_RANGE;
  }
  return VP8A_OK;
}

// Stages planes, per-MB info and (optionally) the source; fills the row
// schedule for whole frames (every_rows = 0) or sampled bands.
vp8a_status stage_lf(vp8a_ctx* ctx, vp8a::Stager& st, const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                     const vp8a_filter_config* base, const vp8a_source* src, uint32_t every_rows, bool write_back,
                     LfInputs* L) {
  if (!planes || !mbs || !base) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (planes->mb_cols == 0 || planes->mb_rows == 0 || planes->mb_cols > 1024 || planes->mb_rows > 1024) {
    vp8a::set_error("plane MB grid out of range");
    return VP8A_E_INVALID_DIMENSIONS;
  }
  if (planes->y_stride < (uint64_t)planes->mb_cols * 16 || planes->uv_stride < (uint64_t)planes->mb_cols * 8) {
    vp8a::set_error("plane stride below the MB-padded width");
    return VP8A_E_INVALID_ARGUMENT;
  }
  vp8a_status s = validate_config(base);
  if (s != VP8A_OK) return s;
  LfArgs& a = L->a;
  const int cols = (int)planes->mb_cols, rows = (int)planes->mb_rows;
  const size_t yb = planes->y_stride * (size_t)rows * 16, cb = planes->uv_stride * (size_t)rows * 8;
  const void* d;
  void* dm;
  if (write_back) {
    if ((s = st.inout(planes->y, yb, &dm)) != VP8A_OK) return s;
    a.y = (const uint8_t*)dm;
    a.oy = (uint8_t*)dm;
    if ((s = st.inout(planes->u, cb, &dm)) != VP8A_OK) return s;
    a.u = (const uint8_t*)dm;
    a.ou = (uint8_t*)dm;
    if ((s = st.inout(planes->v, cb, &dm)) != VP8A_OK) return s;
    a.v = (const uint8_t*)dm;
    a.ov = (uint8_t*)dm;
  } else {
    if ((s = st.in(planes->y, yb, &d)) != VP8A_OK) return s;
    a.y = (const uint8_t*)d;
    if ((s = st.in(planes->u, cb, &d)) != VP8A_OK) return s;
    a.u = (const uint8_t*)d;
    if ((s = st.in(planes->v, cb, &d)) != VP8A_OK) return s;
    a.v = (const uint8_t*)d;
  }
  a.ys = planes->y_stride;
  a.cs = planes->uv_stride;
  a.mb_cols = cols;
  a.mb_rows = rows;
  if ((s = st.in(mbs, sizeof(vp8a_mb_lf_info) * (size_t)cols * rows, &d)) != VP8A_OK) return s;
  a.mbs = (const vp8a_mb_lf_info*)d;
  a.base = *base;
  if (src) {
    if (src->width == 0 || src->height == 0 || src->width > (uint32_t)cols * 16 ||
        src->height > (uint32_t)rows * 16) {
      vp8a::set_error("source size does not fit the MB grid");
      return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
    }
    const uint32_t w = src->width, h = src->height, cw = (w + 1) / 2, ch = (h + 1) / 2;
    if (src->y_stride < w || src->uv_stride < cw) {
      vp8a::set_error("source stride below width");
      return VP8A_E_INVALID_ARGUMENT;
    }
    if ((s = st.in(src->y, src->y_stride * (size_t)(h - 1) + w, &d)) != VP8A_OK) return s;
    a.sy = (const uint8_t*)d;
    if ((s = st.in(src->u, src->uv_stride * (size_t)(ch - 1) + cw, &d)) != VP8A_OK) return s;
    a.su = (const uint8_t*)d;
    if ((s = st.in(src->v, src->uv_stride * (size_t)(ch - 1) + cw, &d)) != VP8A_OK) return s;
    a.sv = (const uint8_t*)d;
    a.sys = src->y_stride;
    a.scs = src->uv_stride;
    a.width = (int)w;
    a.height = (int)h;
  }
  // Row schedule.
  std::vector<int16_t> t0(rows, -1);
  std::vector<uint8_t> top(rows, 0);
  int max_t0 = 0;
  if (every_rows == 0) {
    for (int r = 0; r < rows; r++) {
      t0[r] = (int16_t)(2 * r);
      top[r] = r > 0;
    }
    max_t0 = 2 * (rows - 1);
  } else {
    const int step = every_rows < 2 ? 2 : (int)every_rows;
    for (int fr = 0; fr < rows; fr += step)
      for (int k = 0; k < 2 && fr + k < rows; k++) {
        t0[fr + k] = (int16_t)(2 * k);
        top[fr + k] = k > 0;
        max_t0 = std::max(max_t0, 2 * k);
      }
  }
  // Tails: row r's last RING MBs are final once the scored row below it in
  // the same band has run its last MB (else once row r has), and are scored
  // the step after (tf[r]). Ring sets: a row takes any set whose previous
  // row's tail was scored before the row's first step.
  std::vector<int> tf(rows, -1);
  int steps = 0;
  for (int r = 0; r < rows; r++) {
    if (t0[r] < 0) continue;
    const bool below = r + 1 < rows && t0[r + 1] >= 0 && top[r + 1];
    tf[r] = (below ? t0[r + 1] : t0[r]) + cols;
    steps = std::max(steps, tf[r] + 1);
  }
  std::vector<uint16_t> set(rows, 0);
  std::vector<int> set_free;  // per set: first step it may be taken again
  std::vector<int> order;
  for (int r = 0; r < rows; r++)
    if (t0[r] >= 0) order.push_back(r);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return t0[x] < t0[y]; });
  for (int r : order) {
    int k = -1;
    for (int q = 0; q < (int)set_free.size() && k < 0; q++)
      if (set_free[q] <= t0[r]) k = q;
    if (k < 0) {
      k = (int)set_free.size();
      set_free.push_back(0);
    }
    set[r] = (uint16_t)k;
    set_free[k] = tf[r] + 1;
  }
  // Step schedule: the rows active at step t, in increasing order, and the
  // rows whose tails are scored at step t.
  std::vector<int32_t> off(steps + 1, 0), foff(steps + 1, 0);
  std::vector<uint16_t> sched, fin;
  int max_active = 0;
  for (int t = 0; t < steps; t++) {
    off[t] = (int32_t)sched.size();
    foff[t] = (int32_t)fin.size();
    for (int r = 0; r < rows; r++) {
      if (t0[r] >= 0 && t >= t0[r] && t < t0[r] + cols) sched.push_back((uint16_t)r);
      if (tf[r] == t) fin.push_back((uint16_t)r);
    }
    max_active = std::max(max_active, (int)sched.size() - off[t]);
  }
  off[steps] = (int32_t)sched.size();
  foff[steps] = (int32_t)fin.size();
  // One upload: t0 (int16), top (u8), offsets (int32), rows (u16), sets
  // (u16), tail offsets (int32), tail rows (u16).
  auto a4 = [](size_t x) { return (x + 3) & ~(size_t)3; };
  const size_t o_top = sizeof(int16_t) * rows, o_off = a4(o_top + rows),
               o_row = o_off + sizeof(int32_t) * (steps + 1), o_set = a4(o_row + sizeof(uint16_t) * sched.size()),
               o_foff = a4(o_set + sizeof(uint16_t) * rows), o_fin = o_foff + sizeof(int32_t) * (steps + 1),
               total = o_fin + sizeof(uint16_t) * fin.size();
  std::vector<uint8_t> blob(total, 0);
  memcpy(blob.data(), t0.data(), o_top);
  memcpy(blob.data() + o_top, top.data(), rows);
  memcpy(blob.data() + o_off, off.data(), sizeof(int32_t) * (steps + 1));
  if (!sched.empty()) memcpy(blob.data() + o_row, sched.data(), sizeof(uint16_t) * sched.size());
  memcpy(blob.data() + o_set, set.data(), sizeof(uint16_t) * rows);
  memcpy(blob.data() + o_foff, foff.data(), sizeof(int32_t) * (steps + 1));
  if (!fin.empty()) memcpy(blob.data() + o_fin, fin.data(), sizeof(uint16_t) * fin.size());
  void* dblob;
  if ((s = st.upload(blob.data(), total, &dblob)) != VP8A_OK) return s;
  const uint8_t* db = (const uint8_t*)dblob;
  a.row_t0 = (const int16_t*)db;
  a.row_top = db + o_top;
  a.sched_off = (const int32_t*)(db + o_off);
  a.sched_row = (const uint16_t*)(db + o_row);
  a.row_set = (const uint16_t*)(db + o_set);
  a.fin_off = (const int32_t*)(db + o_foff);
  a.fin_row = (const uint16_t*)(db + o_fin);
  a.n_sets = (int)set_free.size();
  a.max_active = max_active;
  a.steps = steps;
  auto al4 = [](const void* p, uint64_t stride) { return ((uintptr_t)p % 4 == 0) && (stride % 4 == 0); };
  a.recon_words = al4(a.y, a.ys) && al4(a.u, a.cs) && al4(a.v, a.cs);
  a.source_words = a.sy ? (al4(a.sy, a.sys) && al4(a.su, a.scs) && al4(a.sv, a.scs)) : 0;
  auto alk = [](const void* p, uint64_t stride, unsigned k) { return ((uintptr_t)p % k == 0) && (stride % k == 0); };
  a.recon_vec = alk(a.y, a.ys, 16) && alk(a.u, a.cs, 8) && alk(a.v, a.cs, 8);
  a.source_vec = a.sy ? (alk(a.sy, a.sys, 16) && alk(a.su, a.scs, 8) && alk(a.sv, a.scs, 8)) : 0;
  L->max_steps = a.steps;
  return VP8A_OK;
}

// Launch one sweep kernel variant (NC candidates per CTA) for one picture
// (`a`) or over a job table.
template <int NC>
vp8a_status launch_nc(vp8a_ctx* ctx, unsigned grid, int threads, size_t smem, const LfArgs& a, const LfArgs* dj,
                      const uint32_t* ds, int n_jobs) {
  if (dj) {
    VP8A_CUDA(cudaFuncSetAttribute(lf_sweep_batch_kernel<NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    lf_sweep_batch_kernel<NC><<<grid, threads, smem, ctx->stream>>>(dj, ds, n_jobs);
  } else {
    VP8A_CUDA(cudaFuncSetAttribute(lf_sweep_kernel<NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    lf_sweep_kernel<NC><<<grid, threads, smem, ctx->stream>>>(a);
  }
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

vp8a_status launch_variant(vp8a_ctx* ctx, int nc, unsigned grid, int threads, size_t smem, const LfArgs& a,
                           const LfArgs* dj, const uint32_t* ds, int n_jobs) {
  if (nc == 3) return launch_nc<3>(ctx, grid, threads, smem, a, dj, ds, n_jobs);
  if (nc == 2) return launch_nc<2>(ctx, grid, threads, smem, a, dj, ds, n_jobs);
  return launch_nc<1>(ctx, grid, threads, smem, a, dj, ds, n_jobs);
}

// Shared-memory layout of a sweep launch: NC rings of `ring` bytes, then
// the half-warps' staging areas (prefetch). Returns the dynamic bytes.
size_t sweep_smem(int nc, int ring, bool pre, int threads) {
  return (size_t)nc * ring + (pre ? (size_t)(threads / 16) * sizeof(Stage) : 0);
}

// The layouts a sweep of `n` candidates can run with: candidates (passes)
// per CTA, threads per CTA and the prefetch, among those whose shared
// memory fits and that can be resident. A CTA's steps carry every one of
// its candidates' filtering, and a half-warp takes several MBs of a step
// when the CTA has fewer half-warps than the step has MBs; fewer threads
// per CTA let more CTAs share an SM, so one CTA's step barrier is covered
// by the others' work.
struct SweepLayout {
  int nc;
  bool pre;
  size_t smem;
  int threads;
  int per_sm;
};

const void* sweep_kernel_of(int nc, bool batch) {
  return batch ? (nc == 3 ? (const void*)lf_sweep_batch_kernel<3>
                          : nc == 2 ? (const void*)lf_sweep_batch_kernel<2> : (const void*)lf_sweep_batch_kernel<1>)
               : (nc == 3 ? (const void*)lf_sweep_kernel<3>
                          : nc == 2 ? (const void*)lf_sweep_kernel<2> : (const void*)lf_sweep_kernel<1>);
}

vp8a_status sweep_layouts(vp8a_ctx* ctx, int n, int ring, bool pre_ok, int threads_full, bool batch,
                          std::vector<SweepLayout>* out) {
  out->clear();
  int max_smem = 0;
  VP8A_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
  const int tcands[] = {1024, 768, 512, 384, 352, 256, 192, 128};
  for (int nc = 3; nc >= 1; nc--) {
    if (nc > 1 && n < nc) continue;
    const void* k = sweep_kernel_of(nc, batch);
    cudaFuncAttributes fa;
    VP8A_CUDA(cudaFuncGetAttributes(&fa, k));
    for (int pre = pre_ok ? 1 : 0; pre >= 0; pre--) {
      int last_per_sm = 0;
      for (int ti = 0; ti < (int)(sizeof tcands / sizeof tcands[0]); ti++) {
        const int t = ti == 0 ? threads_full : std::min(threads_full, tcands[ti]);
        if (ti > 0 && t >= threads_full) continue;
        const size_t smem = sweep_smem(nc, ring, pre, t);
        if (smem + fa.sharedSizeBytes + 1024 > (size_t)max_smem) continue;
        VP8A_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        VP8A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, t, smem));
        if (per_sm < 1) continue;
        // Fewer threads only pay when more CTAs share an SM.
        if (ti > 0 && per_sm <= last_per_sm) continue;
        last_per_sm = per_sm;
        out->push_back(SweepLayout{nc, pre != 0, smem, t, per_sm});
      }
    }
  }
  return VP8A_OK;
}

// The cost model's pick among `ls` (full thread count only): whole waves of
// CTAs over the GPU x candidates per CTA, 15 % more without the prefetch
// and 20 % less per candidate when a CTA carries several (their filtering
// shares each step's barrier and loads) — factors measured on the 1080p
// and 640x368 sweeps.
bool model_layout(vp8a_ctx* ctx, int n, int threads_full, const std::vector<SweepLayout>& ls, SweepLayout* out) {
  double best = 1e30;
  bool found = false;
  for (const SweepLayout& L : ls) {
    if (L.threads != threads_full) continue;
    const long ctas = (n + L.nc - 1) / L.nc, slots = (long)ctx->sm_count * L.per_sm;
    const double cost =
        (double)((ctas + slots - 1) / slots) * L.nc * (L.pre ? 1.0 : 1.15) * (L.nc > 1 ? 0.8 : 1.0);
    if (cost < best) {
      best = cost;
      *out = L;
      found = true;
    }
  }
  return found;
}

bool pick_layout(vp8a_ctx* ctx, int n, int ring, bool pre_ok, int threads, bool batch, SweepLayout* out) {
  std::vector<SweepLayout> ls;
  if (sweep_layouts(ctx, n, ring, pre_ok, threads, batch, &ls) != VP8A_OK) return false;
  return model_layout(ctx, n, threads, ls, out);
}

// Launch the sweep over `n` candidates (pairs of level, sharpness) already
// in device memory at a.cands, with the slot rings and staging in shared
// memory (a layout of sweep_layouts: forced, measured or modelled);
// otherwise, when `gst` can provide them, with the rings in global memory.
// The prefetch needs planes whose rows allow aligned 16- and 8-byte
// asynchronous copies.
vp8a_status run_sweep(vp8a_ctx* ctx, LfArgs a, int n, vp8a::Stager* gst) {
  if (n == 0) return VP8A_OK;
  a.n_cands = n;
  a.ring_bytes = (a.row_set ? a.n_sets : a.mb_rows) * RING * SLOT_STRIDE;
  int max_smem = 0;
  VP8A_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
  const int threads_full = std::min(1024, std::max(32, (16 * a.max_active + 31) / 32 * 32));
  auto al = [](const void* p, uint64_t stride, unsigned k) { return ((uintptr_t)p % k == 0) && (stride % k == 0); };
  bool pre_ok = al(a.y, a.ys, 16) && al(a.u, a.cs, 8) && al(a.v, a.cs, 8) && (uintptr_t)a.mbs % 8 == 0;
  if (a.ssd_out) pre_ok = pre_ok && al(a.sy, a.sys, 16) && al(a.su, a.scs, 8) && al(a.sv, a.scs, 8);
  cudaFuncAttributes f1;
  VP8A_CUDA(cudaFuncGetAttributes(&f1, lf_sweep_kernel<1>));
  std::vector<SweepLayout> ls;
  vp8a_status s = sweep_layouts(ctx, n, a.ring_bytes, pre_ok, threads_full, false, &ls);
  if (s != VP8A_OK) return s;
  auto launch = [&](const SweepLayout& L) {
    LfArgs b = a;
    b.smem_slots = 1;
    b.gslots = nullptr;
    b.prefetch = L.pre;
    b.stage_off = L.nc * a.ring_bytes;
    ctx->last_layout[0] = L.nc;
    ctx->last_layout[1] = L.threads;
    ctx->last_layout[2] = L.pre;
    ctx->last_layout[3] = L.per_sm;
    return launch_variant(ctx, L.nc, (unsigned)((n + L.nc - 1) / L.nc), L.threads, L.smem, b, nullptr, nullptr, 0);
  };
  if (!ls.empty()) {
    if (ctx->force_layout[0]) {
      // A forced layout (tests): it must be one of the feasible ones.
      for (const SweepLayout& x : ls)
        if (x.nc == ctx->force_layout[0] && x.threads == ctx->force_layout[1] && (int)x.pre == ctx->force_layout[2])
          return launch(x);
      vp8a::set_error("the forced sweep layout does not fit this picture");
      return VP8A_E_INVALID_ARGUMENT;
    }
    SweepLayout L = ls[0];
    // Filtering into the planes (apply mode) or a handful of candidates:
    // the model; a scored sweep: the measured choice for this shape.
    if (!ctx->autotune || !a.ssd_out || n < 16 || ls.size() == 1) {
      model_layout(ctx, n, threads_full, ls, &L);
      return launch(L);
    }
    const std::array<int64_t, 6> key{a.mb_cols, a.mb_rows, n, a.steps, (int64_t)pre_ok, a.row_set != nullptr};
    auto it = ctx->lf_tuned.find(key);
    if (it == ctx->lf_tuned.end()) {
      // Time every feasible layout on this call's own inputs (a scored
      // sweep only writes its table, so repeating it changes nothing) and
      // keep the fastest.
      cudaEvent_t e0, e1;
      VP8A_CUDA(cudaEventCreate(&e0));
      VP8A_CUDA(cudaEventCreate(&e1));
      float best = 1e30f;
      std::array<int, 3> pick{ls[0].nc, ls[0].threads, (int)ls[0].pre};
      for (const SweepLayout& x : ls) {
        if ((s = launch(x)) != VP8A_OK) break;  // warm
        if ((s = vp8a::cuda_ok(cudaEventRecord(e0, ctx->stream), "cudaEventRecord")) != VP8A_OK) break;
        if ((s = launch(x)) != VP8A_OK) break;
        if ((s = vp8a::cuda_ok(cudaEventRecord(e1, ctx->stream), "cudaEventRecord")) != VP8A_OK) break;
        if ((s = vp8a::cuda_ok(cudaEventSynchronize(e1), "cudaEventSynchronize")) != VP8A_OK) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
          best = ms;
          pick = {x.nc, x.threads, (int)x.pre};
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      if (s != VP8A_OK) return s;
      it = ctx->lf_tuned.emplace(key, pick).first;
    }
    for (const SweepLayout& x : ls)
      if (x.nc == it->second[0] && x.threads == it->second[1] && (int)x.pre == it->second[2]) L = x;
    return launch(L);
  }
  if (!gst) {
    vp8a::set_error("the MB rows' slot rings do not fit in shared memory");
    return VP8A_E_INVALID_DIMENSIONS;
  }
  // Rings in global memory, one set per candidate; staging still shared.
  void* g;
  if ((s = gst->scratch((size_t)a.ring_bytes * n, &g)) != VP8A_OK) return s;
  a.smem_slots = 0;
  a.gslots = (uint8_t*)g;
  a.prefetch = pre_ok && sweep_smem(0, 0, true, threads_full) + f1.sharedSizeBytes + 1024 <= (size_t)max_smem;
  a.stage_off = 0;
  ctx->last_layout[0] = 1;
  ctx->last_layout[1] = threads_full;
  ctx->last_layout[2] = a.prefetch;
  ctx->last_layout[3] = 0;
  return launch_variant(ctx, 1, (unsigned)n, threads_full, sweep_smem(0, 0, a.prefetch, threads_full), a, nullptr,
                        nullptr, 0);
}

// The whole 64 x 8 grid as distinct filter passes. Two sharpness values
// of one level filter identically when every MB level the configuration can
// produce from that level (each segment, reference and mode class of
// calculate_mb_filter_level_inter) has the same interior limit under both:
// the interior limit and the level fix every parameter of the §15 filters
// (LoopFilterParams::derive, src/loop_filter.rs:99-148). Each pass fills the
// table entries of its sharpness group (`masks`); level 0 is one pass for
// all eight (score_filter_candidate's unfiltered short cut).
// Writes the passes into `pairs` (2 per pass) and `masks` (1 per pass;
// room for 1 + 63 * 8 passes) and returns their number. No heap memory.
int grid_passes(const vp8a_filter_config& base, uint8_t* pairs, uint8_t* masks) {
  int n = 0;
  pairs[0] = pairs[1] = 0;
  masks[n++] = 0xff;
  vp8a_mb_lf_info classes[4 * 11];
  int nc = 0;
  const int nseg = base.segmentation_enabled ? 4 : 1;
  for (int seg = 0; seg < nseg; seg++) {
    vp8a_mb_lf_info m{};
    m.segment_id = (int8_t)seg;
    m.ref_frame = VP8A_REF_INTRA;
    m.inter_mode = VP8A_MODE_NONE;
    for (int bp = 0; bp < 2; bp++) {
      m.y_mode_is_bpred = (uint8_t)bp;
      classes[nc++] = m;
    }
    m.y_mode_is_bpred = 0;
    for (int ref = VP8A_REF_LAST; ref <= VP8A_REF_ALTREF; ref++)
      for (int mode : {VP8A_MODE_ZERO, VP8A_MODE_SPLIT, VP8A_MODE_NEAREST}) {
        m.ref_frame = (uint8_t)ref;
        m.inter_mode = (uint8_t)mode;
        classes[nc++] = m;
      }
  }
  for (int level = 1; level < 64; level++) {
    uint8_t done = 0;
    for (int s0 = 0; s0 < 8; s0++) {
      if (done >> s0 & 1) continue;
      uint8_t mask = 0;
      for (int s1 = s0; s1 < 8; s1++) {
        bool same = true;
        for (int c = 0; c < nc; c++) {
          const int l = mb_level(base, level, classes[c]);
          if (l != 0 && interior_limit(l, s0) != interior_limit(l, s1)) same = false;
        }
        if (same) mask |= (uint8_t)(1u << s1);
      }
      done |= mask;
      pairs[2 * n] = (uint8_t)level;
      pairs[2 * n + 1] = (uint8_t)s0;
      masks[n++] = mask;
    }
  }
  return n;
}

void grid_candidates(const vp8a_filter_config& base, std::vector<uint8_t>& pairs, std::vector<uint8_t>& masks) {
  pairs.resize(2 * (1 + 63 * 8));
  masks.resize(1 + 63 * 8);
  const int n = grid_passes(base, pairs.data(), masks.data());
  pairs.resize(2 * n);
  masks.resize(n);
}

// Upload a grid's candidate pairs and masks into `a` (level 0 and the
// levels lo..hi).
vp8a_status upload_grid(vp8a_ctx* ctx, vp8a::Stager& st, const vp8a_filter_config& base, LfArgs* a, int lo = 1,
                        int hi = 63) {
  std::vector<uint8_t> all_pairs, all_masks, pairs, masks;
  grid_candidates(base, all_pairs, all_masks);
  for (size_t i = 0; i < all_masks.size(); i++) {
    const int level = all_pairs[2 * i];
    if (level != 0 && (level < lo || level > hi)) continue;
    pairs.push_back(all_pairs[2 * i]);
    pairs.push_back(all_pairs[2 * i + 1]);
    masks.push_back(all_masks[i]);
  }
  const size_t n = masks.size();
  std::vector<uint8_t> blob(3 * n);
  memcpy(blob.data(), pairs.data(), 2 * n);
  memcpy(blob.data() + 2 * n, masks.data(), n);
  void* d;
  vp8a_status s;
  if ((s = st.upload(blob.data(), blob.size(), &d)) != VP8A_OK) return s;
  a->cands = (const uint8_t*)d;
  a->cand_mask = (const uint8_t*)d + 2 * n;
  a->n_cands = (int)n;
  return VP8A_OK;
}

vp8a_status launch_sweep(vp8a_ctx* ctx, vp8a::Stager& st, LfArgs a, const uint8_t* cands, int n) {
  if (n == 0) return VP8A_OK;
  void* dc;
  vp8a_status s;
  if ((s = st.upload(cands, (size_t)n * 2, &dc)) != VP8A_OK) return s;
  a.cands = (const uint8_t*)dc;
  return run_sweep(ctx, a, n, &st);
}

// Score `cands` into `table` (host, 512 entries indexed level * 8 + sharp).
vp8a_status score_candidates(vp8a_ctx* ctx, vp8a::Stager& st, const LfArgs& a, void* dtable,
                             const std::vector<uint8_t>& cands, uint64_t* table) {
  vp8a_status s = launch_sweep(ctx, st, a, cands.data(), (int)(cands.size() / 2));
  if (s != VP8A_OK) return s;
  VP8A_CUDA(cudaMemcpyAsync(table, dtable, 512 * sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx->stream));
  VP8A_CUDA(cudaStreamSynchronize(ctx->stream));
  return VP8A_OK;
}

// ----------------------------------------------- sweep without allocation
//
// vp8a_filter_sweep_noalloc runs the same sweep kernel as vp8a_filter_sweep
// for callers that cannot allocate device memory while they run. Its scratch
// (the candidate list and the step schedule) lives in one fixed array of
// device memory owned by the library, built on the device by a small
// kernel; every buffer the caller names must already be on the device.
constexpr int NA_MAX_MB_COLS = 256;  // 4096 pixels
constexpr int NA_MAX_MB_ROWS = 136;  // 2176 pixels: every row's slot ring fits in shared memory
constexpr int NA_MAX_STEPS = 2 * (NA_MAX_MB_ROWS - 1) + NA_MAX_MB_COLS;
constexpr int NA_CANDIDATES = 1 + 63 * 8;
// Scratch layout (bytes).
constexpr size_t NA_CANDS = 0;                                              // (level, sharpness) pairs
constexpr size_t NA_T0 = 1024;                                              // int16 per MB row
constexpr size_t NA_TOP = NA_T0 + 2 * NA_MAX_MB_ROWS;                       // u8 per MB row
constexpr size_t NA_MASK = 1440;                                            // u8 sharpness mask per pass
constexpr size_t NA_OFF = 2048;                                             // int32 per step + 1
constexpr size_t NA_ROWS = (NA_OFF + 4 * (NA_MAX_STEPS + 1) + 15) & ~(size_t)15;  // u16 per scored MB
constexpr size_t NA_BYTES = NA_ROWS + 2 * (size_t)NA_MAX_MB_ROWS * NA_MAX_MB_COLS;
static_assert(2 * NA_CANDIDATES <= NA_T0 && NA_TOP + NA_MAX_MB_ROWS <= NA_MASK &&
                  NA_MASK + NA_CANDIDATES <= NA_OFF, "scratch layout");

// The grid's filter passes (grid_candidates: level 0, then one pass per
// group of sharpness values that filter identically), passed to the
// schedule kernel by value (1.5 KB of kernel parameters) so that no host
// buffer has to be staged.
struct NaGrid {
  int n;
  uint8_t pairs[2 * NA_CANDIDATES];
  uint8_t masks[NA_CANDIDATES];
};

// The library's only copy; every call on a device shares it (about 72 KiB,
// held by each device that loads the library until the process exits).
static __device__ __align__(256) uint8_t g_sweep_scratch[NA_BYTES];

// Candidates and step schedule of vp8a_filter_sweep (the host-built ones of
// stage_lf and vp8a_filter_sweep), written on the device. One CTA of 1024
// threads: steps <= NA_MAX_STEPS < 1024.
__global__ void __launch_bounds__(1024) sweep_schedule_kernel(uint8_t* scr, int rows, int cols, int every_rows,
                                                              int steps, const __grid_constant__ NaGrid grid) {
  __shared__ int16_t st0[NA_MAX_MB_ROWS];
  __shared__ int cnt[NA_MAX_STEPS];
  uint8_t* cands = scr + NA_CANDS;
  uint8_t* masks = scr + NA_MASK;
  int16_t* t0 = (int16_t*)(scr + NA_T0);
  uint8_t* top = scr + NA_TOP;
  int32_t* off = (int32_t*)(scr + NA_OFF);
  uint16_t* srow = (uint16_t*)(scr + NA_ROWS);
  const int tid = threadIdx.x;
  // The grid's passes and the table entries each one fills.
  for (int i = tid; i < grid.n; i += blockDim.x) {
    cands[2 * i] = grid.pairs[2 * i];
    cands[2 * i + 1] = grid.pairs[2 * i + 1];
    masks[i] = grid.masks[i];
  }
  for (int r = tid; r < rows; r += blockDim.x) {
    int v, t;
    if (every_rows == 0) {
      v = 2 * r;
      t = r > 0;
    } else {
      const int step = every_rows < 2 ? 2 : every_rows, k = r % step;
      v = k < 2 ? 2 * k : -1;
      t = k == 1;
    }
    st0[r] = (int16_t)v;
    t0[r] = (int16_t)v;
    top[r] = (uint8_t)t;
  }
  __syncthreads();
  for (int t = tid; t < steps; t += blockDim.x) {
    int n = 0;
    for (int r = 0; r < rows; r++) n += st0[r] >= 0 && t >= st0[r] && t < st0[r] + cols;
    cnt[t] = n;
  }
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int t = 0; t < steps; t++) {
      off[t] = acc;
      acc += cnt[t];
      cnt[t] = off[t];
    }
    off[steps] = acc;
  }
  __syncthreads();
  for (int t = tid; t < steps; t += blockDim.x) {
    int o = cnt[t];
    for (int r = 0; r < rows; r++)
      if (st0[r] >= 0 && t >= st0[r] && t < st0[r] + cols) srow[o++] = (uint16_t)r;
  }
}

// Device address of g_sweep_scratch on `dev` (current), looked up once per
// device. In host code the array's name only stands in for the symbol.
vp8a_status sweep_scratch(int dev, uint8_t** out) {
  static std::mutex mu;
  static void* ptr[64] = {};
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0 || dev >= 64) {
    vp8a::set_error("device index out of range");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (!ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sweep_scratch);
    if (e != cudaSuccess) return vp8a::cuda_fail(e, "cudaGetSymbolAddress(g_sweep_scratch)");
    ptr[dev] = p;
  }
  *out = (uint8_t*)ptr[dev];
  return VP8A_OK;
}

// True when `p` is device (or managed) memory usable on `dev`.
bool device_resident(const void* p, int dev) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (at.type == cudaMemoryTypeDevice && at.device == dev) || at.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" {

vp8a_status vp8a_filter_frame(vp8a_ctx* ctx, vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                              const vp8a_filter_config* config) {
  if (!ctx) return VP8A_E_INVALID_ARGUMENT;
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  LfInputs L;
  vp8a_status s = stage_lf(ctx, st, planes, mbs, config, nullptr, 0, true, &L);
  if (s != VP8A_OK) return s;
  const uint8_t cand[2] = {config->loop_filter_level, config->sharpness_level};
  L.a.level0_unfiltered = 0;
  if ((s = launch_sweep(ctx, st, L.a, cand, 1)) != VP8A_OK) return s;
  return st.finish();
}

vp8a_status vp8a_reconstruction_ssd(vp8a_ctx* ctx, const vp8a_planes* planes, const vp8a_source* src,
                                    uint64_t* ssd_out) {
  if (!ctx || !planes || !src || !ssd_out) return VP8A_E_INVALID_ARGUMENT;
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  const uint32_t w = src->width, h = src->height, cw = (w + 1) / 2, ch = (h + 1) / 2;
  if (w == 0 || h == 0 || w > planes->mb_cols * 16 || h > planes->mb_rows * 16) {
    vp8a::set_error("source size does not fit the MB grid");
    return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
  }
  vp8a_status s;
  const void *ry, *ru, *rv, *sy, *su, *sv;
  if ((s = st.in(planes->y, planes->y_stride * (size_t)(h - 1) + w, &ry)) != VP8A_OK) return s;
  if ((s = st.in(planes->u, planes->uv_stride * (size_t)(ch - 1) + cw, &ru)) != VP8A_OK) return s;
  if ((s = st.in(planes->v, planes->uv_stride * (size_t)(ch - 1) + cw, &rv)) != VP8A_OK) return s;
  if ((s = st.in(src->y, src->y_stride * (size_t)(h - 1) + w, &sy)) != VP8A_OK) return s;
  if ((s = st.in(src->u, src->uv_stride * (size_t)(ch - 1) + cw, &su)) != VP8A_OK) return s;
  if ((s = st.in(src->v, src->uv_stride * (size_t)(ch - 1) + cw, &sv)) != VP8A_OK) return s;
  void* acc;
  if ((s = st.out(ssd_out, sizeof(uint64_t), &acc)) != VP8A_OK) return s;
  VP8A_CUDA(cudaMemsetAsync(acc, 0, sizeof(uint64_t), ctx->stream));
  unsigned grid = (unsigned)std::max(1, ctx->sm_count * 4);
  ssd_kernel<<<grid, 256, 0, ctx->stream>>>((const uint8_t*)ry, planes->y_stride, (const uint8_t*)sy, src->y_stride,
                                            (int)w, (int)h, (unsigned long long*)acc);
  ssd_kernel<<<grid, 256, 0, ctx->stream>>>((const uint8_t*)ru, planes->uv_stride, (const uint8_t*)su,
                                            src->uv_stride, (int)cw, (int)ch, (unsigned long long*)acc);
  ssd_kernel<<<grid, 256, 0, ctx->stream>>>((const uint8_t*)rv, planes->uv_stride, (const uint8_t*)sv,
                                            src->uv_stride, (int)cw, (int)ch, (unsigned long long*)acc);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches += 3;
  return st.finish();
}

vp8a_status vp8a_filter_sweep(vp8a_ctx* ctx, const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                              const vp8a_filter_config* base, const vp8a_source* src, uint32_t every_rows,
                              uint64_t* ssd_out) {
  if (!ctx || !src || !ssd_out) return VP8A_E_INVALID_ARGUMENT;
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  LfInputs L;
  vp8a_status s = stage_lf(ctx, st, planes, mbs, base, src, every_rows, false, &L);
  if (s != VP8A_OK) return s;
  void* dt;
  if ((s = st.out(ssd_out, 512 * sizeof(uint64_t), &dt)) != VP8A_OK) return s;
  L.a.ssd_out = (uint64_t*)dt;
  L.a.level0_unfiltered = 1;
  if ((s = upload_grid(ctx, st, *base, &L.a)) != VP8A_OK) return s;
  if ((s = run_sweep(ctx, L.a, L.a.n_cands, &st)) != VP8A_OK) return s;
  return st.finish();
}

vp8a_status vp8a_filter_sweep_window(vp8a_ctx* ctx, const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                                     const vp8a_filter_config* base, const vp8a_source* src, uint32_t lo_level,
                                     uint32_t hi_level, uint64_t* ssd_out) {
  if (!ctx || !src || !ssd_out || !base) return VP8A_E_INVALID_ARGUMENT;
  if (lo_level > hi_level || hi_level > 63) {
    vp8a::set_error("window levels must satisfy lo <= hi <= 63");
    return VP8A_E_LOOP_FILTER_LEVEL_OUT_OF_RANGE;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  LfInputs L;
  vp8a_status s = stage_lf(ctx, st, planes, mbs, base, src, 0, false, &L);
  if (s != VP8A_OK) return s;
  void* dt;
  if ((s = st.out(ssd_out, 512 * sizeof(uint64_t), &dt)) != VP8A_OK) return s;
  VP8A_CUDA(cudaMemsetAsync(dt, 0xff, 512 * sizeof(uint64_t), ctx->stream));
  L.a.ssd_out = (uint64_t*)dt;
  L.a.level0_unfiltered = 1;
  if ((s = upload_grid(ctx, st, *base, &L.a, (int)std::max(1u, lo_level), (int)hi_level)) != VP8A_OK) return s;
  if ((s = run_sweep(ctx, L.a, L.a.n_cands, &st)) != VP8A_OK) return s;
  return st.finish();
}

// Every job's candidates (a.cands / a.cand_mask / a.n_cands set, rings
// sized) as one batched launch where their slot rings fit in shared memory
// together, the rest as launches of their own.
vp8a_status run_batch(vp8a_ctx* ctx, vp8a::Stager& st, std::vector<LfArgs>& args) {
  const uint32_t n_jobs = (uint32_t)args.size();
  vp8a_status s;
  // One launch for every job whose slot rings fit in shared memory (two
  // candidates per CTA when the largest job's pair fits, else one), with
  // the most half-warps any job needs; the rest run as their own launches.
  int max_smem = 0;
  VP8A_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
  cudaFuncAttributes f1, f2;
  VP8A_CUDA(cudaFuncGetAttributes(&f1, lf_sweep_batch_kernel<1>));
  VP8A_CUDA(cudaFuncGetAttributes(&f2, lf_sweep_batch_kernel<2>));
  auto al = [](const void* p, uint64_t stride, unsigned k) { return ((uintptr_t)p % k == 0) && (stride % k == 0); };
  auto threads_of = [](const LfArgs& a) { return std::min(1024, std::max(32, (16 * a.max_active + 31) / 32 * 32)); };
  auto pre_of = [&](const LfArgs& a) {
    return al(a.y, a.ys, 16) && al(a.u, a.cs, 8) && al(a.v, a.cs, 8) && (uintptr_t)a.mbs % 8 == 0 &&
           al(a.sy, a.sys, 16) && al(a.su, a.scs, 8) && al(a.sv, a.scs, 8);
  };
  std::vector<uint32_t> group, alone;
  int threads = 32, max_ring = 0;
  bool pre = true;
  for (uint32_t j = 0; j < n_jobs; j++) {
    const int t = std::max(threads, threads_of(args[j]));
    const int r = std::max(max_ring, args[j].ring_bytes);
    const bool p = pre && pre_of(args[j]);
    if (sweep_smem(1, r, p, t) + f1.sharedSizeBytes + 1024 > (size_t)max_smem) {
      alone.push_back(j);
      continue;
    }
    group.push_back(j);
    threads = t;
    max_ring = r;
    pre = p;
  }
  // Largest pictures first: their CTAs run longest, so they start first
  // and the short ones fill in behind them.
  std::stable_sort(group.begin(), group.end(), [&](uint32_t x, uint32_t y) {
    return (long)args[x].mb_cols * args[x].mb_rows > (long)args[y].mb_cols * args[y].mb_rows;
  });
  if (!group.empty()) {
    // The layout for the largest job's rings and the group's candidates
    // (each CTA takes `nc` candidates of one job): measured on the first
    // batch of these picture shapes (autotune), else the cost model.
    long n_all = 0;
    for (uint32_t j : group) n_all += args[j].n_cands;
    std::vector<SweepLayout> ls;
    if ((s = sweep_layouts(ctx, (int)std::min<long>(n_all, 1 << 30), max_ring, pre, threads, true, &ls)) != VP8A_OK)
      return s;
    if (ls.empty()) {
      vp8a::set_error("no sweep layout fits in shared memory");
      return VP8A_E_CUDA;
    }
    auto launch_group = [&](const SweepLayout& L) -> vp8a_status {
      const int nc = L.nc;
      std::vector<LfArgs> table;
      std::vector<uint32_t> start{0};
      for (uint32_t j : group) {
        LfArgs a = args[j];
        a.smem_slots = 1;
        a.gslots = nullptr;
        a.prefetch = L.pre;
        a.stage_off = nc * a.ring_bytes;
        table.push_back(a);
        start.push_back(start.back() + (uint32_t)((a.n_cands + nc - 1) / nc));
      }
      const size_t o_start = sizeof(LfArgs) * table.size(), bytes = o_start + sizeof(uint32_t) * start.size();
      std::vector<uint8_t> blob(bytes);
      memcpy(blob.data(), table.data(), o_start);
      memcpy(blob.data() + o_start, start.data(), sizeof(uint32_t) * start.size());
      void* d;
      vp8a_status e = st.upload(blob.data(), bytes, &d);
      if (e != VP8A_OK) return e;
      ctx->last_layout[0] = L.nc;
      ctx->last_layout[1] = L.threads;
      ctx->last_layout[2] = L.pre;
      ctx->last_layout[3] = L.per_sm;
      return launch_variant(ctx, nc, start.back(), L.threads, L.smem, table[0], (const LfArgs*)d,
                            (const uint32_t*)((const uint8_t*)d + o_start), (int)table.size());
    };
    SweepLayout L = ls[0];
    model_layout(ctx, (int)std::min<long>(n_all, 1 << 30), threads, ls, &L);
    bool scored = true;
    for (uint32_t j : group) scored = scored && args[j].ssd_out != nullptr;
    if (ctx->autotune && scored && ls.size() > 1) {
      std::vector<int64_t> key{(int64_t)pre};
      for (uint32_t j : group) key.insert(key.end(), {args[j].mb_cols, args[j].mb_rows, args[j].n_cands, args[j].steps});
      auto it = ctx->lf_tuned_batch.find(key);
      if (it == ctx->lf_tuned_batch.end()) {
        // Time every feasible layout on this batch (scored sweeps only
        // write their tables, so repeating one changes nothing).
        cudaEvent_t e0, e1;
        VP8A_CUDA(cudaEventCreate(&e0));
        VP8A_CUDA(cudaEventCreate(&e1));
        float best = 1e30f;
        std::array<int, 3> pick{L.nc, L.threads, (int)L.pre};
        for (const SweepLayout& x : ls) {
          if ((s = launch_group(x)) != VP8A_OK) break;  // warm
          if ((s = vp8a::cuda_ok(cudaEventRecord(e0, ctx->stream), "cudaEventRecord")) != VP8A_OK) break;
          if ((s = launch_group(x)) != VP8A_OK) break;
          if ((s = vp8a::cuda_ok(cudaEventRecord(e1, ctx->stream), "cudaEventRecord")) != VP8A_OK) break;
          if ((s = vp8a::cuda_ok(cudaEventSynchronize(e1), "cudaEventSynchronize")) != VP8A_OK) break;
          float ms = 0.f;
          cudaEventElapsedTime(&ms, e0, e1);
          if (ms < best) {
            best = ms;
            pick = {x.nc, x.threads, (int)x.pre};
          }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (s != VP8A_OK) return s;
        it = ctx->lf_tuned_batch.emplace(key, pick).first;
      }
      for (const SweepLayout& x : ls)
        if (x.nc == it->second[0] && x.threads == it->second[1] && (int)x.pre == it->second[2]) L = x;
    }
    if ((s = launch_group(L)) != VP8A_OK) return s;
  }
  for (uint32_t j : alone)
    if ((s = run_sweep(ctx, args[j], args[j].n_cands, &st)) != VP8A_OK) return s;
  return VP8A_OK;
}

vp8a_status vp8a_filter_sweeps(vp8a_ctx* ctx, const vp8a_sweep_job* jobs, uint32_t n_jobs) {
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
  std::vector<LfArgs> args(n_jobs);
  for (uint32_t j = 0; j < n_jobs; j++) {
    const vp8a_sweep_job& J = jobs[j];
    if (!J.ssd_out) {
      vp8a::set_error("null ssd_out");
      return VP8A_E_INVALID_ARGUMENT;
    }
    LfInputs L;
    if ((s = stage_lf(ctx, st, &J.planes, J.mbs, &J.base, &J.src, J.every_rows, false, &L)) != VP8A_OK) return s;
    void* dt;
    if ((s = st.out(J.ssd_out, 512 * sizeof(uint64_t), &dt)) != VP8A_OK) return s;
    L.a.ssd_out = (uint64_t*)dt;
    L.a.level0_unfiltered = 1;
    if ((s = upload_grid(ctx, st, J.base, &L.a)) != VP8A_OK) return s;
    L.a.ring_bytes = L.a.n_sets * RING * SLOT_STRIDE;
    args[j] = L.a;
  }
  if ((s = run_batch(ctx, st, args)) != VP8A_OK) return s;
  return st.finish();
}

vp8a_status vp8a_select_filter_params_batch(vp8a_ctx* ctx, const vp8a_sweep_job* jobs, uint32_t n_jobs,
                                            uint8_t* level_out, uint8_t* sharpness_out) {
  if (!ctx || (!jobs && n_jobs) || (n_jobs && (!level_out || !sharpness_out))) {
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
  std::vector<LfArgs> base_args(n_jobs);
  void* dt;
  if ((s = st.scratch(512 * sizeof(uint64_t) * n_jobs, &dt)) != VP8A_OK) return s;
  VP8A_CUDA(cudaMemsetAsync(dt, 0, 512 * sizeof(uint64_t) * n_jobs, ctx->stream));
  std::vector<uint8_t> bs(n_jobs), best_level(n_jobs, 0), best_sharp(n_jobs);
  std::vector<uint64_t> best(n_jobs), t((size_t)512 * n_jobs, 0);
  for (uint32_t j = 0; j < n_jobs; j++) {
    const vp8a_sweep_job& J = jobs[j];
    if (J.every_rows != 0) {
      vp8a::set_error("vp8a_select_filter_params_batch scores whole frames (every_rows must be 0)");
      return VP8A_E_INVALID_ARGUMENT;
    }
    LfInputs Li;
    if ((s = stage_lf(ctx, st, &J.planes, J.mbs, &J.base, &J.src, 0, false, &Li)) != VP8A_OK) return s;
    Li.a.ssd_out = (uint64_t*)dt + (size_t)512 * j;
    Li.a.level0_unfiltered = 1;
    Li.a.cand_mask = nullptr;
    Li.a.ring_bytes = Li.a.n_sets * RING * SLOT_STRIDE;
    base_args[j] = Li.a;
    bs[j] = J.base.sharpness_level > 7 ? 7 : J.base.sharpness_level;
    best_sharp[j] = bs[j];
  }
  // One stage of the walk: job j scores the (level, sharpness) pairs in
  // cands[j] (none: the job sits the stage out); the tables come back.
  auto stage = [&](const std::vector<std::vector<uint8_t>>& cands) -> vp8a_status {
    std::vector<LfArgs> args;
    for (uint32_t j = 0; j < n_jobs; j++) {
      if (cands[j].empty()) continue;
      LfArgs a = base_args[j];
      void* dc;
      vp8a_status e = st.upload(cands[j].data(), cands[j].size(), &dc);
      if (e != VP8A_OK) return e;
      a.cands = (const uint8_t*)dc;
      a.n_cands = (int)(cands[j].size() / 2);
      args.push_back(a);
    }
    if (args.empty()) return VP8A_OK;
    vp8a_status e = run_batch(ctx, st, args);
    if (e != VP8A_OK) return e;
    VP8A_CUDA(cudaMemcpyAsync(t.data(), dt, t.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx->stream));
    VP8A_CUDA(cudaStreamSynchronize(ctx->stream));
    return VP8A_OK;
  };
  std::vector<std::vector<uint8_t>> c(n_jobs);
  // Stage 1: grid 0, 4, ..., 60, 63 at the base sharpness.
  for (uint32_t j = 0; j < n_jobs; j++) {
    for (int l = 0; l <= 60; l += 4) c[j].insert(c[j].end(), {(uint8_t)l, bs[j]});
    c[j].insert(c[j].end(), {63, bs[j]});
  }
  if ((s = stage(c)) != VP8A_OK) return s;
  for (uint32_t j = 0; j < n_jobs; j++) {
    const uint64_t* tj = t.data() + (size_t)512 * j;
    best[j] = tj[0 * 8 + bs[j]];
    for (size_t i = 2; i < c[j].size(); i += 2)
      if (tj[c[j][i] * 8 + bs[j]] < best[j]) {
        best[j] = tj[c[j][i] * 8 + bs[j]];
        best_level[j] = c[j][i];
      }
  }
  // Refine +/-3 around each grid winner, excluding it.
  for (uint32_t j = 0; j < n_jobs; j++) {
    c[j].clear();
    const int lo = best_level[j] >= 3 ? best_level[j] - 3 : 0, hi = std::min(63, best_level[j] + 3);
    for (int l = lo; l <= hi; l++)
      if (l != best_level[j]) c[j].insert(c[j].end(), {(uint8_t)l, bs[j]});
  }
  if ((s = stage(c)) != VP8A_OK) return s;
  for (uint32_t j = 0; j < n_jobs; j++) {
    const uint64_t* tj = t.data() + (size_t)512 * j;
    for (size_t i = 0; i < c[j].size(); i += 2)
      if (tj[c[j][i] * 8 + bs[j]] < best[j]) {
        best[j] = tj[c[j][i] * 8 + bs[j]];
        best_level[j] = c[j][i];
      }
  }
  // Stage 2: the other sharpness values at each chosen non-zero level.
  for (uint32_t j = 0; j < n_jobs; j++) {
    c[j].clear();
    if (best_level[j] == 0) continue;
    for (int sh = 0; sh < 8; sh++)
      if (sh != bs[j]) c[j].insert(c[j].end(), {best_level[j], (uint8_t)sh});
  }
  if ((s = stage(c)) != VP8A_OK) return s;
  for (uint32_t j = 0; j < n_jobs; j++) {
    const uint64_t* tj = t.data() + (size_t)512 * j;
    for (size_t i = 0; i < c[j].size(); i += 2)
      if (tj[best_level[j] * 8 + c[j][i + 1]] < best[j]) {
        best[j] = tj[best_level[j] * 8 + c[j][i + 1]];
        best_sharp[j] = c[j][i + 1];
      }
    level_out[j] = best_level[j];
    sharpness_out[j] = best_sharp[j];
  }
  return st.finish();
}

vp8a_status vp8a_select_filter_params(vp8a_ctx* ctx, const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                                      const vp8a_filter_config* base, const vp8a_source* src, uint8_t* level_out,
                                      uint8_t* sharpness_out) {
  if (!ctx || !src || !level_out || !sharpness_out) return VP8A_E_INVALID_ARGUMENT;
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  LfInputs L;
  vp8a_status s = stage_lf(ctx, st, planes, mbs, base, src, 0, false, &L);
  if (s != VP8A_OK) return s;
  void* dt;
  if ((s = st.scratch(512 * sizeof(uint64_t), &dt)) != VP8A_OK) return s;
  VP8A_CUDA(cudaMemsetAsync(dt, 0, 512 * sizeof(uint64_t), ctx->stream));
  L.a.ssd_out = (uint64_t*)dt;
  L.a.level0_unfiltered = 1;
  std::vector<uint64_t> t(512, 0);
  const uint8_t bs = base->sharpness_level > 7 ? 7 : base->sharpness_level;
  // Stage 1: grid 0, 4, ..., 60, 63 at the base sharpness.
  std::vector<uint8_t> c;
  for (int l = 0; l <= 60; l += 4) {
    c.push_back((uint8_t)l);
    c.push_back(bs);
  }
  c.push_back(63);
  c.push_back(bs);
  if ((s = score_candidates(ctx, st, L.a, dt, c, t.data())) != VP8A_OK) return s;
  uint8_t best_level = 0;
  uint64_t best = t[0 * 8 + bs];
  for (size_t i = 2; i < c.size(); i += 2)
    if (t[c[i] * 8 + bs] < best) {
      best = t[c[i] * 8 + bs];
      best_level = c[i];
    }
  // Refine +/-3 around the grid winner, excluding it.
  const int lo = best_level >= 3 ? best_level - 3 : 0, hi = std::min(63, best_level + 3);
  c.clear();
  for (int l = lo; l <= hi; l++)
    if (l != best_level) {
      c.push_back((uint8_t)l);
      c.push_back(bs);
    }
  if ((s = score_candidates(ctx, st, L.a, dt, c, t.data())) != VP8A_OK) return s;
  for (size_t i = 0; i < c.size(); i += 2)
    if (t[c[i] * 8 + bs] < best) {
      best = t[c[i] * 8 + bs];
      best_level = c[i];
    }
  if (best_level == 0) {
    const uint8_t zero = 0;
    if ((s = st.write_from_host(level_out, &zero, 1)) != VP8A_OK) return s;
    if ((s = st.write_from_host(sharpness_out, &bs, 1)) != VP8A_OK) return s;
      return st.finish();
  }
  // Stage 2: the other sharpness values at the chosen level.
  c.clear();
  for (int sh = 0; sh < 8; sh++)
    if (sh != bs) {
      c.push_back(best_level);
      c.push_back((uint8_t)sh);
    }
  if ((s = score_candidates(ctx, st, L.a, dt, c, t.data())) != VP8A_OK) return s;
  uint8_t best_sharp = bs;
  for (size_t i = 0; i < c.size(); i += 2)
    if (t[best_level * 8 + c[i + 1]] < best) {
      best = t[best_level * 8 + c[i + 1]];
      best_sharp = c[i + 1];
    }
  if ((s = st.write_from_host(level_out, &best_level, 1)) != VP8A_OK) return s;
  if ((s = st.write_from_host(sharpness_out, &best_sharp, 1)) != VP8A_OK) return s;
  return st.finish();
}

void vp8a_key_frame_sampling(uint32_t mb_rows, uint32_t* every_rows, uint32_t* sweep_sharpness) {
  // bands = clamp(mb_rows / 32, 3, 6); every_rows = max(mb_rows / bands, 2).
  const uint32_t bands = std::min<uint32_t>(std::max<uint32_t>(mb_rows / 32, 3), 6);
  if (every_rows) *every_rows = std::max<uint32_t>(mb_rows / bands, 2);
  if (sweep_sharpness) *sweep_sharpness = 1;
}

vp8a_status vp8a_select_filter_params_sampled(vp8a_ctx* ctx, const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                                              const vp8a_filter_config* base, const vp8a_source* src,
                                              uint32_t every_rows, uint32_t sweep_sharpness, uint8_t* level_out,
                                              uint8_t* sharpness_out) {
  if (!ctx || !src || !level_out || !sharpness_out) return VP8A_E_INVALID_ARGUMENT;
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  LfInputs L;
  const uint32_t er = every_rows < 2 ? 2 : every_rows;
  vp8a_status s = stage_lf(ctx, st, planes, mbs, base, src, er, false, &L);
  if (s != VP8A_OK) return s;
  void* dt;
  if ((s = st.scratch(512 * sizeof(uint64_t), &dt)) != VP8A_OK) return s;
  VP8A_CUDA(cudaMemsetAsync(dt, 0, 512 * sizeof(uint64_t), ctx->stream));
  L.a.ssd_out = (uint64_t*)dt;
  L.a.level0_unfiltered = 1;
  std::vector<uint64_t> t(512, 0);
  const uint8_t bs = base->sharpness_level > 7 ? 7 : base->sharpness_level;
  static const uint8_t coarse[9] = {0, 8, 16, 24, 32, 40, 48, 56, 63};
  std::vector<uint8_t> c;
  for (uint8_t l : coarse) {
    c.push_back(l);
    c.push_back(bs);
  }
  if ((s = score_candidates(ctx, st, L.a, dt, c, t.data())) != VP8A_OK) return s;
  uint8_t best_level = 0;
  uint64_t best = t[0 * 8 + bs];
  for (int i = 1; i < 9; i++)
    if (t[coarse[i] * 8 + bs] < best) {
      best = t[coarse[i] * 8 + bs];
      best_level = coarse[i];
    }
  for (uint8_t stp : {4, 2, 1}) {
    c.clear();
    if (best_level >= stp) {
      c.push_back((uint8_t)(best_level - stp));
      c.push_back(bs);
    }
    if (best_level + stp <= 63) {
      c.push_back((uint8_t)(best_level + stp));
      c.push_back(bs);
    }
    if ((s = score_candidates(ctx, st, L.a, dt, c, t.data())) != VP8A_OK) return s;
    uint8_t bl = best_level;
    for (size_t i = 0; i < c.size(); i += 2)
      if (t[c[i] * 8 + bs] < best) {
        best = t[c[i] * 8 + bs];
        bl = c[i];
      }
    best_level = bl;
  }
  uint8_t best_sharp = bs;
  if (sweep_sharpness && best_level != 0) {
    c.clear();
    for (int sh = 0; sh < 8; sh++)
      if (sh != bs) {
        c.push_back(best_level);
        c.push_back((uint8_t)sh);
      }
    if ((s = score_candidates(ctx, st, L.a, dt, c, t.data())) != VP8A_OK) return s;
    for (size_t i = 0; i < c.size(); i += 2)
      if (t[best_level * 8 + c[i + 1]] < best) {
        best = t[best_level * 8 + c[i + 1]];
        best_sharp = c[i + 1];
      }
  }
  if ((s = st.write_from_host(level_out, &best_level, 1)) != VP8A_OK) return s;
  if ((s = st.write_from_host(sharpness_out, &best_sharp, 1)) != VP8A_OK) return s;
  return st.finish();
}

// The sweep of vp8a_filter_sweep without any allocation: see the header.
vp8a_status vp8a_filter_sweep_noalloc(vp8a_ctx* ctx, const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                                      const vp8a_filter_config* base, const vp8a_source* src, uint32_t every_rows,
                                      uint64_t* ssd_out) {
  if (!ctx || !planes || !mbs || !base || !src || !ssd_out) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  const int cols = (int)planes->mb_cols, rows = (int)planes->mb_rows;
  if (cols < 1 || rows < 1 || cols > NA_MAX_MB_COLS || rows > NA_MAX_MB_ROWS) {
    vp8a::set_error("vp8a_filter_sweep_noalloc: the MB grid must be 1..256 columns by 1..136 rows "
                    "(its fixed scratch holds the schedule of at most 4096x2176 pixels)");
    return VP8A_E_INVALID_DIMENSIONS;
  }
  if (planes->y_stride < (uint64_t)cols * 16 || planes->uv_stride < (uint64_t)cols * 8) {
    vp8a::set_error("plane stride below the MB-padded width");
    return VP8A_E_INVALID_ARGUMENT;
  }
  vp8a_status s = validate_config(base);
  if (s != VP8A_OK) return s;
  if (src->width == 0 || src->height == 0 || src->width > (uint32_t)cols * 16 || src->height > (uint32_t)rows * 16) {
    vp8a::set_error("source size does not fit the MB grid");
    return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
  }
  const uint32_t cw = (src->width + 1) / 2;
  if (src->y_stride < src->width || src->uv_stride < cw) {
    vp8a::set_error("source stride below width");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  const void* bufs[8] = {planes->y, planes->u, planes->v, mbs, src->y, src->u, src->v, ssd_out};
  for (const void* b : bufs)
    if (!device_resident(b, ctx->device)) {
      vp8a::set_error("vp8a_filter_sweep_noalloc: every buffer must be device memory of the context's GPU "
                      "(this entry point stages nothing)");
      return VP8A_E_INVALID_ARGUMENT;
    }
  uint8_t* scr = nullptr;
  if ((s = sweep_scratch(ctx->device, &scr)) != VP8A_OK) return s;
  // Host-side schedule extent: steps and the busiest step's row count.
  const int max_t0 = every_rows == 0 ? 2 * (rows - 1) : (rows >= 2 ? 2 : 0);
  const int steps = max_t0 + cols;
  int max_active = 0;
  for (int t = 0; t < steps; t++) {
    int n = 0;
    for (int r = 0; r < rows; r++) {
      int v;
      if (every_rows == 0) {
        v = 2 * r;
      } else {
        const int step = every_rows < 2 ? 2 : (int)every_rows, k = r % step;
        v = k < 2 ? 2 * k : -1;
      }
      n += v >= 0 && t >= v && t < v + cols;
    }
    max_active = std::max(max_active, n);
  }
  NaGrid grid{};
  grid.n = grid_passes(*base, grid.pairs, grid.masks);  // <= NA_CANDIDATES
  sweep_schedule_kernel<<<1, 1024, 0, ctx->stream>>>(scr, rows, cols, (int)every_rows, steps, grid);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;

  LfArgs a{};
  a.y = (const uint8_t*)planes->y;
  a.u = (const uint8_t*)planes->u;
  a.v = (const uint8_t*)planes->v;
  a.ys = planes->y_stride;
  a.cs = planes->uv_stride;
  a.mb_cols = cols;
  a.mb_rows = rows;
  a.mbs = mbs;
  a.base = *base;
  a.sy = (const uint8_t*)src->y;
  a.su = (const uint8_t*)src->u;
  a.sv = (const uint8_t*)src->v;
  a.sys = src->y_stride;
  a.scs = src->uv_stride;
  a.width = (int)src->width;
  a.height = (int)src->height;
  a.cands = scr + NA_CANDS;
  a.cand_mask = scr + NA_MASK;
  a.row_t0 = (const int16_t*)(scr + NA_T0);
  a.row_top = scr + NA_TOP;
  a.sched_off = (const int32_t*)(scr + NA_OFF);
  a.sched_row = (const uint16_t*)(scr + NA_ROWS);
  a.steps = steps;
  a.max_active = max_active;
  auto al4 = [](const void* p, uint64_t stride) { return ((uintptr_t)p % 4 == 0) && (stride % 4 == 0); };
  a.recon_words = al4(a.y, a.ys) && al4(a.u, a.cs) && al4(a.v, a.cs);
  a.source_words = al4(a.sy, a.sys) && al4(a.su, a.scs) && al4(a.sv, a.scs);
  a.ssd_out = ssd_out;
  a.level0_unfiltered = 1;
  a.smem_slots = 1;
  a.gslots = nullptr;
  // The level-0 pass writes all eight sharpness entries itself.
  return run_sweep(ctx, a, grid.n, nullptr);
}

}  // extern "C"
