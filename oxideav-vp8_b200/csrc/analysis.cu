// analysis.cu — the exhaustive inter analysis of a P frame on the device.
//
// vp8a_analyse_inter_frame replaces analyse_inter_frame
// (src/encoder/inter.rs:263) with decide_mb_exhaustive (:537) and intra
// picking off: per MB, every reference runs pick_mb_for_ref's search and
// mode decision (src/encoder.rs:8546-8702: census, ZEROMV SAD, diamond,
// half/quarter refinement, NEAREST/NEAR SADs, SPLITMV partitions), the
// references are compared on J + ref_frame_tree_bits, and the winner's
// census record feeds later MBs.
//
// Scheduling. The census makes MB (r, c) depend on (r, c-1), (r-1, c) and
// (r-1, c-1); the reference's wavefront lets row r run while row r-1 is two
// MBs ahead (src/encoder/inter.rs:376-379). Here a persistent grid of
// co-resident CTAs owns MB rows round-robin; a CTA processes its rows left
// to right and, before MB (r, c), waits until row r-1 has published
// min(c+2, mb_cols) MBs. Rows are claimed in increasing order and every
// waited-on row belongs to a resident CTA, so the wait always ends; it is
// still bounded, and a wait that runs out sets the device status word and
// the whole grid returns (VP8A_E_DEVICE_TIMEOUT on the host).
//
// Per MB, one staging phase fetches (edge-clamped, all loads in flight
// together) everything the searches read: per reference the search window
// around the predictor, the NEAREST/NEAR six-tap halos and the 16x16
// blocks at the ZERO and neighbour vectors. Then each reference gets one
// "main" warp (ZEROMV, diamond, half via shared half-pel planes, quarter,
// NEAREST, NEAR) and four SPLITMV warps (one per partition, groups in
// parallel across lanes). The f64 RD decision runs on one thread with the
// reference's operation order; the library is built with -fmad=false so no
// multiply-add is fused.
#include <cstddef>

#include "census.cuh"

namespace {
using namespace vp8a_dev;


constexpr int MAX_REFS = 3;
constexpr int WARPS_PER_REF = 5;

struct AnArgs {
  const uint8_t* fy;
  uint64_t fys;
  int fw, fh;
  MePlane refs[MAX_REFS];
  uint8_t ref_ids[MAX_REFS];
  int n_refs;
  int mb_cols, mb_rows;
  vp8a_mv_contexts ctx;
  double lambda;
  const double* bit_cost;
  const double* mvbits;  // mv_component_bits per context and value (2 x 2047)
  MbInfoDev* infos;
  unsigned* progress;
  unsigned* status;
  vp8a_mb_decision* dec;
  vp8a_ref_search* trace;
  unsigned long long spin_limit;
};

// ------------------------------------------------------------- staging

// Regions staged per (MB, reference) before any search runs: the 40x40
// search window around the predictor, the 21x21 six-tap halos of the
// NEAREST and NEAR vectors, and 16x16 blocks at the integer offsets of the
// ZERO vector and of the left/above neighbours' vectors (the SPLITMV
// LEFT4X4 / ABOVE4X4 / ZERO4X4 candidates). Every byte is fetched
// edge-clamped, so later reads need no bounds checks.
constexpr int HS = 24;        // halo stride
constexpr int MAX_BLOCKS = 9; // zero + 4 left + 4 above offsets
constexpr int CMAX = 25;      // SPLITMV candidate vectors per partition

struct __align__(16) RefSmem {
  WarpScratch ws;                       // window + six-tap scratch + half planes
  uint8_t halo_nearest[21 * HS + 8];    // 512
  uint8_t halo_near[21 * HS + 8];       // 512
  uint8_t blocks[MAX_BLOCKS][256];      // read as 32-bit words (sad_block16)
};
static_assert(sizeof(RefSmem) % 16 == 0 && offsetof(RefSmem, blocks) % 16 == 0, "RefSmem alignment");

struct MainOut {
  uint32_t sad_zero, sad_nearest, sad_near;
  vp8a_search_result whole, half, quarter;
};

// One reference's mode decision (pick_mb_for_ref's result).
struct RefDec {
  double j, total;
  vp8a_mv mv;
  int mode, pid;
};

struct SplitOut {
  double j;
  vp8a_mv split_mvs[16];
  uint8_t modes[16];
  int valid;
};

// SPLITMV scratch of one warp. Candidate column layout (fixed, no
// de-duplication): 0 = ZERO, 1..4 = LEFT vectors of the MB's left column
// anchors 0/4/8/12, 5..8 = ABOVE vectors of the top-row anchors 0..3,
// 9..24 = the NEW4X4 result of group 0..15.
struct SplitScratch {
  uint32_t table[16 * CMAX];  // group g's SAD at column m: table[g * CMAX + m]
  vp8a_mv cmv[CMAX];
  double new_bits[16];        // NEW4X4 vector bits of group g (when new_ok)
  uint32_t new_sad[16];
  uint8_t new_ok[16];         // group g's NEW differential lies in [-1023, 1023]
  uint8_t chosen[16];         // column each group chose
};
struct Plan {
  int wx0, wy0;        // window origin (plane pixels)
  int hn_x, hn_y;      // NEAREST halo origin
  int hr_x, hr_y;      // NEAR halo origin
  int nblocks;
  int box[MAX_BLOCKS], boy[MAX_BLOCKS];  // block integer offsets
};

// Geometry of SPLITMV group g of partition p (PartitionGroups::build,
// src/encoder.rs:7912-7980): row0, col0, width, height, anchor.
__constant__ int8_t c_geom[4][16][5] = {
    {{0, 0, 16, 8, 0}, {8, 0, 16, 8, 8}},
    {{0, 0, 8, 16, 0}, {0, 8, 8, 16, 2}},
    {{0, 0, 8, 8, 0}, {0, 8, 8, 8, 2}, {8, 0, 8, 8, 8}, {8, 8, 8, 8, 10}},
    {{0, 0, 4, 4, 0},   {0, 4, 4, 4, 1},   {0, 8, 4, 4, 2},   {0, 12, 4, 4, 3},
     {4, 0, 4, 4, 4},   {4, 4, 4, 4, 5},   {4, 8, 4, 4, 6},   {4, 12, 4, 4, 7},
     {8, 0, 4, 4, 8},   {8, 4, 4, 4, 9},   {8, 8, 4, 4, 10},  {8, 12, 4, 4, 11},
     {12, 0, 4, 4, 12}, {12, 4, 4, 4, 13}, {12, 8, 4, 4, 14}, {12, 12, 4, 4, 15}}};

__device__ __forceinline__ int int_off(int16_t v) { return eighth(v) >> 3; }

// External LEFT4X4 / ABOVE4X4 vectors (left_block_mv / above_block_mv for
// anchors on the MB's left column / top row, src/near_mv.rs:722-760).
__device__ __forceinline__ vp8a_mv ext_left(const MbInfoDev& l, int anchor) {
  if (l.ref_frame == VP8A_REF_INTRA) return vp8a_mv{0, 0};
  return l.is_split ? l.split_mvs[anchor + 3] : l.mv;
}
__device__ __forceinline__ vp8a_mv ext_above(const MbInfoDev& a, int anchor) {
  if (a.ref_frame == VP8A_REF_INTRA) return vp8a_mv{0, 0};
  return a.is_split ? a.split_mvs[anchor + 12] : a.mv;
}

// Stage every region of every reference; each thread keeps up to BATCH
// loads in flight before storing.
template <int BATCH>
__device__ void stage(const AnArgs& a, RefSmem* rs, const Plan& pl, int mbx, int mby, int tid, int nthreads) {
  const int per_ref = 40 * 40 + 2 * 441 + pl.nblocks * 256;
  const int total = a.n_refs * per_ref;
  for (int base = tid; base < total; base += nthreads * BATCH) {
    uint8_t v[BATCH];
    uint8_t* d[BATCH];
#pragma unroll
    for (int j = 0; j < BATCH; j++) {
      const int e = base + j * nthreads;
      d[j] = nullptr;
      if (e < total) {
        const int k = e < per_ref ? 0 : (e < 2 * per_ref ? 1 : 2);
        const int rem = e - k * per_ref;
        const MePlane& P = a.refs[k];
        int x, y;
        if (rem < 1600) {
          const int r = rem / 40, c = rem - r * 40;
          x = pl.wx0 + c;
          y = pl.wy0 + r;
          d[j] = rs[k].ws.win + r * WS + c;
        } else if (rem < 1600 + 2 * 441) {
          const int q = rem - 1600, h = q >= 441, qq = q - h * 441;
          const int r = qq / 21, c = qq - r * 21;
          x = (h ? pl.hr_x : pl.hn_x) + c;
          y = (h ? pl.hr_y : pl.hn_y) + r;
          d[j] = (h ? rs[k].halo_near : rs[k].halo_nearest) + r * HS + c;
        } else {
          const int q = rem - 1600 - 2 * 441, b = q >> 8, r = (q >> 4) & 15, c = q & 15;
          x = mbx + pl.box[b] + c;
          y = mby + pl.boy[b] + r;
          d[j] = rs[k].blocks[b] + r * 16 + c;
        }
        v[j] = P.plane[(size_t)clampi(y, 0, P.height - 1) * P.stride + clampi(x, 0, P.width - 1)];
      }
    }
#pragma unroll
    for (int j = 0; j < BATCH; j++)
      if (d[j]) *d[j] = v[j];
  }
}

// -------------------------------------------------------------- SPLITMV

// Columns of the candidate table each partition needs (see SplitScratch):
// ZERO, the LEFT/ABOVE vectors of its left-column / top-row anchors, and
// its groups' NEW results.
__constant__ uint32_t c_need_cols[4] = {
    (1u << 0) | (1u << 1) | (1u << 3) | (1u << 5) | (0x3u << 9),   // TopBottom: anchors 0, 8
    (1u << 0) | (1u << 1) | (1u << 5) | (1u << 7) | (0x3u << 9),   // LeftRight: anchors 0, 2
    (1u << 0) | (1u << 1) | (1u << 3) | (1u << 5) | (1u << 7) | (0xfu << 9),  // Quarters: 0, 2, 8, 10
    0x1ffffffu};                                                   // Mv16: every column

// Unaligned 4-byte read from shared memory.
__device__ __forceinline__ uint32_t load4u(const uint8_t* p) {
  uintptr_t a = (uintptr_t)p;
  const uint32_t* w = (const uint32_t*)(a & ~(uintptr_t)3);
  return __funnelshift_r(w[0], w[1], (unsigned)(a & 3) * 8u);
}

// This lane's 8 pixels of its group: one run of 8 (groups 8 or 16 wide) or
// two rows of 4 (4x4 groups). off0/off1 are (row*stride + col) with the
// row/col in MB coordinates.
struct LanePix {
  int r0, c0, r1, c1;
  bool wide;
  uint32_t s0, s1;  // the source bytes as two little-endian words
};

__device__ __forceinline__ LanePix lane_pixels(int row0, int col0, int gw, int s, const uint8_t* src) {
  LanePix p;
  if (gw == 16) {
    p.r0 = row0 + (s >> 1);
    p.c0 = col0 + (s & 1) * 8;
    p.wide = true;
  } else if (gw == 8) {
    p.r0 = row0 + s;
    p.c0 = col0;
    p.wide = true;
  } else {
    p.r0 = row0 + 2 * s;
    p.c0 = col0;
    p.wide = false;
  }
  p.r1 = p.wide ? p.r0 : p.r0 + 1;
  p.c1 = p.wide ? p.c0 + 4 : p.c0;
  p.s0 = *(const uint32_t*)(src + p.r0 * 16 + p.c0);
  p.s1 = *(const uint32_t*)(src + p.r1 * 16 + p.c1);
  return p;
}

// Partial SAD of this lane's pixels for the MB-extent block whose top-left
// is plane pixel (bx, by): from the window, a staged block, or clamped
// global loads.
__device__ __forceinline__ uint32_t lane_gsad(const MePlane& P, const RefSmem& R, const Plan& pl, int mbx, int mby,
                                              const LanePix& q, int bx, int by) {
  const int lx = bx - pl.wx0, ly = by - pl.wy0;
  const uint8_t* base = nullptr;
  int st = 0;
  if (lx >= 0 && ly >= 0 && lx + 16 <= WS && ly + 16 <= WS) {
    base = R.ws.win + ly * WS + lx;
    st = WS;
  } else {
    for (int b = 0; b < pl.nblocks; b++)
      if (mbx + pl.box[b] == bx && mby + pl.boy[b] == by) {
        base = R.blocks[b];
        st = 16;
        break;
      }
  }
  uint32_t r0, r1;
  if (base) {
    r0 = load4u(base + q.r0 * st + q.c0);
    r1 = load4u(base + q.r1 * st + q.c1);
  } else {
    r0 = r1 = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const uint32_t b0 =
          P.plane[(size_t)clampi(by + q.r0, 0, P.height - 1) * P.stride + clampi(bx + q.c0 + i, 0, P.width - 1)];
      const uint32_t b1 =
          P.plane[(size_t)clampi(by + q.r1, 0, P.height - 1) * P.stride + clampi(bx + q.c1 + i, 0, P.width - 1)];
      r0 |= b0 << (8 * i);
      r1 |= b1 << (8 * i);
    }
  }
  return __vsadu4(r0, q.s0) + __vsadu4(r1, q.s1);
}

__device__ __forceinline__ uint32_t group_reduce(uint32_t v, int L) {
  for (int o = L >> 1; o >= 1; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

__device__ __forceinline__ double submv_ref_bits(const double* t, const uint8_t* p, int mode) {
  switch (mode) {
    case VP8A_SUBMV_LEFT: return bb(t, p[0], 0);
    case VP8A_SUBMV_ABOVE: return bb(t, p[0], 1) + bb(t, p[1], 0);
    case VP8A_SUBMV_ZERO: return bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 0);
    default: return bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 1);
  }
}

__device__ __forceinline__ double mv_partition_bits(const double* t, int pid) {
  const uint8_t* p = c_partition_probs;
  switch (pid) {
    case VP8A_PART_MV16: return bb(t, p[0], 0);
    case VP8A_PART_QUARTERS: return bb(t, p[0], 1) + bb(t, p[1], 0);
    case VP8A_PART_TOP_BOTTOM: return bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 0);
    default: return bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 1);
  }
}

// score_split_partition (src/encoder.rs:8080-8246) on one warp. Groups run
// in parallel (32/G lanes each) for their NEW4X4 diamonds and for a table
// of group SADs at every vector the sub-MV choice can consider (ZERO, the
// external neighbours' vectors, every group's NEW result); the sequential
// LEFT/ABOVE/ZERO/NEW choice over groups then reads that table.
//
// The per-group costs that do not depend on the chain are computed before
// it: sbits[ctx * 4 + mode] = submv_ref_bits of each context and mode, and
// each group's NEW vector bits. Every value is the same expression the
// reference evaluates, so the chain's sums are unchanged.
__device__ void split_partition(const AnArgs& a, const double* t, const double* sbits, const MePlane& P,
                                const RefSmem& R, const Plan& pl, int mbx, int mby, const uint8_t* src, vp8a_mv bp,
                                const MbInfoDev& above, const MbInfoDev& left, int pid, SplitScratch& W,
                                SplitOut* out, int lane) {
  const int G = pid == 3 ? 16 : (pid == 2 ? 4 : 2);
  const int L = 32 / G, g = lane / L, s = lane - g * L;
  const int row0 = c_geom[pid][g][0], col0 = c_geom[pid][g][1], gw = c_geom[pid][g][2];
  const LanePix q = lane_pixels(row0, col0, gw, s, src);
  // group_small_diamond_search (src/encoder.rs:7812-7879) for every group
  // at once: snap then clamp the centre; N, S, W, E clamped, not snapped.
  vp8a_mv best;
  best.row = (int16_t)clampi((bp.row / 4) * 4, -1023, 1023);
  best.col = (int16_t)clampi((bp.col / 4) * 4, -1023, 1023);
  uint32_t bs = group_reduce(lane_gsad(P, R, pl, mbx, mby, q, mbx + int_off(best.col), mby + int_off(best.row)), L);
  bool active = true;
  for (int it = 0; it < 4; it++) {
    bool improved = false;
    const int dr[4] = {-4, 4, 0, 0}, dc[4] = {0, 0, -4, 4};
#pragma unroll
    for (int d = 0; d < 4; d++) {
      vp8a_mv c;
      c.row = (int16_t)clampi(best.row + dr[d], -1023, 1023);
      c.col = (int16_t)clampi(best.col + dc[d], -1023, 1023);
      const uint32_t sv =
          group_reduce(lane_gsad(P, R, pl, mbx, mby, q, mbx + int_off(c.col), mby + int_off(c.row)), L);
      if (active && !mv_eq(c, best) && sv < bs) {
        bs = sv;
        best = c;
        improved = true;
      }
    }
    if (!improved) active = false;
  }
  // Candidate columns.
  if (s == 0) {
    W.cmv[9 + g] = best;
    W.new_sad[g] = bs;
    const int dr = (int)best.row - bp.row, dc = (int)best.col - bp.col;
    const bool ok = dr >= -1023 && dr <= 1023 && dc >= -1023 && dc <= 1023;
    W.new_ok[g] = ok;
    W.new_bits[g] = ok ? mv_bits_lookup(a.mvbits, 0, dr) + mv_bits_lookup(a.mvbits, 1, dc) : 0.0;
  }
  if (lane == 0) {
    W.cmv[0] = vp8a_mv{0, 0};
    for (int k = 0; k < 4; k++) W.cmv[1 + k] = ext_left(left, 4 * k);
    for (int k = 0; k < 4; k++) W.cmv[5 + k] = ext_above(above, k);
  }
  __syncwarp();
  const uint32_t need = c_need_cols[pid];
  for (int m = 0; m < CMAX; m++) {
    if (!((need >> m) & 1u)) continue;
    const vp8a_mv mv = W.cmv[m];
    const uint32_t sv = group_reduce(lane_gsad(P, R, pl, mbx, mby, q, mbx + int_off(mv.col), mby + int_off(mv.row)), L);
    if (s == 0) W.table[g * CMAX + m] = sv;
  }
  __syncwarp();
  // The sequential sub-MV choice (uniform on every lane; lane 0 records).
  uint32_t total_sad = 0;
  double total_bits = 0.0;
  for (int gg = 0; gg < G; gg++) {
    const int anchor = c_geom[pid][gg][4];
    const int lidx = (anchor & 3) == 0 ? 1 + (anchor >> 2) : W.chosen[c_partitions[pid][anchor - 1]];
    const int aidx = anchor < 4 ? 5 + anchor : W.chosen[c_partitions[pid][anchor - 4]];
    const vp8a_mv lmv = W.cmv[lidx], amv = W.cmv[aidx];
    const bool lez = mv_zero(lmv), aez = mv_zero(amv), lea = mv_eq(lmv, amv);
    const int ctxi = (lea && lez) ? 4 : (lea ? 3 : (aez ? 2 : (lez ? 1 : 0)));
    const double* mb = sbits + ctxi * 4;
    const uint32_t* trow = W.table + gg * CMAX;
    // LEFT, ABOVE, ZERO, then NEW; strict '<' keeps the first minimum.
    const double j0 = (double)trow[lidx] + a.lambda * (mb[0] + 0.0);
    const double j1 = (double)trow[aidx] + a.lambda * (mb[1] + 0.0);
    const double j2 = (double)trow[0] + a.lambda * (mb[2] + 0.0);
    double best_j = __longlong_as_double(0x7ff0000000000000LL);
    int best_mode = VP8A_SUBMV_ZERO, best_col = 0;
    if (j0 < best_j) {
      best_j = j0;
      best_mode = VP8A_SUBMV_LEFT;
      best_col = lidx;
    }
    if (j1 < best_j) {
      best_j = j1;
      best_mode = VP8A_SUBMV_ABOVE;
      best_col = aidx;
    }
    if (j2 < best_j) {
      best_j = j2;
      best_mode = VP8A_SUBMV_ZERO;
      best_col = 0;
    }
    if (W.new_ok[gg]) {
      const double jn = (double)W.new_sad[gg] + a.lambda * (mb[3] + W.new_bits[gg]);
      if (jn < best_j) {
        best_j = jn;
        best_mode = VP8A_SUBMV_NEW;
        best_col = 9 + gg;
      }
    }
    if (!isfinite(best_j)) {
      if (lane == 0) out->valid = 0;
      return;
    }
    total_sad += trow[best_col];
    total_bits += mb[best_mode];
    if (best_mode == VP8A_SUBMV_NEW) total_bits += W.new_bits[gg];
    __syncwarp();
    if (lane == 0) {
      W.chosen[gg] = (uint8_t)best_col;
      out->modes[gg] = (uint8_t)best_mode;
    }
    __syncwarp();
  }
  const double partition_bits = mv_partition_bits(t, pid);
  if (lane == 0) {
    out->j = (double)total_sad + a.lambda * (partition_bits + total_bits);
    for (int i = G; i < 16; i++) out->modes[i] = VP8A_SUBMV_ZERO;
    out->valid = 1;
  }
  if (lane < 16) out->split_mvs[lane] = W.cmv[W.chosen[c_partitions[pid][lane]]];
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// SAD of the 16x16 source against a staged 16x16 block.
__device__ __forceinline__ uint32_t sad_block16(const uint8_t* blk, const uint8_t* src, int lane) {
  const int row = lane >> 1, c0 = (lane & 1) * 8;
  const uint32_t* b = (const uint32_t*)(blk + row * 16 + c0);
  const uint32_t* sp = (const uint32_t*)(src + row * 16 + c0);
  return __reduce_add_sync(FULL, __vsadu4(b[0], sp[0]) + __vsadu4(b[1], sp[1]));
}

__global__ void __launch_bounds__(MAX_REFS* WARPS_PER_REF * 32) analysis_kernel(AnArgs a) {
  __shared__ RefSmem rs[MAX_REFS];
  __shared__ SplitScratch ss[MAX_REFS * 4];
  __shared__ __align__(16) uint8_t src[256];
  __shared__ double bit_cost[256];
  __shared__ double sbits[5 * 4];  // submv_ref_bits per context and mode
  __shared__ MainOut mains[MAX_REFS];
  __shared__ SplitOut splits[MAX_REFS][4];
  __shared__ RefDec decs[MAX_REFS];
  __shared__ MbInfoDev nb[3];  // above, left, aboveleft
  __shared__ Census cen;
  __shared__ Plan plan;
  __shared__ int s_abort;
  const int tid = threadIdx.x, nthreads = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int ref = warp / WARPS_PER_REF, role = warp % WARPS_PER_REF;  // role 0 = main, 1..4 = split pid
  for (int i = tid; i < 256; i += nthreads) bit_cost[i] = a.bit_cost[i];
  __syncthreads();
  if (tid < 20) sbits[tid] = submv_ref_bits(bit_cost, c_submv_probs[tid >> 2], tid & 3);
  const MbInfoDev border = {VP8A_REF_INTRA, 0, 0, 0, {0, 0}, {}};

  for (int r = blockIdx.x; r < a.mb_rows; r += gridDim.x) {
    for (int c = 0; c < a.mb_cols; c++) {
      if (tid == 0) {
        int abort = 0;
        if (r > 0) {
          const unsigned need = (unsigned)min(c + 2, a.mb_cols);
          unsigned long long it = 0;
          while (ld_acquire(&a.progress[r - 1]) < need) {
            if (*(volatile unsigned*)a.status != 0u || ++it > a.spin_limit) {
              atomicCAS(a.status, 0u, (unsigned)vp8a::DEV_TIMEOUT);
              abort = 1;
              break;
            }
            __nanosleep(64);
          }
        } else if (*(volatile unsigned*)a.status != 0u) {
          abort = 1;
        }
        s_abort = abort;
      }
      __syncthreads();
      if (s_abort) return;
      // Neighbour records and the edge-replicated source MB
      // (extract_mb, src/encoder.rs:5549).
      if (tid < 3) {
        const int nr = tid == 1 ? r : r - 1, nc = tid == 0 ? c : c - 1;
        nb[tid] = (nr >= 0 && nc >= 0) ? a.infos[(size_t)nr * a.mb_cols + nc] : border;
      }
      if (tid < 256) {
        const int y = min(r * 16 + (tid >> 4), a.fh - 1), x = min(c * 16 + (tid & 15), a.fw - 1);
        src[tid] = a.fy[(size_t)y * a.fys + x];
      }
      __syncthreads();
      const int mbx = c * 16, mby = r * 16;
      if (tid == 0) {
        cen = census(nb[0], nb[1], nb[2], c, r, a.mb_cols, a.mb_rows);
        Plan p;
        const vp8a_mv bp = cen.best_predictor;
        p.wx0 = mbx + snap_whole(clamp_component(bp.col)) / 4 - WIN_LEAD;
        p.wy0 = mby + snap_whole(clamp_component(bp.row)) / 4 - WIN_LEAD;
        p.hn_x = mbx + int_off(cen.nearest.col) - 2;
        p.hn_y = mby + int_off(cen.nearest.row) - 2;
        p.hr_x = mbx + int_off(cen.near_.col) - 2;
        p.hr_y = mby + int_off(cen.near_.row) - 2;
        p.nblocks = 0;
        auto addb = [&](vp8a_mv m) {
          const int ox = int_off(m.col), oy = int_off(m.row);
          for (int i = 0; i < p.nblocks; i++)
            if (p.box[i] == ox && p.boy[i] == oy) return;
          p.box[p.nblocks] = ox;
          p.boy[p.nblocks] = oy;
          p.nblocks++;
        };
        addb(vp8a_mv{0, 0});
        for (int anc = 0; anc < 16; anc += 4) addb(ext_left(nb[1], anc));
        for (int anc = 0; anc < 4; anc++) addb(ext_above(nb[0], anc));
        plan = p;
      }
      __syncthreads();
      stage<24>(a, rs, plan, mbx, mby, tid, nthreads);
      __syncthreads();
      if (ref < a.n_refs) {
        const MePlane& P = a.refs[ref];
        RefSmem& R = rs[ref];
        const vp8a_mv bp = cen.best_predictor;
        if (role == 0) {
          MainOut m;
          m.sad_zero = sad_block16(R.blocks[0], src, lane);
          m.whole = diamond(P, R.ws, plan.wx0, plan.wy0, mbx, mby, bp, 8, src, lane);
          if (!half_refine_planes(R.ws, plan.wx0, plan.wy0, mbx, mby, m.whole.mv, src, lane, &m.half))
            m.half = refine(P, R.ws, plan.wx0, plan.wy0, mbx, mby, m.whole.mv, 2, src, lane);
          m.quarter = refine(P, R.ws, plan.wx0, plan.wy0, mbx, mby, m.half.mv, 1, src, lane, m.half.sad);
          const int en_r = eighth(cen.nearest.row), en_c = eighth(cen.nearest.col);
          m.sad_nearest = subpel_sad(R.halo_nearest, HS, en_c & 7, en_r & 7, src, R.ws.temp, lane);
          const int er_r = eighth(cen.near_.row), er_c = eighth(cen.near_.col);
          m.sad_near = subpel_sad(R.halo_near, HS, er_c & 7, er_r & 7, src, R.ws.temp, lane);
          if (lane == 0) mains[ref] = m;
        } else {
          split_partition(a, bit_cost, sbits, P, R, plan, mbx, mby, src, bp, nb[0], nb[1], role - 1,
                          ss[ref * 4 + role - 1], &splits[ref][role - 1], lane);
        }
      }
      if (ref < a.n_refs) {
        // The reference's five warps meet; its main warp's lane 0 decides
        // its mode (pick_mb_for_ref, src/encoder.rs:8598-8652).
        asm volatile("bar.sync %0, %1;" ::"r"(1 + ref), "r"(WARPS_PER_REF * 32) : "memory");
        if (role == 0 && lane == 0) {
          const int k = ref;
          const double* t = bit_cost;
          const double lambda = a.lambda;
          const uint8_t* p = cen.p;
          const vp8a_mv bp = cen.best_predictor;
          const MainOut& m = mains[k];
          const double bits_zero = bb(t, p[0], 0);
          const double bits_nearest = bb(t, p[0], 1) + bb(t, p[1], 0);
          const double bits_near = bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 0);
          const double bits_new = bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 1) + bb(t, p[3], 0);
          const int dr = (int)m.quarter.mv.row - bp.row, dc = (int)m.quarter.mv.col - bp.col;
          const bool in_range = dr >= -1023 && dr <= 1023 && dc >= -1023 && dc <= 1023;
          const double bits_mv = in_range ? mv_bits_lookup(a.mvbits, 0, dr) + mv_bits_lookup(a.mvbits, 1, dc)
                                          : __longlong_as_double(0x7ff0000000000000LL);
          const double j_zero = (double)m.sad_zero + lambda * bits_zero;
          const double j_nearest = (double)m.sad_nearest + lambda * bits_nearest;
          const double j_near = (double)m.sad_near + lambda * bits_near;
          const double j_new = (double)m.quarter.sad + lambda * (bits_new + bits_mv);
          int mode = VP8A_MODE_ZERO, pid = VP8A_PART_NONE;
          vp8a_mv mv = {0, 0};
          double cj = j_zero;
          if (!mv_zero(cen.nearest) && j_nearest < cj) {
            mode = VP8A_MODE_NEAREST;
            mv = cen.nearest;
            cj = j_nearest;
          }
          if (!mv_zero(cen.near_) && j_near < cj) {
            mode = VP8A_MODE_NEAR;
            mv = cen.near_;
            cj = j_near;
          }
          if (in_range && !mv_zero(m.quarter.mv) && j_new < cj) {
            mode = VP8A_MODE_NEW;
            mv = m.quarter.mv;
            cj = j_new;
          }
          const double bits_split = bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 1) + bb(t, p[3], 1);
          int have = 0, sp = -1;
          double sj = 0.0;
          for (int qq = 0; qq < 4; qq++) {
            if (!splits[k][qq].valid) continue;
            const double total_j = splits[k][qq].j + lambda * bits_split;
            // The stored best already includes bits_split and the
            // comparison adds it again (src/encoder.rs:8679-8683).
            if (!have || total_j < sj + lambda * bits_split) {
              sj = total_j;
              sp = qq;
              have = 1;
            }
          }
          if (have && sj < cj) {
            mode = VP8A_MODE_SPLIT;
            mv = splits[k][sp].split_mvs[15];
            cj = sj;
            pid = sp;
          }
          // ref_frame_tree_bits(ref, 128, 128) (src/encoder.rs:9108).
          const uint8_t id = a.ref_ids[k];
          const double rbits = id == VP8A_REF_LAST ? bb(t, 128, 0)
                               : id == VP8A_REF_GOLDEN ? bb(t, 128, 1) + bb(t, 128, 0)
                                                       : bb(t, 128, 1) + bb(t, 128, 1);
          const double total = cj + lambda * rbits;
          if (a.trace) {
            vp8a_ref_search tr;
            tr.best_predictor = bp;
            tr.nearest_mv = cen.nearest;
            tr.near_mv = cen.near_;
            tr.sad_zero = m.sad_zero;
            tr.whole = m.whole;
            tr.half = m.half;
            tr.quarter = m.quarter;
            tr.sad_nearest = m.sad_nearest;
            tr.sad_near = m.sad_near;
            tr.chosen_mode = (uint8_t)mode;
            tr.split_partition = (uint8_t)pid;
            tr.reserved[0] = tr.reserved[1] = 0;
            tr.j = cj;
            a.trace[((size_t)r * a.mb_cols + c) * a.n_refs + k] = tr;
          }
          decs[k] = RefDec{cj, total, mv, mode, pid};
        }
      }
      __syncthreads();
      if (tid == 0) {
        // decide_mb_exhaustive's reference comparison: first strict minimum
        // of J + ref_frame_tree_bits in reference order.
        double best_total = __longlong_as_double(0x7ff0000000000000LL);
        int best_k = -1, best_mode = 0, best_pid = VP8A_PART_NONE;
        vp8a_mv best_mv = {0, 0};
        double best_j = 0.0;
        for (int k = 0; k < a.n_refs; k++) {
          const RefDec& rd = decs[k];
          if (rd.total < best_total) {
            best_total = rd.total;
            best_k = k;
            best_mode = rd.mode;
            best_mv = rd.mv;
            best_j = rd.j;
            best_pid = rd.pid;
          }
        }
        vp8a_mb_decision d;
        memset(&d, 0, sizeof d);
        MbInfoDev info;
        memset(&info, 0, sizeof info);
        if (best_k >= 0) {
          d.ref_frame = a.ref_ids[best_k];
          d.mode = (uint8_t)best_mode;
          d.partition = (uint8_t)best_pid;
          d.mv = best_mv;
          d.j = best_j;
          d.total = best_total;
          for (int i = 0; i < 16; i++) {
            d.split_mvs[i] = best_mode == VP8A_MODE_SPLIT ? splits[best_k][best_pid].split_mvs[i] : vp8a_mv{0, 0};
            d.submv_modes[i] = best_mode == VP8A_MODE_SPLIT ? splits[best_k][best_pid].modes[i] : (uint8_t)VP8A_SUBMV_ZERO;
          }
          info.ref_frame = d.ref_frame;
          info.mv = best_mv;
          info.is_split = best_mode == VP8A_MODE_SPLIT;
          info.has_split_mvs = info.is_split;
          for (int i = 0; i < 16; i++) info.split_mvs[i] = d.split_mvs[i];
        }
        a.dec[(size_t)r * a.mb_cols + c] = d;
        a.infos[(size_t)r * a.mb_cols + c] = info;
        __threadfence();
        st_release(&a.progress[r], (unsigned)(c + 1));
      }
      // The next MB's first barrier orders these shared results.
    }
  }
}

}  // namespace

extern "C" vp8a_status vp8a_analyse_inter_frame(vp8a_ctx* ctx, const vp8a_i420* frame, const vp8a_planes* refs,
                                                const uint8_t* ref_ids, uint32_t n_refs,
                                                const vp8a_mv_contexts* mv_contexts, double lambda,
                                                vp8a_mb_decision* decisions, vp8a_ref_search* trace) {
  if (!ctx || !frame || !refs || !ref_ids || !decisions) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (frame->width == 0 || frame->height == 0 || frame->width > 0x3FFF || frame->height > 0x3FFF) {
    vp8a::set_error("invalid dimensions");
    return VP8A_E_INVALID_DIMENSIONS;
  }
  if (n_refs == 0 || n_refs > (uint32_t)MAX_REFS) {
    vp8a::set_error("n_refs must be 1..3");
    return VP8A_E_INVALID_ARGUMENT;
  }
  const int mb_cols = (int)((frame->width + 15) / 16), mb_rows = (int)((frame->height + 15) / 16);
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  vp8a_status s;
  // The reference ids steer host-side validation; fetch them wherever they live.
  uint8_t ids[MAX_REFS];
  if ((s = st.read_to_host(ref_ids, n_refs, ids)) != VP8A_OK) return s;
  ref_ids = ids;
  for (uint32_t k = 0; k < n_refs; k++) {
    if ((int)refs[k].mb_cols != mb_cols || (int)refs[k].mb_rows != mb_rows) {
      vp8a::set_error("reference planes do not match the frame's MB grid");
      return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
    }
    if (ref_ids[k] < VP8A_REF_LAST || ref_ids[k] > VP8A_REF_ALTREF || !refs[k].y ||
        refs[k].y_stride < (uint64_t)mb_cols * 16) {
      vp8a::set_error("bad reference id, plane or stride");
      return VP8A_E_INVALID_ARGUMENT;
    }
  }
  if (!frame->y || frame->y_stride < frame->width) {
    vp8a::set_error("bad source plane");
    return VP8A_E_INVALID_ARGUMENT;
  }
  AnArgs a{};
  const void* d;
  if ((s = st.in(frame->y, frame->y_stride * (size_t)(frame->height - 1) + frame->width, &d)) != VP8A_OK) return s;
  a.fy = (const uint8_t*)d;
  a.fys = frame->y_stride;
  a.fw = (int)frame->width;
  a.fh = (int)frame->height;
  for (uint32_t k = 0; k < n_refs; k++) {
    const size_t bytes = refs[k].y_stride * (size_t)(mb_rows * 16 - 1) + (size_t)mb_cols * 16;
    if ((s = st.in(refs[k].y, bytes, &d)) != VP8A_OK) return s;
    a.refs[k].plane = (const uint8_t*)d;
    a.refs[k].stride = refs[k].y_stride;
    a.refs[k].width = mb_cols * 16;
    a.refs[k].height = mb_rows * 16;
    a.ref_ids[k] = ref_ids[k];
  }
  a.n_refs = (int)n_refs;
  a.mb_cols = mb_cols;
  a.mb_rows = mb_rows;
  if (mv_contexts) {
    a.ctx = *mv_contexts;
  } else {
    static const uint8_t dflt[2][19] = {
        {162, 128, 225, 146, 172, 147, 214, 39, 156, 128, 129, 132, 75, 145, 178, 206, 239, 254, 254},
        {164, 128, 204, 170, 119, 235, 140, 230, 228, 128, 130, 130, 74, 148, 180, 203, 236, 254, 254}};
    memcpy(a.ctx.p, dflt, sizeof dflt);
  }
  a.lambda = lambda;
  a.bit_cost = ctx->d_bit_cost;
  const size_t nmb = (size_t)mb_cols * mb_rows;
  void *dinfo, *dprog, *ddec, *dtr = nullptr, *dmvb;
  if ((s = st.scratch(sizeof(double) * 2 * MV_BITS_SPAN, &dmvb)) != VP8A_OK) return s;
  mv_bits_table_kernel<<<(2 * MV_BITS_SPAN + 255) / 256, 256, 0, ctx->stream>>>(ctx->d_bit_cost, a.ctx,
                                                                               (double*)dmvb);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  a.mvbits = (const double*)dmvb;
  if ((s = st.scratch(sizeof(MbInfoDev) * nmb, &dinfo)) != VP8A_OK) return s;
  if ((s = st.scratch(sizeof(unsigned) * mb_rows, &dprog)) != VP8A_OK) return s;
  VP8A_CUDA(cudaMemsetAsync(dprog, 0, sizeof(unsigned) * mb_rows, ctx->stream));
  if ((s = st.out(decisions, sizeof(vp8a_mb_decision) * nmb, &ddec)) != VP8A_OK) return s;
  if (trace && (s = st.out(trace, sizeof(vp8a_ref_search) * nmb * n_refs, &dtr)) != VP8A_OK) return s;
  a.infos = (MbInfoDev*)dinfo;
  a.progress = (unsigned*)dprog;
  a.status = ctx->d_status;
  a.dec = (vp8a_mb_decision*)ddec;
  a.trace = (vp8a_ref_search*)dtr;
  a.spin_limit = 1ull << 24;
  const int threads = MAX_REFS * WARPS_PER_REF * 32;
  int per_sm = 0;
  VP8A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, analysis_kernel, threads, 0));
  if (per_sm < 1) {
    vp8a::set_error("analysis kernel cannot be resident");
    return VP8A_E_CUDA;
  }
  const int grid = std::min(mb_rows, per_sm * ctx->sm_count);
  analysis_kernel<<<grid, threads, 0, ctx->stream>>>(a);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  if ((s = vp8a::check_device_status(ctx)) != VP8A_OK) return s;
  return st.finish();
}
