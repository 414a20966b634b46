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
#include <cooperative_groups.h>
#include <algorithm>
#include <cstddef>
#include <cstring>
#include <utility>
#include <vector>

#include "census.cuh"

namespace {
using namespace vp8a_dev;


constexpr int MAX_REFS = 3;

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
  int words;  // reference planes allow 32-bit loads (4-byte aligned base and stride)
  // The 16 sub-pel planes of each reference (subpel_planes_kernel), or
  // null: plane (fx, fy) of reference k starts at spl[k] + (fy / 2 * 4 +
  // fx / 2) * sp_plane, pixel (x, y) at ((y + SPB) * sp_pitch + x + SPB).
  const uint8_t* spl[MAX_REFS];
  uint64_t sp_pitch, sp_plane;
  // One proposed vector per (MB, reference), n_refs per MB in raster
  // order, or null: a second NEWMV candidate (the learned proposal's).
  const vp8a_mv* props;
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
static_assert(sizeof(WarpScratch) - offsetof(WarpScratch, temp) >= 3 * 22 * 16,
              "the quarter-pel planes fit in the window's six-tap scratch");

struct MainOut {
  uint32_t sad_zero, sad_nearest, sad_near;
  vp8a_search_result whole, half, quarter;
};

// One reference's mode decision (pick_mb_for_ref's result), with the
// chosen partition's sub-MVs; each CTA writes its own into rank 0.
struct __align__(16) RefDec {
  double j, total;
  vp8a_mv mv;
  int mode, pid;
  vp8a_mv split_mvs[16];
  uint8_t submv_modes[16];
};
static_assert(sizeof(RefDec) == 112 && offsetof(RefDec, mv) == 16 && offsetof(RefDec, split_mvs) == 28 &&
                  offsetof(RefDec, submv_modes) == 92,
              "RefDec is copied as words");
static_assert(offsetof(vp8a_mb_decision, mv) == 4 && offsetof(vp8a_mb_decision, j) == 8 &&
                  offsetof(vp8a_mb_decision, split_mvs) == 24 && offsetof(vp8a_mb_decision, submv_modes) == 88 &&
                  sizeof(vp8a_mb_decision) == 104,
              "vp8a_mb_decision is written as words");

struct SplitOut {
  double j;
  vp8a_mv split_mvs[16];
  uint8_t modes[16];
  int valid;
};

// SPLITMV scratch of one warp. Candidate column layout (fixed, no
// de-duplication): 0 = ZERO, 1..4 = LEFT vectors of the MB's left column
// anchors 0/4/8/12, 5..8 = ABOVE vectors of the top-row anchors 0..3,
// 9..24 = the NEW4X4 result of group 0..15. Aligned to 16 bytes with a
// size that is a multiple of 16: every warp's copy moves table columns as
// 16-byte vectors.
struct __align__(16) SplitScratch {
  uint32_t table[CMAX * 16];  // group g's SAD at column m: table[m * 16 + g], needed columns only
  double new_cost[16 * 5];    // lambda * (NEW4X4 mode bits of context x + group g's vector bits)
  double terms[32];           // group g's reference bits [g] and NEW vector bits [16 + g], for the total
  vp8a_mv cmv[CMAX];
};
static_assert(sizeof(SplitScratch) % 16 == 0, "SplitScratch copies stay 16-byte aligned");
struct Plan {
  int wx0, wy0;        // window origin (plane pixels)
  int hn_x, hn_y;      // NEAREST halo origin
  int hr_x, hr_y;      // NEAR halo origin
  int nblocks;
  int box[MAX_BLOCKS], boy[MAX_BLOCKS];  // block integer offsets
  int colblk[9];       // staged block of SPLITMV column m < 9 (ZERO, LEFT x4, ABOVE x4)
};

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

// Stage this CTA's reference: every region row is copied as 32-bit words
// (two aligned loads and a funnel shift per word); a word whose plane bytes
// are not all inside the row — at the frame edges — is fetched byte by byte
// with edge clamping. Each thread keeps up to 8 words in flight.
__device__ void stage_ref(const MePlane& P, RefSmem& R, const Plan& pl, int mbx, int mby, bool words, int tid,
                          int nthreads) {
  constexpr int N_WIN = 40 * 10, N_HALO = 21 * 6;
  const int total = N_WIN + 2 * N_HALO + pl.nblocks * 64;
  for (int base = tid; base < total; base += nthreads * 8) {
    uint32_t v[8];
    uint32_t* d[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int e = base + j * nthreads;
      d[j] = nullptr;
      v[j] = 0;
      if (e < total) {
        int row, word, x0, y0;
        uint8_t* dst;
        if (e < N_WIN) {
          row = e / 10;
          word = e - row * 10;
          x0 = pl.wx0;
          y0 = pl.wy0;
          dst = R.ws.win + row * WS;
        } else if (e < N_WIN + 2 * N_HALO) {
          const int q = e - N_WIN, h = q >= N_HALO, qq = q - h * N_HALO;
          row = qq / 6;
          word = qq - row * 6;
          x0 = h ? pl.hr_x : pl.hn_x;
          y0 = h ? pl.hr_y : pl.hn_y;
          dst = (h ? R.halo_near : R.halo_nearest) + row * HS;
        } else {
          const int q = e - N_WIN - 2 * N_HALO, b = q >> 6;
          row = (q >> 2) & 15;
          word = q & 3;
          x0 = mbx + pl.box[b];
          y0 = mby + pl.boy[b];
          dst = R.blocks[b] + row * 16;
        }
        const uint8_t* rp = P.plane + (size_t)clampi(y0 + row, 0, P.height - 1) * P.stride;
        const int x = x0 + 4 * word, sh = x & 3, xa = x - sh;
        if (words && x >= 0 && xa + (sh ? 8 : 4) <= P.width) {
          const uint32_t lo = *(const uint32_t*)(rp + xa);
          const uint32_t hi = sh ? *(const uint32_t*)(rp + xa + 4) : 0u;
          v[j] = __funnelshift_r(lo, hi, 8u * (unsigned)sh);
        } else {
#pragma unroll
          for (int k = 0; k < 4; k++) v[j] |= (uint32_t)rp[clampi(x + k, 0, P.width - 1)] << (8 * k);
        }
        d[j] = (uint32_t*)(dst + 4 * word);
      }
    }
#pragma unroll
    for (int j = 0; j < 8; j++)
      if (d[j]) *d[j] = v[j];
  }
}

// ------------------------------------------------------ whole-pel field

// Whole-pel SADs of every position within +-FR pixels of the search start
// (the snapped, clamped best predictor), per 4x4 block: a group SAD of any
// SPLITMV partition at such a position is the sum of its blocks, and the
// 16x16 SAD the sum of all 16. Both diamonds (the MB's, at most 8 steps of
// one pixel, and every SPLITMV group's, at most 4) stay inside the field,
// so they become table walks; vectors outside it (ZERO, the neighbours'
// vectors) are served by the staged blocks.
constexpr int FR = 8, FN = 2 * FR + 1, FP = FN * FN;
static_assert(WIN_LEAD - FR >= 0 && WIN_LEAD + FR + 16 <= WS, "the window covers the field");

struct __align__(16) FieldSmem {
  uint16_t blk[FP][16];  // 4x4 block SADs at each position (raster block order)
  uint32_t full[FP];     // 16x16 SADs
  uint16_t grp[FP][8];   // TopBottom 0,1 | LeftRight 0,1 | Quarters 0..3
};

__device__ __forceinline__ int fpos(int dx, int dy) {
  return (dx >= -FR && dx <= FR && dy >= -FR && dy <= FR) ? (dy + FR) * FN + dx + FR : -1;
}

// Block SADs: one thread per (block, row of positions); the 17 positions
// of a row share each window row's six words.
__device__ __forceinline__ void field_blocks(const uint8_t* win, const uint8_t* src, FieldSmem& F, int tid) {
  if (tid >= 16 * FN) return;
  const int b = tid & 15, dyi = tid >> 4;
  const int bx4 = (b & 3) * 4, by4 = (b >> 2) * 4;
  uint32_t acc[FN];
#pragma unroll
  for (int i = 0; i < FN; i++) acc[i] = 0;
#pragma unroll
  for (int row = 0; row < 4; row++) {
    const uint32_t sw = *(const uint32_t*)(src + (by4 + row) * 16 + bx4);
    const uint32_t* w = (const uint32_t*)(win + (WIN_LEAD - FR + dyi + by4 + row) * WS + bx4);
    uint32_t wd[6];
#pragma unroll
    for (int k = 0; k < 6; k++) wd[k] = w[k];
#pragma unroll
    for (int dxi = 0; dxi < FN; dxi++) {
      constexpr int base = WIN_LEAD - FR;
      const int o = base + dxi;
      acc[dxi] += __vsadu4(__funnelshift_r(wd[o >> 2], wd[(o >> 2) + 1], (unsigned)(o & 3) * 8u), sw);
    }
  }
#pragma unroll
  for (int dxi = 0; dxi < FN; dxi++) F.blk[dyi * FN + dxi][b] = (uint16_t)acc[dxi];
}

// 16x16 and partition-group sums per position.
__device__ __forceinline__ void field_sums(FieldSmem& F, int tid, int nthreads) {
  for (int pos = tid; pos < FP; pos += nthreads) {
    const uint32_t* v = (const uint32_t*)F.blk[pos];
    uint32_t b[16];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const uint32_t w = v[k];
      b[2 * k] = w & 0xffffu;
      b[2 * k + 1] = w >> 16;
    }
    const uint32_t q0 = b[0] + b[1] + b[4] + b[5], q1 = b[2] + b[3] + b[6] + b[7];
    const uint32_t q2 = b[8] + b[9] + b[12] + b[13], q3 = b[10] + b[11] + b[14] + b[15];
    F.full[pos] = q0 + q1 + q2 + q3;
    uint32_t* g = (uint32_t*)F.grp[pos];
    g[0] = (q0 + q1) | ((q2 + q3) << 16);
    g[1] = (q0 + q2) | ((q1 + q3) << 16);
    g[2] = q0 | (q1 << 16);
    g[3] = q2 | (q3 << 16);
  }
}

// 4x4 block SADs of the staged 16x16 blocks (ZERO and neighbour vectors).
__device__ __forceinline__ void staged_block_sads(const RefSmem& R, const uint8_t* src, int nblocks,
                                                  uint16_t (*xs)[16], int tid, int nthreads) {
  for (int t = tid; t < nblocks * 16; t += nthreads) {
    const int j = t >> 4, b = t & 15, bx4 = (b & 3) * 4, by4 = (b >> 2) * 4;
    uint32_t acc = 0;
#pragma unroll
    for (int row = 0; row < 4; row++)
      acc += __vsadu4(*(const uint32_t*)(R.blocks[j] + (by4 + row) * 16 + bx4),
                      *(const uint32_t*)(src + (by4 + row) * 16 + bx4));
    xs[j][b] = (uint16_t)acc;
  }
}

// One round of the N, S, W, E walk away from the +-1023 clamp, where every
// candidate is the running best moved by one pixel and none collapses: with
// the 3x3 neighbourhood of the round's start (r[4] = its SAD), N moves if it
// beats the start, else S; then W from the row reached, else E (a candidate
// that steps back onto an earlier position cannot beat it). Returns the
// move (dx, dy) and the new best SAD; (0, 0) ends the walk.
__device__ __forceinline__ void walk_round(const uint32_t (&r)[9], int& dx, int& dy, uint32_t& b) {
  b = r[4];
  dy = 0;
  if (r[1] < b) {
    dy = -1;
    b = r[1];
  } else if (r[7] < b) {
    dy = 1;
    b = r[7];
  }
  const uint32_t wv = dy < 0 ? r[0] : (dy == 0 ? r[3] : r[6]);
  const uint32_t ev = dy < 0 ? r[2] : (dy == 0 ? r[5] : r[8]);
  dx = 0;
  if (wv < b) {
    dx = -1;
    b = wv;
  } else if (ev < b) {
    dx = 1;
    b = ev;
  }
}

// small_diamond_search_luma (src/motion_search.rs:381-442) walked over the
// field: N, S, W, E from the running best, strict '<', collapse skips, at
// most max_iters rounds. Warp-uniform; a position outside the field (not
// reachable from an in-range start) is computed from the plane.
__device__ vp8a_search_result diamond_field(const FieldSmem& F, const MePlane& P, const uint8_t* win, int wx0,
                                            int wy0, int mbx, int mby, int cxp, int cyp, vp8a_mv center,
                                            int max_iters, const uint8_t* src, int lane) {
  auto sad = [&](vp8a_mv m) -> uint32_t {
    const int x = mbx + m.col / 4, y = mby + m.row / 4;
    const int p = fpos(x - cxp, y - cyp);
    return p >= 0 ? F.full[p] : sad_whole_at(P, win, wx0, wy0, x, y, src, lane);
  };
  vp8a_mv best;
  best.row = snap_whole(clamp_component(center.row));
  best.col = snap_whole(clamp_component(center.col));
  const int x0 = mbx + best.col / 4 - cxp, y0 = mby + best.row / 4 - cyp;
  const int lim = 1020 - 4 * max_iters;
  if (best.row >= -lim && best.row <= lim && best.col >= -lim && best.col <= lim && max_iters <= FR &&
      x0 == 0 && y0 == 0) {
    // No candidate of the walk is clamped and every round's neighbourhood
    // lies in the field: read it whole, decide the round with selects.
    int x = 0, y = 0;
    uint32_t bs = F.full[fpos(0, 0)];
    for (int it = 0; it < max_iters; it++) {
      const uint32_t* c0 = F.full + fpos(x, y);
      const uint32_t r[9] = {c0[-FN - 1], c0[-FN], c0[-FN + 1], c0[-1], bs, c0[1], c0[FN - 1], c0[FN], c0[FN + 1]};
      int dx, dy;
      uint32_t b;
      walk_round(r, dx, dy, b);
      if (dx == 0 && dy == 0) break;
      x += dx;
      y += dy;
      bs = b;
    }
    vp8a_search_result res;
    res.mv.row = (int16_t)(best.row + 4 * y);
    res.mv.col = (int16_t)(best.col + 4 * x);
    res.sad = bs;
    return res;
  }
  uint32_t best_sad = sad(best);
  for (int it = 0; it < max_iters; it++) {
    bool improved = false;
    const int dr[4] = {-4, 4, 0, 0}, dc[4] = {0, 0, -4, 4};
#pragma unroll
    for (int d = 0; d < 4; d++) {
      vp8a_mv cand;
      cand.row = snap_whole(clamp_component(best.row + dr[d]));
      cand.col = snap_whole(clamp_component(best.col + dc[d]));
      if (cand.row == best.row && cand.col == best.col) continue;
      const uint32_t s = sad(cand);
      if (s < best_sad) {
        best_sad = s;
        best = cand;
        improved = true;
      }
    }
    if (!improved) break;
  }
  vp8a_search_result res;
  res.mv = best;
  res.sad = best_sad;
  return res;
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

// 4x4 blocks of group g of partition p, as a bit mask over raster blocks
// (PartitionGroups::build, src/encoder.rs:7912-7980). Groups are numbered
// in raster order over the partition's gh x gw group grid: TopBottom 2x1,
// LeftRight 1x2, Quarters 2x2, Mv16 4x4.
__constant__ uint16_t c_group_blocks[4][16] = {
    {0x00ff, 0xff00},
    {0x3333, 0xcccc},
    {0x0033, 0x00cc, 0x3300, 0xcc00},
    {0x0001, 0x0002, 0x0004, 0x0008, 0x0010, 0x0020, 0x0040, 0x0080, 0x0100, 0x0200, 0x0400, 0x0800, 0x1000,
     0x2000, 0x4000, 0x8000}};

__device__ __forceinline__ uint32_t group_sum(const uint16_t* v16, int pid, int g) {
  const uint32_t m = c_group_blocks[pid][g];
  uint32_t s = 0;
#pragma unroll
  for (int b = 0; b < 16; b++)
    if ((m >> b) & 1u) s += v16[b];
  return s;
}

// A group's whole-pel SAD at pixel (x, y) computed from the plane with
// edge clamping, by one lane (only for positions neither the field nor a
// staged block covers).
__device__ uint32_t direct_group_sad(const MePlane& P, const uint8_t* src, int x, int y, int pid, int g) {
  const uint32_t m = c_group_blocks[pid][g];
  uint32_t s = 0;
  for (int b = 0; b < 16; b++) {
    if (!((m >> b) & 1u)) continue;
    const int bx4 = (b & 3) * 4, by4 = (b >> 2) * 4;
    for (int r = 0; r < 4; r++) {
      const uint8_t* row = P.plane + (size_t)clampi(y + by4 + r, 0, P.height - 1) * P.stride;
      for (int c = 0; c < 4; c++) {
        const int d = (int)row[clampi(x + bx4 + c, 0, P.width - 1)] - (int)src[(by4 + r) * 16 + bx4 + c];
        s += (uint32_t)(d < 0 ? -d : d);
      }
    }
  }
  return s;
}

struct FieldView {
  const FieldSmem* F;
  const uint16_t (*xs)[16];
  const Plan* pl;
  int mbx, mby, cxp, cyp;
};

// Group g's SAD at integer offset of `m`: field, staged block, or plane.
__device__ __forceinline__ uint32_t group_sad(const FieldView& v, const MePlane& P, const uint8_t* src, int pid,
                                              int g, vp8a_mv m) {
  const int x = v.mbx + int_off(m.col), y = v.mby + int_off(m.row);
  const int p = fpos(x - v.cxp, y - v.cyp);
  if (p >= 0) {
    if (pid == 3) return v.F->blk[p][g];
    return v.F->grp[p][(pid == 0 ? 0 : (pid == 1 ? 2 : 4)) + g];
  }
  for (int j = 0; j < v.pl->nblocks; j++)
    if (v.mbx + v.pl->box[j] == x && v.mby + v.pl->boy[j] == y) return group_sum(v.xs[j], pid, g);
  return direct_group_sad(P, src, x, y, pid, g);
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

// score_split_partition (src/encoder.rs:8080-8246) on one warp: lane g
// walks group g's NEW4X4 diamond over the field, the lanes then fill a
// table of group SADs at every vector the sub-MV choice can consider (ZERO,
// the external neighbours' vectors, every group's NEW result), and the
// sequential LEFT/ABOVE/ZERO/NEW choice over groups reads that table.
//
// The per-group costs that do not depend on the chain are computed before
// it: sbits[ctx * 4 + mode] = submv_ref_bits of each context and mode, and
// each group's NEW vector bits. Every value is the same expression the
// reference evaluates, so the chain's sums are unchanged.
__device__ void split_partition(const AnArgs& a, const double* pbits, const double* sbits, const double* lterm,
                                const double* mvb, const FieldView& fv, const MePlane& P, const uint8_t* src, vp8a_mv bp,
                                const MbInfoDev& above, const MbInfoDev& left, int pid, SplitScratch& W,
                                SplitOut* out, int lane) {
  const int G = pid == 3 ? 16 : (pid == 2 ? 4 : 2);
  const int goff = pid == 0 ? 0 : (pid == 1 ? 2 : 4);
  // Group `lane`'s NEW4X4 result (lanes < G).
  bool my_new_ok = false;
  uint32_t my_new_sad = 0;
  double my_new_bits = 0.0;
  if (lane < G) {
    // group_small_diamond_search (src/encoder.rs:7812-7879): snap then
    // clamp the centre; N, S, W, E clamped, not snapped; four rounds. Every
    // candidate of a round lies within one pixel of the round's start, so
    // the round reads that 3x3 neighbourhood first and replays the walk.
    const int g = lane;
    vp8a_mv best;
    best.row = (int16_t)clampi((bp.row / 4) * 4, -1023, 1023);
    best.col = (int16_t)clampi((bp.col / 4) * 4, -1023, 1023);
    uint32_t bs = group_sad(fv, P, src, pid, g, best);
    const uint16_t* fbase = pid == 3 ? &fv.F->blk[0][g] : &fv.F->grp[0][goff + g];
    const int fstride = pid == 3 ? 16 : 8;  // u16 entries per field position
    const int sx = fv.mbx + int_off(best.col) - fv.cxp, sy = fv.mby + int_off(best.row) - fv.cyp;
    if (!(best.row & 3) && !(best.col & 3) && best.row >= -1007 && best.row <= 1007 && best.col >= -1007 &&
        best.col <= 1007 && sx >= -(FR - 4) && sx <= FR - 4 && sy >= -(FR - 4) && sy <= FR - 4) {
      // Four rounds away from the clamp, inside the field (walk_round).
      int x = sx, y = sy;
      for (int it = 0; it < 4; it++) {
        const uint16_t* c0 = fbase + fpos(x, y) * fstride;
        const uint32_t r[9] = {c0[(-FN - 1) * fstride], c0[-FN * fstride], c0[(-FN + 1) * fstride],
                               c0[-fstride],            bs,                c0[fstride],
                               c0[(FN - 1) * fstride],  c0[FN * fstride],  c0[(FN + 1) * fstride]};
        int dx, dy;
        uint32_t b;
        walk_round(r, dx, dy, b);
        if (dx == 0 && dy == 0) break;
        x += dx;
        y += dy;
        bs = b;
      }
      best.row = (int16_t)(best.row + 4 * (y - sy));
      best.col = (int16_t)(best.col + 4 * (x - sx));
    } else
    for (int it = 0; it < 4; it++) {
      const int dx0 = fv.mbx + int_off(best.col) - fv.cxp, dy0 = fv.mby + int_off(best.row) - fv.cyp;
      const vp8a_mv b0 = best;
      const uint32_t r11 = bs;  // the SAD at the round's start
      bool improved = false;
      const int dr[4] = {-4, 4, 0, 0}, dc[4] = {0, 0, -4, 4};
      if (dx0 > -FR && dx0 < FR && dy0 > -FR && dy0 < FR) {
        // The round's 3x3 neighbourhood, read together.
        const uint16_t* c0 = fbase + fpos(dx0, dy0) * fstride;
        const uint32_t r00 = c0[(-FN - 1) * fstride], r01 = c0[-FN * fstride], r02 = c0[(-FN + 1) * fstride];
        const uint32_t r10 = c0[-fstride], r12 = c0[fstride];
        const uint32_t r20 = c0[(FN - 1) * fstride], r21 = c0[FN * fstride], r22 = c0[(FN + 1) * fstride];
#pragma unroll
        for (int d = 0; d < 4; d++) {
          vp8a_mv c;
          c.row = (int16_t)clampi(best.row + dr[d], -1023, 1023);
          c.col = (int16_t)clampi(best.col + dc[d], -1023, 1023);
          if (mv_eq(c, best)) continue;
          const int ox = int_off(c.col) - int_off(b0.col), oy = int_off(c.row) - int_off(b0.row);
          const uint32_t top = ox < 0 ? r00 : (ox == 0 ? r01 : r02);
          const uint32_t mid = ox < 0 ? r10 : (ox == 0 ? r11 : r12);
          const uint32_t bot = ox < 0 ? r20 : (ox == 0 ? r21 : r22);
          const uint32_t sv = oy < 0 ? top : (oy == 0 ? mid : bot);
          if (sv < bs) {
            bs = sv;
            best = c;
            improved = true;
          }
        }
      } else {
#pragma unroll 1
        for (int d = 0; d < 4; d++) {
          vp8a_mv c;
          c.row = (int16_t)clampi(best.row + dr[d], -1023, 1023);
          c.col = (int16_t)clampi(best.col + dc[d], -1023, 1023);
          if (mv_eq(c, best)) continue;
          const uint32_t sv = group_sad(fv, P, src, pid, g, c);
          if (sv < bs) {
            bs = sv;
            best = c;
            improved = true;
          }
        }
      }
      if (!improved) break;
    }
    W.cmv[9 + g] = best;
    const int dr = (int)best.row - bp.row, dc = (int)best.col - bp.col;
    const bool ok = dr >= -1023 && dr <= 1023 && dc >= -1023 && dc <= 1023;
    const double nb = ok ? mvb[dr + 1023] + mvb[MV_BITS_SPAN + dc + 1023] : 0.0;
    my_new_ok = ok;
    my_new_sad = bs;
    my_new_bits = nb;
#pragma unroll
    for (int x = 0; x < 5; x++) W.new_cost[g * 5 + x] = a.lambda * (sbits[x * 4 + VP8A_SUBMV_NEW] + nb);
  }
  // Columns 0-8: ZERO, the left neighbour's vectors at anchors 0/4/8/12,
  // the above neighbour's at anchors 0-3 (one lane each).
  if (lane < 9)
    W.cmv[lane] = lane == 0 ? vp8a_mv{0, 0} : (lane < 5 ? ext_left(left, 4 * (lane - 1)) : ext_above(above, lane - 5));
  __syncwarp();
  // Lane m < 9 + G holds column m's vector, packed (equal vectors, equal
  // words; the zero vector is 0).
  const int ncol = 9 + G;
  const vp8a_mv mvm = lane < ncol ? W.cmv[lane] : vp8a_mv{0, 0};
  const uint32_t cvec = (uint32_t)(uint16_t)mvm.row | ((uint32_t)(uint16_t)mvm.col << 16);
  // The candidate table: lane m fills column m for every group. Columns
  // 0-8 (ZERO and the neighbours' vectors) are staged blocks; columns 9+
  // (the groups' NEW results) lie in the field, or, beyond it, are summed
  // from the plane. Only the columns the partition's choice can reach.
  const uint32_t need = c_need_cols[pid];
  if (lane < ncol && ((need >> lane) & 1u)) {
    const int x = fv.mbx + int_off(mvm.col), y = fv.mby + int_off(mvm.row);
    const int cp = lane < 9 ? fv.pl->colblk[lane] : fpos(x - fv.cxp, y - fv.cyp);
    uint32_t* col = W.table + lane * 16;
    if (pid == 3 && (lane < 9 || cp >= 0)) {
      // The 16 block SADs of a staged block or a field position are one
      // 32-byte row.
      const uint4* row = lane < 9 ? (const uint4*)fv.xs[cp] : (const uint4*)fv.F->blk[cp];
      const uint4 lo = row[0], hi = row[1];
      const uint32_t w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
#pragma unroll
      for (int q = 0; q < 4; q++)
        ((uint4*)col)[q] = make_uint4(w[2 * q] & 0xffffu, w[2 * q] >> 16, w[2 * q + 1] & 0xffffu, w[2 * q + 1] >> 16);
    } else {
      for (int g = 0; g < G; g++) {
        uint32_t v;
        if (lane < 9) v = pid == 3 ? fv.xs[cp][g] : group_sum(fv.xs[cp], pid, g);
        else if (cp >= 0) v = pid == 3 ? fv.F->blk[cp][g] : fv.F->grp[cp][goff + g];
        else v = direct_group_sad(P, src, x, y, pid, g);
        col[g] = v;
      }
    }
  }
  __syncwarp();
  // The sub-MV choice. Lane g decides group g. A group's LEFT/ABOVE come
  // from the group to its left and above, so the groups of one
  // anti-diagonal of the partition's group grid are independent: step s
  // decides them in parallel. The columns the neighbouring groups chose
  // and the vectors they stand for travel by shuffles.
  // The group grid is gh x gw = 2^lgh x 2^lgw groups of (4 >> lgh) x
  // (4 >> lgw) blocks.
  const int lgh = pid == 1 ? 0 : (pid == 3 ? 2 : 1), lgw = pid == 0 ? 0 : (pid == 3 ? 2 : 1);
  const int gh = 1 << lgh, gw = 1 << lgw;
  const int gr = lane >> lgw, gc = lane & (gw - 1);
  // The group's top-left block; the blocks left of and above it belong to
  // the groups (gr, gc - 1) and (gr - 1, gc), or lie outside the MB.
  const int anchor = ((gr << (2 - lgh)) << 2) + (gc << (2 - lgw));
  // A group on the MB's left or top edge takes its LEFT or ABOVE vector
  // from the neighbour MB's column; lane g's NEW result is column 9 + g.
  const int ext_l = 1 + (anchor >> 2), ext_a = 5 + anchor;
  const uint32_t ext_lv = __shfl_sync(FULL, cvec, ext_l & 31), ext_av = __shfl_sync(FULL, cvec, ext_a & 31);
  const uint32_t new_vec = __shfl_sync(FULL, cvec, (9 + lane) & 31);
  // The group's choice: its column and that column's vector.
  int chosen = 0, mode = VP8A_SUBMV_ZERO, my_ctx = 0;
  uint32_t chosen_vec = 0, my_sad = 0;
  bool my_bad = false;
  for (int st = 0; st < gh + gw - 1; st++) {
    const int lsrc = gc == 0 ? lane : lane - 1, asrc = gr == 0 ? lane : lane - gw;
    const int lch = __shfl_sync(FULL, chosen, lsrc), ach = __shfl_sync(FULL, chosen, asrc);
    const uint32_t lchv = __shfl_sync(FULL, chosen_vec, lsrc), achv = __shfl_sync(FULL, chosen_vec, asrc);
    if (lane < G && gr + gc == st) {
      const int lidx = gc == 0 ? ext_l : lch, aidx = gr == 0 ? ext_a : ach;
      const uint32_t lv = gc == 0 ? ext_lv : lchv, av = gr == 0 ? ext_av : achv;
      const bool lez = lv == 0u, aez = av == 0u, lea = lv == av;
      const int ctxi = (lea && lez) ? 4 : (lea ? 3 : (aez ? 2 : (lez ? 1 : 0)));
      const double* lt = lterm + ctxi * 4;
      const uint32_t tl = W.table[lidx * 16 + lane], ta = W.table[aidx * 16 + lane], tz = W.table[lane];
      // LEFT, ABOVE, ZERO, then NEW (sad + lambda * (mode bits + vector
      // bits), the vector bits 0 for the first three); the reference keeps
      // the first strict minimum in that order. Every J here is a finite sum
      // of non-negative terms, so J order is the order of the doubles' bit
      // patterns as unsigned integers, and the first minimum of the four is
      // the first minimum of the first minima of (LEFT, ABOVE) and (ZERO,
      // NEW).
      const uint64_t j0 = (uint64_t)__double_as_longlong((double)tl + lt[0]);
      const uint64_t j1 = (uint64_t)__double_as_longlong((double)ta + lt[1]);
      const uint64_t j2 = (uint64_t)__double_as_longlong((double)tz + lt[2]);
      const uint64_t jn = my_new_ok ? (uint64_t)__double_as_longlong((double)my_new_sad + W.new_cost[lane * 5 + ctxi])
                                    : 0xffffffffffffffffull;
      const bool above_first = j1 < j0, new_second = jn < j2;
      const uint64_t v01 = above_first ? j1 : j0, v2n = new_second ? jn : j2;
      const bool second = v2n < v01;
      const uint64_t best_j = second ? v2n : v01;
      mode = second ? (new_second ? VP8A_SUBMV_NEW : VP8A_SUBMV_ZERO)
                    : (above_first ? VP8A_SUBMV_ABOVE : VP8A_SUBMV_LEFT);
      chosen = second ? (new_second ? 9 + lane : 0) : (above_first ? aidx : lidx);
      chosen_vec = second ? (new_second ? new_vec : 0u) : (above_first ? av : lv);
      my_sad = second ? (new_second ? my_new_sad : tz) : (above_first ? ta : tl);
      my_ctx = ctxi;
      my_bad = best_j >= 0x7ff0000000000000ull;
    }
  }
  if (lane < G) out->modes[lane] = (uint8_t)mode;
  // Totals in the reference's group order (the f64 sum is order-sensitive):
  // the groups' terms go through shared memory and lane 0 sums them in
  // order.
  const bool mine = lane < G;
  const bool isn = mine && mode == VP8A_SUBMV_NEW;
  if (mine) {
    W.terms[lane] = sbits[my_ctx * 4 + mode];
    W.terms[16 + lane] = my_new_bits;
  }
  const uint32_t total_sad = __reduce_add_sync(FULL, mine ? my_sad : 0u);
  const unsigned any_bad = __ballot_sync(FULL, mine && my_bad), news = __ballot_sync(FULL, isn);
  __syncwarp();
  if (lane == 0) {
    // The reference stops at the first group without a finite choice.
    out->valid = any_bad == 0u;
    if (any_bad == 0u) {
      double total_bits = 0.0;
#pragma unroll
      for (int gg = 0; gg < 16; gg++) {
        if (gg < G) {
          total_bits += W.terms[gg];
          if ((news >> gg) & 1u) total_bits += W.terms[16 + gg];
        }
      }
      out->j = (double)total_sad + a.lambda * (pbits[pid] + total_bits);
      for (int i = G; i < 16; i++) out->modes[i] = VP8A_SUBMV_ZERO;
    }
  }
  // Block b's vector: the column its group chose.
  const int gb = lane < 16 ? (((lane >> 2) >> (2 - lgh)) << lgw) + ((lane & 3) >> (2 - lgw)) : 0;
  const uint32_t vb = __shfl_sync(FULL, chosen_vec, gb);
  if (lane < 16) out->split_mvs[lane] = vp8a_mv{(int16_t)(vb & 0xffffu), (int16_t)(vb >> 16)};
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ------------------------------------------------------ sub-pel planes
//
// The §18.3 sub-pel sample at integer position (x, y) with eighth-pel
// fraction (fx, fy) depends only on the edge-clamped reference around it:
// a horizontal six-tap pass over rows y - 2 .. y + 3 (skipped when fx is
// 0), the 8-bit intermediate, then a vertical pass (skipped when fy is 0)
// — the two-pass listing of sixtap_mb_luma (src/motion_comp.rs:1018-1057)
// with its identity elision, whatever block the sample belongs to. The
// luma vectors of the analysis have even eighth-pel fractions, so 16
// planes (fx, fy in {0, 2, 4, 6}) hold every sample its half- and
// quarter-pel refinements read. A parallel pre-pass builds them over the
// MB-padded plane plus a border of SPB pixels; the wavefront's refinement
// steps then read each candidate's 16 x 16 prediction as plain bytes
// instead of synthesising it in the per-MB critical path. Candidates whose
// block leaves the border keep the in-kernel synthesis.
constexpr int SPB = 32;                  // border around the MB-padded plane
constexpr int SP_TW = 64, SP_TH = 32;    // pre-pass output tile

struct SubpelArgs {
  const uint8_t* ref;
  uint64_t stride;
  int pw, ph;  // MB-padded plane (the clamp bounds)
  uint8_t* out;
  uint64_t pitch, plane;
};

// One CTA per 64 x 32 output tile of all 16 planes of one reference.
__global__ void __launch_bounds__(256) subpel_planes_kernel(SubpelArgs a) {
  __shared__ uint8_t E[SP_TH + 5][SP_TW + 8];
  __shared__ __align__(4) uint8_t Hs[SP_TH + 5][SP_TW];
  const int tid = threadIdx.x;
  const int tx0 = (int)blockIdx.x * SP_TW - SPB, ty0 = (int)blockIdx.y * SP_TH - SPB;
  // The edge-clamped reference under the tile and its six-tap reach.
  for (int i = tid; i < (SP_TH + 5) * (SP_TW + 5); i += 256) {
    const int r = i / (SP_TW + 5), c = i - r * (SP_TW + 5);
    const int y = clampi(ty0 - 2 + r, 0, a.ph - 1), x = clampi(tx0 - 2 + c, 0, a.pw - 1);
    E[r][c] = __ldg(a.ref + (size_t)y * a.stride + x);
  }
  __syncthreads();
  for (int fxi = 0; fxi < 4; fxi++) {
    const int* fh = c_sixtap[2 * fxi];
    for (int i = tid; i < (SP_TH + 5) * SP_TW; i += 256) {
      const int r = i / SP_TW, c = i - r * SP_TW;
      const uint8_t* p = &E[r][c];
      Hs[r][c] = fxi ? (uint8_t)interp6(fh, p[0], p[1], p[2], p[3], p[4], p[5]) : p[2];
    }
    __syncthreads();
    for (int fyi = 0; fyi < 4; fyi++) {
      const int* fv = c_sixtap[2 * fyi];
      uint8_t* op = a.out + (size_t)(fyi * 4 + fxi) * a.plane + (size_t)(ty0 + SPB) * a.pitch + (tx0 + SPB);
      for (int w = tid; w < SP_TH * SP_TW / 4; w += 256) {
        const int r = w / (SP_TW / 4), c = 4 * (w - r * (SP_TW / 4));
        uint32_t o = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int v = fyi ? interp6(fv, Hs[r][c + j], Hs[r + 1][c + j], Hs[r + 2][c + j], Hs[r + 3][c + j],
                                      Hs[r + 4][c + j], Hs[r + 5][c + j])
                            : Hs[r + 2][c + j];
          o |= (uint32_t)v << (8 * j);
        }
        *reinterpret_cast<uint32_t*>(op + (size_t)r * a.pitch + c) = o;
      }
    }
    __syncthreads();
  }
}

// Sub-pel plane geometry of a reference: row pitch and plane size in bytes
// (whole pre-pass tiles, so the kernel needs no bounds checks). The pitch
// keeps at least 16 bytes after the extent's last column, where the
// aligned word reads of a block at the right edge end.
__host__ __device__ inline uint64_t sp_pitch_of(int pw) {
  return (uint64_t)((pw + 2 * SPB + 16 + SP_TW - 1) / SP_TW * SP_TW);
}
__host__ __device__ inline int sp_rows_of(int ph) { return (ph + 2 * SPB + SP_TH - 1) / SP_TH * SP_TH; }

// Whether a 16 x 16 block at (ix, iy) lies inside the planes' extent.
__device__ __forceinline__ bool sp_inside(const MePlane& P, int ix, int iy) {
  return ix >= -SPB && iy >= -SPB && ix + 16 <= P.width + SPB && iy + 16 <= P.height + SPB;
}

// Row `row` of the 16 x 16 block at (ix, iy) of a sub-pel plane against the
// source row, summed over the half-warp (every lane of it gets the SAD).
// The five aligned words cover the sixteen bytes and end at most 19 bytes
// after the block's first column; the pitch's 16 spare bytes keep them
// inside the row.
__device__ __forceinline__ uint32_t sp_block_sad(const uint8_t* plane, uint64_t pitch, int ix, int iy,
                                                 const uint8_t* src, int row) {
  const uint8_t* p = plane + (size_t)(iy + SPB + row) * pitch + (ix + SPB);
  const uintptr_t ad = (uintptr_t)p;
  const uint32_t* w = reinterpret_cast<const uint32_t*>(ad & ~(uintptr_t)3);
  const unsigned sh = (unsigned)(ad & 3) * 8u;
  const uint32_t w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2), w3 = __ldg(w + 3), w4 = __ldg(w + 4);
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src + row * 16);
  uint32_t sad = __vsadu4(__funnelshift_r(w0, w1, sh), s[0]) + __vsadu4(__funnelshift_r(w1, w2, sh), s[1]) +
                 __vsadu4(__funnelshift_r(w2, w3, sh), s[2]) + __vsadu4(__funnelshift_r(w3, w4, sh), s[3]);
  const unsigned hm = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
#pragma unroll
  for (int o = 8; o >= 1; o >>= 1) sad += __shfl_xor_sync(hm, sad, o);
  return sad;
}

// ------------------------------------------------------ sub-pel stages

constexpr int NW = 9;                 // warps per CTA (one reference)
constexpr int AN_THREADS = NW * 32;
constexpr int MAIN_WARPS = 5;         // warps 0 and 5-8: the MB search chain
constexpr int MAIN_THREADS = MAIN_WARPS * 32;

// Offsets (row, col) of the eight refinement candidates in the reference's
// order: (-1,-1) (-1,0) (-1,1) (0,-1) (0,1) (1,-1) (1,0) (1,1).
__device__ __forceinline__ int cand_dr(int k) { return (k < 3) ? -1 : (k < 5 ? 0 : 1); }
__device__ __forceinline__ int cand_dc(int k) { return (k == 0 || k == 3 || k == 5) ? -1 : ((k == 1 || k == 6) ? 0 : 1); }

// The H, V and D half-pel planes around a whole-pel centre whose block
// origin in the window is (bx, by) (the planes of half_plane_sads, filled
// by the main group's MAIN_THREADS threads): H and V first, then D from H.
// Each thread's outputs are independent; the loops are unrolled so that
// all of a thread's window reads are in flight together.
__device__ __forceinline__ void half_planes_hv(WarpScratch& S, int bx, int by, int tid) {
  constexpr int NH = 22 * 17, NO = NH + 17 * 16;
#pragma unroll
  for (int it = 0; it < (NO + MAIN_THREADS - 1) / MAIN_THREADS; it++) {
    const int o = tid + it * MAIN_THREADS;
    if (o < NH) {
      const int r = o / 17, i = o - r * 17;
      const uint8_t* p = S.win + (by - 3 + r) * WS + bx + i - 3;
      S.hp[o] = (uint8_t)interp6_half(p[0], p[1], p[2], p[3], p[4], p[5]);
    } else if (o < NO) {
      const int q = o - NH, r = q >> 4, c = q & 15;
      const uint8_t* p = S.win + (by + r - 3) * WS + bx + c;
      S.vp[q] = (uint8_t)interp6_half(p[0], p[WS], p[2 * WS], p[3 * WS], p[4 * WS], p[5 * WS]);
    }
  }
}

// The D plane, from H (after H is complete).
__device__ __forceinline__ void half_planes_d(WarpScratch& S, int tid) {
#pragma unroll
  for (int it = 0; it < (17 * 17 + MAIN_THREADS - 1) / MAIN_THREADS; it++) {
    const int o = tid + it * MAIN_THREADS;
    if (o < 17 * 17) {
      const int r = o / 17, i = o - r * 17;
      const uint8_t* p = S.hp + r * 17 + i;
      S.dp[o] = (uint8_t)interp6_half(p[0], p[17], p[34], p[51], p[68], p[85]);
    }
  }
}

// SAD of half-pel candidate k against the planes (one warp).
__device__ __forceinline__ uint32_t half_cand_sad(const WarpScratch& S, int k, const uint8_t* src, int lane) {
  const int dy = cand_dr(k), dx = cand_dc(k);
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
  const int c = lane & 15, r0 = (lane >> 4) * 8;
  uint32_t s = 0;
#pragma unroll
  for (int r = r0; r < r0 + 8; r++) {
    const int d = (int)pl[r * st + c] - (int)src[r * 16 + c];
    s += (uint32_t)(d < 0 ? -d : d);
  }
  return __reduce_add_sync(FULL, s);
}

// quarter_pixel_refine_luma's eight candidates around `qc` share three
// horizontal six-tap planes, one per candidate column (the columns are
// qc.col - 1, qc.col, qc.col + 1 quarter-pels; a column whose eighth-pel
// fraction is 0 keeps the unfiltered pixels, the reference's identity
// elision). Each candidate's prediction is then its vertical pass over its
// column's plane: the same taps, the same 8-bit intermediate and the same
// edge-clamped source as its own two-pass synthesis.
struct QuarterGeom {
  int ix[3], fx[3], iy[3], fy[3], iy0;
};

// Fills the geometry; false when the window does not cover every
// candidate's halo.
__device__ __forceinline__ bool quarter_geom(vp8a_mv qc, int mbx, int mby, int wx0, int wy0, QuarterGeom& q) {
  int xmin = 1 << 30, xmax = -(1 << 30), ymin = 1 << 30, ymax = -(1 << 30);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int ec = eighth(clamp_component(qc.col + k - 1)), er = eighth(clamp_component(qc.row + k - 1));
    q.ix[k] = mbx + (ec >> 3) - wx0;
    q.fx[k] = ec & 7;
    q.iy[k] = mby + (er >> 3) - wy0;
    q.fy[k] = er & 7;
    xmin = min(xmin, q.ix[k]);
    xmax = max(xmax, q.ix[k]);
    ymin = min(ymin, q.iy[k]);
    ymax = max(ymax, q.iy[k]);
  }
  q.iy0 = ymin - 2;  // first plane row (window coordinates)
  // Planes span window rows iy0 .. iy0 + 21 and columns ix - 2 .. ix + 18.
  return xmin >= 2 && xmax + 19 <= WS && ymin >= 2 && ymin + 20 <= WS && ymax - ymin <= 1;
}

// Horizontal planes: qh[k * 352 + rr * 16 + c], rr = 0..21 from window row
// iy0 (filled by the main group; unrolled, as the half-pel planes).
__device__ __forceinline__ void quarter_planes_h(const uint8_t* win, uint8_t* qh, const QuarterGeom& q, int t) {
#pragma unroll
  for (int it = 0; it < (3 * 22 * 16 + MAIN_THREADS - 1) / MAIN_THREADS; it++) {
    const int o = t + it * MAIN_THREADS;
    if (o < 3 * 22 * 16) {
      const int k = o / 352, rem = o - k * 352, rr = rem >> 4, c = rem & 15;
      const uint8_t* p = win + (q.iy0 + rr) * WS + q.ix[k] + c;
      int v;
      if (q.fx[k]) {
        const int* f = c_sixtap[q.fx[k]];
        v = interp6(f, p[-2], p[-1], p[0], p[1], p[2], p[3]);
      } else {
        v = p[0];
      }
      qh[o] = (uint8_t)v;
    }
  }
}

// Vertical pass and SAD of candidate t >> 4 at column t & 15, reduced over
// the half-warp; the SAD is valid on lane (t & 15) == 0 of each half-warp.
__device__ __forceinline__ uint32_t quarter_vsad(const uint8_t* qh, const QuarterGeom& q, const uint8_t* src, int t) {
  const int k = t >> 4, c = t & 15;
  const int kc = cand_dc(k) + 1, kr = cand_dr(k) + 1;
  const uint8_t* pl = qh + kc * 352 + (q.iy[kr] - 2 - q.iy0) * 16 + c;  // plane row of prediction row -2
  const int fy = q.fy[kr];
  uint32_t s = 0;
  if (fy) {
    const int* fp = c_sixtap[fy];
    const int f0 = fp[0], f1 = fp[1], f2 = fp[2], f3 = fp[3], f4 = fp[4], f5 = fp[5];
    int w0 = pl[0], w1 = pl[16], w2 = pl[32], w3 = pl[48], w4 = pl[64];
#pragma unroll
    for (int r = 0; r < 16; r++) {
      const int w5 = pl[(r + 5) * 16];
      const int a = w0 * f0 + w1 * f1 + w2 * f2 + w3 * f3 + w4 * f4 + w5 * f5;
      const int v = clampi((a + 64) >> 7, 0, 255);
      const int d = v - (int)src[r * 16 + c];
      s += (uint32_t)(d < 0 ? -d : d);
      w0 = w1;
      w1 = w2;
      w2 = w3;
      w3 = w4;
      w4 = w5;
    }
  } else {
#pragma unroll
    for (int r = 0; r < 16; r++) {
      const int d = (int)pl[(r + 2) * 16] - (int)src[r * 16 + c];
      s += (uint32_t)(d < 0 ? -d : d);
    }
  }
  const unsigned hm = (t & 16) ? 0xffff0000u : 0x0000ffffu;
#pragma unroll
  for (int o = 8; o >= 1; o >>= 1) s += __shfl_xor_sync(hm, s, o);
  return s;
}

struct __align__(16) WarpTemp {
  uint8_t temp[21 * 16 + 16];  // six-tap first pass
  uint8_t halo[21 * 24 + 24];  // out-of-window halo
};

// -------------------------------------------------------------- kernel


// Barrier 1: the main group only.
__device__ __forceinline__ void main_sync() { asm volatile("bar.sync 1, %0;" ::"n"(MAIN_THREADS) : "memory"); }
static_assert(AN_THREADS >= 16 * FN, "one thread per field task");

// Work items: one MB row each. A single frame (BATCH false) takes rows
// 0..a0.mb_rows-1 of a0; a batch takes items[i] = job << 16 | row over the
// job table `jobs`, ordered so that every row comes after the row above it
// (a job's rows are consecutive). Clusters take items round-robin and all
// are resident, so the row a wait depends on is always held by a running
// cluster. Every job of one launch has cluster-size (n_refs) references.
// Two CTAs per SM (96 registers a thread): at 1080p all 68 rows' clusters
// are resident at once, so no row waits for a cluster to free (the
// wavefront is mb_cols + mb_rows MB steps); sharing an SM costs each MB
// less than that saves (1080p analysis 3.06 -> 2.40 ms).
template <bool BATCH>
__global__ void __launch_bounds__(AN_THREADS, 2)
    analysis_kernel(AnArgs a0, const AnArgs* __restrict__ jobs, const uint32_t* __restrict__ items, int n_items) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  __shared__ AnArgs a;  // the current item's job
  __shared__ const double* s_mvb_src;
  __shared__ RefSmem R;
  __shared__ FieldSmem F;
  __shared__ WarpTemp wt[NW];
  // Dynamic shared memory: the four SPLITMV scratch areas, then this
  // call's mv_component_bits table (2 x 2047 doubles).
  extern __shared__ __align__(16) uint8_t dyn_smem[];
  SplitScratch* ss = (SplitScratch*)dyn_smem;
  double* mvb = (double*)(dyn_smem + 4 * sizeof(SplitScratch));
  __shared__ __align__(16) uint16_t xs[MAX_BLOCKS][16];
  __shared__ __align__(16) uint8_t src[256];
  __shared__ double bit_cost[256];
  __shared__ double sbits[5 * 4];  // submv_ref_bits per context and mode
  __shared__ double lterm[5 * 4];  // lambda * (sbits + 0.0): the LEFT/ABOVE/ZERO cost terms
  __shared__ MainOut mo;
  __shared__ uint32_t cand_sad[8];
  __shared__ SplitOut splits[4];
  __shared__ RefDec mydec;
  __shared__ RefDec decs[MAX_REFS];  // rank 0: every reference's decision
  __shared__ __align__(16) MbInfoDev nb[3];  // above, left, aboveleft
  __shared__ Census cen;
  __shared__ Plan plan;
  __shared__ int s_abort, s_qok;
  __shared__ vp8a_mv s_prop_mv;
  __shared__ uint32_t s_prop_sad;
  __shared__ int s_prop_ok;
  // Per-MB cost terms of the mode decision (from the census probabilities),
  // filled during the search by warp 7; per-CTA constants below.
  __shared__ double dz, dnearest, dnear, dnew_bits, dsplit;
  __shared__ double lrbits, pbits[4];
  __shared__ QuarterGeom s_qg;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int k = (int)cl.block_rank();  // the reference this CTA searches
  const int csize = (int)cl.num_blocks();
  const int cid = blockIdx.x / csize, n_clusters = gridDim.x / csize;
  const MePlane& P = a.refs[k];
  uint32_t* dec_slot = (uint32_t*)cl.map_shared_rank(&decs[k], 0);
  const int* abort0 = cl.map_shared_rank(&s_abort, 0);
  if (tid == 0) s_mvb_src = nullptr;
  const int n_it = BATCH ? n_items : a0.mb_rows;
  int cur = -1;

  for (int it = cid; it < n_it; it += n_clusters) {
    int r = it, job = 0;
    if (BATCH) {
      const uint32_t w = items[it];
      job = (int)(w >> 16);
      r = (int)(w & 0xffffu);
    }
    if (job != cur) {
      // Load the job and its per-job constants. The barrier first: the
      // previous MB's last writes still read the old job's pointers.
      __syncthreads();
      if (tid == 0) a = BATCH ? jobs[job] : a0;
      __syncthreads();
      for (int i = tid; i < 256; i += AN_THREADS) bit_cost[i] = a.bit_cost[i];
      if (s_mvb_src != a.mvbits)
        for (int i = tid; i < 2 * MV_BITS_SPAN; i += AN_THREADS) mvb[i] = a.mvbits[i];
      __syncthreads();
      if (tid < 20) {
        const double b = submv_ref_bits(bit_cost, c_submv_probs[tid >> 2], tid & 3);
        sbits[tid] = b;
        lterm[tid] = a.lambda * (b + 0.0);
      } else if (tid < 24) {
        pbits[tid - 20] = mv_partition_bits(bit_cost, tid - 20);
      } else if (tid == 24) {
        // lambda * ref_frame_tree_bits(ref, 128, 128) (src/encoder.rs:9108).
        const double* t = bit_cost;
        const uint8_t id = a.ref_ids[k];
        const double rbits = id == VP8A_REF_LAST ? bb(t, 128, 0)
                             : id == VP8A_REF_GOLDEN ? bb(t, 128, 1) + bb(t, 128, 0)
                                                     : bb(t, 128, 1) + bb(t, 128, 1);
        lrbits = a.lambda * rbits;
      } else if (tid == 32) {
        s_mvb_src = a.mvbits;
      }
      __syncthreads();
      cur = job;
    }
    for (int c = 0; c < a.mb_cols; c++) {
      // Rank 0 waits for the row above; the cluster follows its verdict.
      // MB (r, c) reads the records of its above, left and above-left
      // neighbours only (find_near_mvs, SPLITMV LEFT/ABOVE sub-MVs), so it
      // needs MB (r - 1, c) done. The reference's row contract waits for
      // (r - 1, c + 1) (src/encoder/inter.rs:350-513) because its intra
      // candidates predict from the above-right MB's reconstruction; with
      // intra picking off nothing here reads that MB, and the decisions do
      // not depend on the schedule.
      if (k == 0 && tid == 0) {
        int abort = 0;
        if (r > 0) {
          const unsigned need = (unsigned)(c + 1);
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
      cl.sync();
      if (*abort0) {
        cl.sync();  // rank 0's shared memory stays live until every CTA has read it
        return;
      }
      // Neighbour records (read past L1: rank 0 and other clusters write
      // them) and the edge-replicated source MB (extract_mb,
      // src/encoder.rs:5549).
      if (tid < 3 * 18) {
        const int n = tid / 18, w = tid - n * 18;
        const int nr = n == 1 ? r : r - 1, nc = n == 0 ? c : c - 1;
        const uint32_t* g = (const uint32_t*)(a.infos + (size_t)nr * a.mb_cols + nc);
        // Outside the frame: an intra record (ref_frame in byte 0, the rest 0).
        ((uint32_t*)&nb[n])[w] = (nr >= 0 && nc >= 0) ? __ldcg(g + w) : (w == 0 ? (uint32_t)VP8A_REF_INTRA : 0u);
      }
      for (int i = tid; i < 256; i += AN_THREADS) {
        const int y = min(r * 16 + (i >> 4), a.fh - 1), x = min(c * 16 + (i & 15), a.fw - 1);
        src[i] = a.fy[(size_t)y * a.fys + x];
      }
      __syncthreads();
      const int mbx = c * 16, mby = r * 16;
      if (warp == 0) {
        // The census (every lane, registers only) and the staging plan: lanes
        // 0-8 hold the SPLITMV column vectors (ZERO, the left neighbour's
        // at anchors 0/4/8/12, the above neighbour's at 0-3); vectors with
        // equal integer offsets share one staged block, numbered in column
        // order of first appearance.
        const Census cs = census(nb[0], nb[1], nb[2], c, r, a.mb_cols, a.mb_rows);
        const vp8a_mv m = lane == 0 ? vp8a_mv{0, 0}
                                    : (lane < 5 ? ext_left(nb[1], 4 * ((lane - 1) & 3)) : ext_above(nb[0], (lane - 5) & 3));
        const int ox = int_off(m.col), oy = int_off(m.row);
        const unsigned key = ((unsigned)(uint16_t)oy << 16) | (uint16_t)ox;
        const unsigned cols9 = 0x1ffu;
        const unsigned same = __match_any_sync(FULL, lane < 9 ? key : 0xffffffffu) & cols9;
        const int leader = __ffs(same) - 1;
        const unsigned leaders = __ballot_sync(FULL, lane < 9 && leader == lane);
        if (lane < 9) {
          const int idx = __popc(leaders & ((1u << leader) - 1u));
          plan.colblk[lane] = idx;
          if (leader == lane) {
            plan.box[idx] = ox;
            plan.boy[idx] = oy;
          }
        }
        if (lane == 0) {
          cen = cs;
          const vp8a_mv bp = cs.best_predictor;
          plan.wx0 = mbx + snap_whole(clamp_component(bp.col)) / 4 - WIN_LEAD;
          plan.wy0 = mby + snap_whole(clamp_component(bp.row)) / 4 - WIN_LEAD;
          plan.hn_x = mbx + int_off(cs.nearest.col) - 2;
          plan.hn_y = mby + int_off(cs.nearest.row) - 2;
          plan.hr_x = mbx + int_off(cs.near_.col) - 2;
          plan.hr_y = mby + int_off(cs.near_.row) - 2;
          plan.nblocks = __popc(leaders);
        }
      }
      __syncthreads();
      stage_ref(P, R, plan, mbx, mby, a.words, tid, AN_THREADS);
      __syncthreads();
      field_blocks(R.ws.win, src, F, tid);
      __syncthreads();
      field_sums(F, tid, AN_THREADS);
      staged_block_sads(R, src, plan.nblocks, xs, tid, AN_THREADS);
      __syncthreads();
      const vp8a_mv bp = cen.best_predictor;
      const int cxp = plan.wx0 + WIN_LEAD, cyp = plan.wy0 + WIN_LEAD;  // field centre (plane pixels)
      const FieldView fv{&F, xs, &plan, mbx, mby, cxp, cyp};
      if (warp >= 1 && warp <= 4) {
        split_partition(a, pbits, sbits, lterm, mvb, fv, P, src, bp, nb[0], nb[1], warp - 1, ss[warp - 1],
                        &splits[warp - 1], lane);
      } else {
        // The main group (warps 0 and 5-8) runs the MB search chain while
        // warps 1-4 score the SPLITMV partitions.
        const int slot = warp == 0 ? 0 : warp - 4, mt = slot * 32 + lane;
        if (warp == 0) {
          // ZEROMV SAD and the whole-pel diamond (src/encoder.rs:8560-8576).
          uint32_t z = 0;
          if (lane < 16) z = xs[0][lane];
          z = __reduce_add_sync(FULL, z);
          const vp8a_search_result w =
              diamond_field(F, P, R.ws.win, plan.wx0, plan.wy0, mbx, mby, cxp, cyp, bp, 8, src, lane);
          if (lane == 0) {
            mo.sad_zero = z;
            mo.whole = w;
          }
        } else if (warp == 5) {
          const int er = eighth(cen.nearest.row), ec = eighth(cen.nearest.col);
          const uint32_t sv = subpel_sad(R.halo_nearest, HS, ec & 7, er & 7, src, wt[5].temp, lane);
          if (lane == 0) mo.sad_nearest = sv;
        } else if (warp == 6) {
          const int er = eighth(cen.near_.row), ec = eighth(cen.near_.col);
          const uint32_t sv = subpel_sad(R.halo_near, HS, ec & 7, er & 7, src, wt[6].temp, lane);
          if (lane == 0) mo.sad_near = sv;
        } else if (warp == 8) {
          // The proposed vector's exact SAD (a second NEWMV candidate).
          vp8a_mv pv = {0, 0};
          if (a.props) pv = a.props[((size_t)r * a.mb_cols + c) * a.n_refs + k];
          const bool ok = a.props && !mv_zero(pv) && pv.row >= -1023 && pv.row <= 1023 && pv.col >= -1023 &&
                          pv.col <= 1023;
          uint32_t sv = 0;
          if (ok) sv = sad_at_mv(P, R.ws.win, wt[8].temp, wt[8].halo, plan.wx0, plan.wy0, mbx, mby, pv.row, pv.col,
                                 src, lane);
          if (lane == 0) {
            s_prop_ok = ok;
            s_prop_mv = pv;
            s_prop_sad = sv;
          }
        } else if (warp == 7 && lane == 0) {
          // The mode tree's bits under this MB's census probabilities.
          const double* t = bit_cost;
          const uint8_t* p = cen.p;
          dz = a.lambda * bb(t, p[0], 0);
          dnearest = a.lambda * (bb(t, p[0], 1) + bb(t, p[1], 0));
          dnear = a.lambda * (bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 0));
          dnew_bits = bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 1) + bb(t, p[3], 0);
          dsplit = a.lambda * (bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 1) + bb(t, p[3], 1));
        }
        main_sync();
        // half_pixel_refine_luma around the whole-pel result: planes shared
        // by the group, candidates spread over its warps, first strict
        // minimum in order. For a whole-pel centre inside [-1020, 1020] no
        // candidate is clamped.
        const vp8a_mv hc = mo.whole.mv;
        const int hbx = mbx + hc.col / 4 - plan.wx0, hby = mby + hc.row / 4 - plan.wy0;
        const bool whole_c = hc.row >= -1020 && hc.row <= 1020 && hc.col >= -1020 && hc.col <= 1020 &&
                             !(hc.row & 3) && !(hc.col & 3);
        const uint8_t* spb = a.spl[k];
        const int hix = mbx + hc.col / 4, hiy = mby + hc.row / 4;
        const bool gplanes = spb != nullptr && whole_c && sp_inside(P, hix - 1, hiy - 1) && sp_inside(P, hix, hiy);
        const bool planes = whole_c && hbx >= 3 && hby >= 3 && hbx + 19 <= WS && hby + 19 <= WS;
        if (gplanes || planes) {
          if (gplanes) {
            // Candidate q's prediction is a block of the precomputed plane
            // (fx, fy) = (4 if dc, 4 if dr), one block row per thread.
            if (mt < 128) {
              const int q = mt >> 4, dr = cand_dr(q), dc = cand_dc(q);
              const uint32_t sv = sp_block_sad(spb + (size_t)((dr ? 8 : 0) + (dc ? 2 : 0)) * a.sp_plane, a.sp_pitch,
                                               hix + (dc < 0 ? -1 : 0), hiy + (dr < 0 ? -1 : 0), src, mt & 15);
              if ((mt & 15) == 0) cand_sad[q] = sv;
            }
          } else {
            half_planes_hv(R.ws, hbx, hby, mt);
            main_sync();
            half_planes_d(R.ws, mt);
            main_sync();
            for (int q = slot; q < 8; q += MAIN_WARPS) {
              const uint32_t sv = half_cand_sad(R.ws, q, src, lane);
              if (lane == 0) cand_sad[q] = sv;
            }
          }
          main_sync();
          if (warp == 0) {
            // The first strictly better candidate in order = the smallest
            // (SAD, index) if its SAD beats the centre's.
            const uint32_t m = __reduce_min_sync(FULL, lane < 8 ? (cand_sad[lane] << 3) | (uint32_t)lane : ~0u);
            if (lane == 0) {
              vp8a_mv best = hc;
              uint32_t best_sad = mo.whole.sad;
              const int q = (int)(m & 7u);
              if ((m >> 3) < best_sad) {
                best_sad = m >> 3;
                best.row = (int16_t)(hc.row + 2 * cand_dr(q));
                best.col = (int16_t)(hc.col + 2 * cand_dc(q));
              }
              mo.half = vp8a_search_result{best, best_sad};
              s_qok = quarter_geom(best, mbx, mby, plan.wx0, plan.wy0, s_qg);
            }
          }
        } else if (warp == 0) {
          const vp8a_search_result h = refine(P, R.ws, plan.wx0, plan.wy0, mbx, mby, hc, 2, src, lane, mo.whole.sad);
          if (lane == 0) {
            mo.half = h;
            s_qok = quarter_geom(h.mv, mbx, mby, plan.wx0, plan.wy0, s_qg);
          }
        }
        main_sync();
        // quarter_pixel_refine_luma around the half-pel result; the centre's
        // SAD is the half-pel result's.
        const vp8a_mv qc = mo.half.mv;
        // The eight candidates' blocks span the integer offsets of the
        // columns qc.col - 1 .. qc.col + 1 and rows qc.row - 1 .. qc.row + 1.
        const bool gq = spb != nullptr &&
                        sp_inside(P, mbx + (eighth(clamp_component(qc.col - 1)) >> 3),
                                  mby + (eighth(clamp_component(qc.row - 1)) >> 3)) &&
                        sp_inside(P, mbx + (eighth(clamp_component(qc.col + 1)) >> 3),
                                  mby + (eighth(clamp_component(qc.row + 1)) >> 3));
        if (gq) {
          if (mt < 128) {
            const int q = mt >> 4;
            const int er = eighth(clamp_component(qc.row + cand_dr(q))), ec = eighth(clamp_component(qc.col + cand_dc(q)));
            const uint32_t sv = sp_block_sad(spb + (size_t)((er & 7) / 2 * 4 + (ec & 7) / 2) * a.sp_plane, a.sp_pitch,
                                             mbx + (ec >> 3), mby + (er >> 3), src, mt & 15);
            if ((mt & 15) == 0) cand_sad[q] = sv;
          }
        } else if (s_qok) {
          uint8_t* qh = R.ws.temp;  // the six-tap scratch and half planes are free now
          quarter_planes_h(R.ws.win, qh, s_qg, mt);
          main_sync();
          if (mt < 128) {
            const uint32_t sv = quarter_vsad(qh, s_qg, src, mt);
            if ((mt & 15) == 0) cand_sad[mt >> 4] = sv;
          }
        } else {
          for (int q = slot; q < 8; q += MAIN_WARPS) {
            const int16_t rr = clamp_component(qc.row + cand_dr(q)), cc = clamp_component(qc.col + cand_dc(q));
            const uint32_t sv =
                sad_at_mv(P, R.ws.win, wt[warp].temp, wt[warp].halo, plan.wx0, plan.wy0, mbx, mby, rr, cc, src, lane);
            if (lane == 0) cand_sad[q] = sv;
          }
        }
        main_sync();
        if (warp == 0) {
          const uint32_t m = __reduce_min_sync(FULL, lane < 8 ? (cand_sad[lane] << 3) | (uint32_t)lane : ~0u);
          if (lane == 0) {
            vp8a_mv best = qc;
            uint32_t best_sad = mo.half.sad;
            const int q = (int)(m & 7u);
            if ((m >> 3) < best_sad) {
              best_sad = m >> 3;
              best.row = clamp_component(qc.row + cand_dr(q));
              best.col = clamp_component(qc.col + cand_dc(q));
            }
            mo.quarter = vp8a_search_result{best, best_sad};
          }
        }
      }
      __syncthreads();
      if (tid == 0) {
        // pick_mb_for_ref's mode decision (src/encoder.rs:8598-8652).
        // Every product lambda * bits below is the reference's own; the ones
        // that depend only on the census or the reference were formed
        // during the search.
        const double lambda = a.lambda;
        const MainOut& m = mo;
        const int dr = (int)m.quarter.mv.row - bp.row, dc = (int)m.quarter.mv.col - bp.col;
        const bool in_range = dr >= -1023 && dr <= 1023 && dc >= -1023 && dc <= 1023;
        const double bits_mv = in_range ? mvb[dr + 1023] + mvb[MV_BITS_SPAN + dc + 1023]
                                        : __longlong_as_double(0x7ff0000000000000LL);
        const double j_zero = (double)m.sad_zero + dz;
        const double j_nearest = (double)m.sad_nearest + dnearest;
        const double j_near = (double)m.sad_near + dnear;
        double j_new = (double)m.quarter.sad + lambda * (dnew_bits + bits_mv);
        bool new_ok = in_range && !mv_zero(m.quarter.mv);
        vp8a_mv new_mv = m.quarter.mv;
        if (s_prop_ok) {
          // The proposal replaces the searched vector when strictly cheaper
          // (or when that one is not eligible).
          const int pr = (int)s_prop_mv.row - bp.row, pc = (int)s_prop_mv.col - bp.col;
          if (pr >= -1023 && pr <= 1023 && pc >= -1023 && pc <= 1023) {
            const double j_p =
                (double)s_prop_sad + lambda * (dnew_bits + (mvb[pr + 1023] + mvb[MV_BITS_SPAN + pc + 1023]));
            if (!new_ok || j_p < j_new) {
              j_new = j_p;
              new_mv = s_prop_mv;
              new_ok = true;
            }
          }
        }
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
        if (new_ok && j_new < cj) {
          mode = VP8A_MODE_NEW;
          mv = new_mv;
          cj = j_new;
        }
        int have = 0, sp = -1;
        double sj = 0.0;
        for (int qq = 0; qq < 4; qq++) {
          if (!splits[qq].valid) continue;
          const double total_j = splits[qq].j + dsplit;
          // The stored best already includes bits_split and the
          // comparison adds it again (src/encoder.rs:8679-8683).
          if (!have || total_j < sj + dsplit) {
            sj = total_j;
            sp = qq;
            have = 1;
          }
        }
        if (have && sj < cj) {
          mode = VP8A_MODE_SPLIT;
          mv = splits[sp].split_mvs[15];
          cj = sj;
          pid = sp;
        }
        const double total = cj + lrbits;
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
        mydec.j = cj;
        mydec.total = total;
        mydec.mv = mv;
        mydec.mode = mode;
        mydec.pid = pid;
      }
      __syncthreads();
      // Into rank 0, word by word; the sub-MVs and sub-MV modes come from
      // the chosen partition (ZERO vectors and ZERO4X4 modes otherwise).
      if (tid < (int)(sizeof(RefDec) / 4)) {
        const bool spl = mydec.mode == VP8A_MODE_SPLIT;
        uint32_t w;
        if (tid < 7) w = ((const uint32_t*)&mydec)[tid];
        else if (tid < 23) w = spl ? ((const uint32_t*)splits[mydec.pid].split_mvs)[tid - 7] : 0u;
        else if (tid < 27) w = spl ? ((const uint32_t*)splits[mydec.pid].modes)[tid - 23] : 0x01010101u * VP8A_SUBMV_ZERO;
        else w = 0u;
        dec_slot[tid] = w;
      }
      cl.sync();
      if (k == 0 && warp == 0) {
        // decide_mb_exhaustive's reference comparison: first strict minimum
        // of J + ref_frame_tree_bits in reference order (every lane), then
        // the decision and census records written word by word.
        double best_total = __longlong_as_double(0x7ff0000000000000LL);
        int best_k = -1;
        for (int q = 0; q < a.n_refs; q++)
          if (decs[q].total < best_total) {
            best_total = decs[q].total;
            best_k = q;
          }
        const uint32_t* b = (const uint32_t*)&decs[best_k < 0 ? 0 : best_k];
        const bool ok = best_k >= 0;
        const uint32_t mode = ok ? (uint32_t)decs[best_k].mode : 0u, pid = ok ? (uint32_t)decs[best_k].pid : 0u;
        const uint32_t id = ok ? (uint32_t)a.ref_ids[best_k] : 0u, spl = mode == VP8A_MODE_SPLIT;
        uint32_t* dw = (uint32_t*)(a.dec + (size_t)r * a.mb_cols + c);
        uint32_t* iw = (uint32_t*)(a.infos + (size_t)r * a.mb_cols + c);
        if (lane < 26) {  // vp8a_mb_decision
          uint32_t w;
          if (lane == 0) w = id | (mode & 0xffu) << 8 | (pid & 0xffu) << 16;
          else if (lane == 1) w = b[4];         // mv
          else if (lane < 6) w = b[lane - 2];   // j, total
          else w = b[lane + 1];                 // split_mvs, submv_modes
          dw[lane] = ok ? w : 0u;
        }
        if (lane < 18) {  // the census record
          uint32_t w;
          if (lane == 0) w = id | spl << 8 | spl << 16;
          else if (lane == 1) w = b[4];
          else w = b[lane + 5];
          iw[lane] = ok ? w : 0u;
        }
        __syncwarp();
        // The release orders the warp's record writes before the count.
        if (lane == 0) st_release(&a.progress[r], (unsigned)(c + 1));
      }
      // The next MB's first cluster barrier orders these results.
    }
  }
}

}  // namespace

namespace {

const uint8_t kDefaultMvContexts[2][19] = {
    {162, 128, 225, 146, 172, 147, 214, 39, 156, 128, 129, 132, 75, 145, 178, 206, 239, 254, 254},
    {164, 128, 204, 170, 119, 235, 140, 230, 228, 128, 130, 130, 74, 148, 180, 203, 236, 254, 254}};

// mv_component_bits tables already built by this call, one per distinct
// set of MV contexts.
struct MvBitsCache {
  std::vector<std::pair<vp8a_mv_contexts, const double*>> tables;
};

// Validate one frame's arguments and fill its kernel arguments: inputs
// staged, scratch (census records, row progress) allocated, progress
// counters cleared, the mv_component_bits table built or shared.
vp8a_status prepare_job(vp8a_ctx* ctx, vp8a::Stager& st, MvBitsCache& mc, const vp8a_i420* frame,
                        const vp8a_planes* refs, const uint8_t* ref_ids, uint32_t n_refs,
                        const vp8a_mv_contexts* mv_contexts, double lambda, vp8a_mb_decision* decisions,
                        vp8a_ref_search* trace, AnArgs* out, const vp8a_mv* proposals = nullptr) {
  if (!frame || !refs || !ref_ids || !decisions) {
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
  // rd_lambda is finite and non-negative; the SPLITMV choice compares its
  // costs (sums of non-negative terms) by their bit patterns.
  if (!(lambda >= 0.0) || lambda > 1.0e300) {
    vp8a::set_error("lambda must be a finite, non-negative RD multiplier");
    return VP8A_E_INVALID_ARGUMENT;
  }
  const int mb_cols = (int)((frame->width + 15) / 16), mb_rows = (int)((frame->height + 15) / 16);
  vp8a_status s;
  // The reference ids steer host-side validation; fetch them wherever they live.
  uint8_t ids[MAX_REFS];
  if ((s = st.read_to_host(ref_ids, n_refs, ids)) != VP8A_OK) return s;
  for (uint32_t k = 0; k < n_refs; k++) {
    if ((int)refs[k].mb_cols != mb_cols || (int)refs[k].mb_rows != mb_rows) {
      vp8a::set_error("reference planes do not match the frame's MB grid");
      return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
    }
    if (ids[k] < VP8A_REF_LAST || ids[k] > VP8A_REF_ALTREF || !refs[k].y ||
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
    a.ref_ids[k] = ids[k];
  }
  a.n_refs = (int)n_refs;
  a.mb_cols = mb_cols;
  a.mb_rows = mb_rows;
  if (mv_contexts) a.ctx = *mv_contexts;
  else memcpy(a.ctx.p, kDefaultMvContexts, sizeof kDefaultMvContexts);
  a.lambda = lambda;
  a.bit_cost = ctx->d_bit_cost;
  a.mvbits = nullptr;
  for (const auto& e : mc.tables)
    if (memcmp(&e.first, &a.ctx, sizeof a.ctx) == 0) a.mvbits = e.second;
  if (!a.mvbits) {
    void* dmvb;
    if ((s = st.scratch(sizeof(double) * 2 * MV_BITS_SPAN, &dmvb)) != VP8A_OK) return s;
    mv_bits_table_kernel<<<(2 * MV_BITS_SPAN + 255) / 256, 256, 0, ctx->stream>>>(ctx->d_bit_cost, a.ctx,
                                                                                 (double*)dmvb);
    VP8A_CUDA(cudaGetLastError());
    ctx->launches++;
    a.mvbits = (const double*)dmvb;
    mc.tables.emplace_back(a.ctx, a.mvbits);
  }
  const size_t nmb = (size_t)mb_cols * mb_rows;
  void *dinfo, *dprog, *ddec, *dtr = nullptr;
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
  a.spin_limit = ctx->wait_limit;
  if (proposals) {
    const void* dp;
    if ((s = st.in(proposals, sizeof(vp8a_mv) * nmb * n_refs, &dp)) != VP8A_OK) return s;
    a.props = (const vp8a_mv*)dp;
  }
  // The references' sub-pel planes, built before the wavefront starts.
  if (ctx->subpel_planes) {
    const int pw = mb_cols * 16, ph = mb_rows * 16;
    a.sp_pitch = sp_pitch_of(pw);
    a.sp_plane = a.sp_pitch * (uint64_t)sp_rows_of(ph);
    void* dsp;
    if ((s = st.scratch(16 * a.sp_plane * n_refs, &dsp)) != VP8A_OK) return s;
    for (uint32_t k = 0; k < n_refs; k++) {
      uint8_t* o = (uint8_t*)dsp + 16 * a.sp_plane * k;
      const SubpelArgs sa{a.refs[k].plane, a.refs[k].stride, pw, ph, o, a.sp_pitch, a.sp_plane};
      subpel_planes_kernel<<<dim3((unsigned)(a.sp_pitch / SP_TW), (unsigned)(sp_rows_of(ph) / SP_TH)), 256, 0,
                             ctx->stream>>>(sa);
      VP8A_CUDA(cudaGetLastError());
      ctx->launches++;
      a.spl[k] = o;
    }
  }
  a.words = 1;
  for (uint32_t k = 0; k < n_refs; k++)
    if ((uintptr_t)a.refs[k].plane % 4 != 0 || a.refs[k].stride % 4 != 0) a.words = 0;
  *out = a;
  return VP8A_OK;
}

// One launch over `n_items` MB rows with n_refs-CTA clusters: the frame a0
// (batch false) or the items of the job table (batch true).
template <bool BATCH>
vp8a_status launch_analysis(vp8a_ctx* ctx, int n_refs, const AnArgs& a0, const AnArgs* djobs,
                            const uint32_t* ditems, int n_items) {
  // One CTA per reference, the references of one MB row in one thread-block
  // cluster, two CTAs per SM.
  auto kern = analysis_kernel<BATCH>;
  cudaFuncAttributes fa;
  VP8A_CUDA(cudaFuncGetAttributes(&fa, kern));
  int smem_sm = 0;
  VP8A_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device));
  const int dyn = (int)(4 * sizeof(SplitScratch) + 2 * MV_BITS_SPAN * sizeof(double));
  // At most two CTAs per SM (the register budget allows no more anyway).
  const int pad = std::max(dyn, smem_sm / 3 + 1 - (int)fa.sharedSizeBytes);
  VP8A_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, pad));
  VP8A_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 0));
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = n_refs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(AN_THREADS);
  cfg.dynamicSmemBytes = (size_t)pad;
  cfg.stream = ctx->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(n_refs * (unsigned)n_items);
  int max_clusters = 0;
  VP8A_CUDA(cudaOccupancyMaxActiveClusters(&max_clusters, kern, &cfg));
  if (max_clusters < 1) {
    vp8a::set_error("analysis kernel cannot be resident");
    return VP8A_E_CUDA;
  }
  // Every cluster must be resident at once: items are handed out
  // round-robin and a row waits on the one above it.
  const int n_clusters = std::min(n_items, max_clusters);
  cfg.gridDim = dim3(n_refs * (unsigned)n_clusters);
  VP8A_CUDA(cudaLaunchKernelEx(&cfg, kern, a0, djobs, ditems, n_items));
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return VP8A_OK;
}

// Ends an analysis call. With host buffers the call has waited for its
// kernels (to copy the decisions back), so a wavefront wait that ran out is
// reported now; with device buffers the call stays asynchronous and the
// next vp8a_ctx_synchronize reports it.
vp8a_status finish_analysis(vp8a_ctx* ctx, vp8a::Stager& st) {
  vp8a_status s = st.finish();
  if (s != VP8A_OK) return s;
  return st.touched_host() ? vp8a::check_device_status(ctx) : VP8A_OK;
}

}  // namespace

extern "C" vp8a_status vp8a_analyse_inter_frame(vp8a_ctx* ctx, const vp8a_i420* frame, const vp8a_planes* refs,
                                                const uint8_t* ref_ids, uint32_t n_refs,
                                                const vp8a_mv_contexts* mv_contexts, double lambda,
                                                vp8a_mb_decision* decisions, vp8a_ref_search* trace) {
  if (!ctx) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  MvBitsCache mc;
  AnArgs a{};
  vp8a_status s = prepare_job(ctx, st, mc, frame, refs, ref_ids, n_refs, mv_contexts, lambda, decisions, trace, &a);
  if (s != VP8A_OK) return s;
  if ((s = launch_analysis<false>(ctx, a.n_refs, a, nullptr, nullptr, a.mb_rows)) != VP8A_OK) return s;
  return finish_analysis(ctx, st);
}

extern "C" vp8a_status vp8a_analyse_inter_frame_proposals(vp8a_ctx* ctx, const vp8a_i420* frame,
                                                          const vp8a_planes* refs, const uint8_t* ref_ids,
                                                          uint32_t n_refs, const vp8a_mv_contexts* mv_contexts,
                                                          double lambda, const vp8a_mv* proposals,
                                                          vp8a_mb_decision* decisions, vp8a_ref_search* trace) {
  if (!ctx || !proposals) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  MvBitsCache mc;
  AnArgs a{};
  vp8a_status s =
      prepare_job(ctx, st, mc, frame, refs, ref_ids, n_refs, mv_contexts, lambda, decisions, trace, &a, proposals);
  if (s != VP8A_OK) return s;
  if ((s = launch_analysis<false>(ctx, a.n_refs, a, nullptr, nullptr, a.mb_rows)) != VP8A_OK) return s;
  return finish_analysis(ctx, st);
}

// The work-list analysis; `proposals` (optional) holds, per job, that job's
// proposal vectors or null.
static vp8a_status analyse_frames(vp8a_ctx* ctx, const vp8a_analysis_job* jobs, uint32_t n_jobs,
                                  const vp8a_mv* const* proposals) {
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
  MvBitsCache mc;
  std::vector<AnArgs> args(n_jobs);
  vp8a_status s;
  for (uint32_t j = 0; j < n_jobs; j++) {
    const vp8a_analysis_job& J = jobs[j];
    if ((s = prepare_job(ctx, st, mc, &J.frame, J.refs, J.ref_ids, J.n_refs, J.mv_contexts, J.lambda,
                         J.decisions, J.trace, &args[j], proposals ? proposals[j] : nullptr)) != VP8A_OK)
      return s;
  }
  // One launch per reference count (the cluster size). Within a launch the
  // jobs with the longest wavefront (mb_cols + 2 mb_rows MB steps) come
  // first, so that they start while the short ones fill in behind them.
  for (int nr = 1; nr <= MAX_REFS; nr++) {
    std::vector<uint32_t> order;
    for (uint32_t j = 0; j < n_jobs; j++)
      if (args[j].n_refs == nr) order.push_back(j);
    if (order.empty()) continue;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
      return args[x].mb_cols + 2 * args[x].mb_rows > args[y].mb_cols + 2 * args[y].mb_rows;
    });
    std::vector<AnArgs> table;
    std::vector<uint32_t> items;
    for (uint32_t j : order) {
      const uint32_t q = (uint32_t)table.size();
      table.push_back(args[j]);
      for (int r = 0; r < args[j].mb_rows; r++) items.push_back(q << 16 | (uint32_t)r);
    }
    void *dt, *di;
    if ((s = st.upload(table.data(), sizeof(AnArgs) * table.size(), &dt)) != VP8A_OK) return s;
    if ((s = st.upload(items.data(), sizeof(uint32_t) * items.size(), &di)) != VP8A_OK) return s;
    if ((s = launch_analysis<true>(ctx, nr, table[0], (const AnArgs*)dt, (const uint32_t*)di, (int)items.size())) !=
        VP8A_OK)
      return s;
  }
  return finish_analysis(ctx, st);
}

extern "C" vp8a_status vp8a_analyse_inter_frames(vp8a_ctx* ctx, const vp8a_analysis_job* jobs, uint32_t n_jobs) {
  return analyse_frames(ctx, jobs, n_jobs, nullptr);
}

extern "C" vp8a_status vp8a_analyse_inter_frames_proposals(vp8a_ctx* ctx, const vp8a_analysis_job* jobs,
                                                           uint32_t n_jobs, const vp8a_mv* const* proposals) {
  if (!proposals && n_jobs) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  return analyse_frames(ctx, jobs, n_jobs, proposals);
}
