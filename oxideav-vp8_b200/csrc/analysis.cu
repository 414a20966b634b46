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
// Inside a CTA, each reference gets one "main" warp (ZEROMV, diamond,
// half, quarter, NEAREST, NEAR) and four SPLITMV warps (one per
// partition), all reading the reference window the main warp staged. The
// f64 RD decision runs on one thread with the reference's operation order;
// the library is built with -fmad=false so no multiply-add is fused.
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
  MbInfoDev* infos;
  unsigned* progress;
  unsigned* status;
  vp8a_mb_decision* dec;
  vp8a_ref_search* trace;
  unsigned long long spin_limit;
};

// group_sad_at_whole_mv(_shaped) (src/encoder.rs:7650-7797): SAD over the
// group rectangle at the integer part of the eighth-pel vector.
__device__ uint32_t group_sad(const MePlane& P, const uint8_t* win, int wx0, int wy0, int mbx, int mby,
                              const uint8_t* src, int row0, int col0, int gw, int gh, vp8a_mv mv, int lane) {
  const int bx = mbx + (eighth(mv.col) >> 3), by = mby + (eighth(mv.row) >> 3);
  const int lx = bx + col0 - wx0, ly = by + row0 - wy0;
  const bool inwin = lx >= 0 && ly >= 0 && lx + gw <= WS && ly + gh <= WS;
  uint32_t s = 0;
  const int n = gw * gh;
  for (int i = lane; i < n; i += 32) {
    const int rr = i / gw, cc = i - rr * gw;
    int ref;
    if (inwin) ref = win[(ly + rr) * WS + lx + cc];
    else
      ref = P.plane[(size_t)clampi(by + row0 + rr, 0, P.height - 1) * P.stride + clampi(bx + col0 + cc, 0, P.width - 1)];
    int d = (int)src[(row0 + rr) * 16 + col0 + cc] - ref;
    s += (uint32_t)(d < 0 ? -d : d);
  }
  return __reduce_add_sync(FULL, s);
}

struct SplitOut {
  double j;
  vp8a_mv split_mvs[16];
  uint8_t modes[16];
  int valid;
};

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

// score_split_partition (src/encoder.rs:8080-8246) on one warp.
__device__ void split_partition(const AnArgs& a, const double* t, const MePlane& P, const uint8_t* win, int wx0,
                                int wy0, int mbx, int mby, const uint8_t* src, vp8a_mv bp, const MbInfoDev& above,
                                const MbInfoDev& left, int pid, SplitOut* out, int lane) {
  vp8a_mv split[16];
  for (int i = 0; i < 16; i++) split[i] = vp8a_mv{0, 0};
  uint8_t modes[16];
  for (int i = 0; i < 16; i++) modes[i] = VP8A_SUBMV_ZERO;
  uint32_t total_sad = 0;
  double total_bits = 0.0;
  const int ngroups = pid == 3 ? 16 : (pid == 2 ? 4 : 2);
  for (int g = 0; g < ngroups; g++) {
    // Members (ascending) and bounding rectangle (PartitionGroups::build).
    int anchor = -1, min_r = 3, max_r = 0, min_c = 3, max_c = 0;
    for (int b = 0; b < 16; b++)
      if (c_partitions[pid][b] == g) {
        if (anchor < 0) anchor = b;
        min_r = min(min_r, b >> 2);
        max_r = max(max_r, b >> 2);
        min_c = min(min_c, b & 3);
        max_c = max(max_c, b & 3);
      }
    const int row0 = min_r * 4, col0 = min_c * 4, gw = (max_c + 1 - min_c) * 4, gh = (max_r + 1 - min_r) * 4;
    // left_block_mv / above_block_mv (src/near_mv.rs:722-760).
    vp8a_mv lmv, amv;
    if ((anchor & 3) == 0) {
      lmv = left.ref_frame == VP8A_REF_INTRA ? vp8a_mv{0, 0} : (left.is_split ? left.split_mvs[anchor + 3] : left.mv);
    } else {
      lmv = split[anchor - 1];
    }
    if (anchor < 4) {
      amv = above.ref_frame == VP8A_REF_INTRA ? vp8a_mv{0, 0} : (above.is_split ? above.split_mvs[anchor + 12] : above.mv);
    } else {
      amv = split[anchor - 4];
    }
    int ctxi;
    {
      const bool lez = mv_zero(lmv), aez = mv_zero(amv), lea = mv_eq(lmv, amv);
      ctxi = (lea && lez) ? 4 : (lea ? 3 : (aez ? 2 : (lez ? 1 : 0)));
    }
    const uint8_t* probs = c_submv_probs[ctxi];
    // group_small_diamond_search (src/encoder.rs:7812-7879).
    vp8a_mv best;
    best.row = (int16_t)clampi((bp.row / 4) * 4, -1023, 1023);
    best.col = (int16_t)clampi((bp.col / 4) * 4, -1023, 1023);
    uint32_t best_sad = group_sad(P, win, wx0, wy0, mbx, mby, src, row0, col0, gw, gh, best, lane);
    for (int it = 0; it < 4; it++) {
      bool improved = false;
      const int dr[4] = {-4, 4, 0, 0}, dc[4] = {0, 0, -4, 4};
#pragma unroll
      for (int d = 0; d < 4; d++) {
        vp8a_mv c;
        c.row = (int16_t)clampi(best.row + dr[d], -1023, 1023);
        c.col = (int16_t)clampi(best.col + dc[d], -1023, 1023);
        if (mv_eq(c, best)) continue;
        uint32_t s = group_sad(P, win, wx0, wy0, mbx, mby, src, row0, col0, gw, gh, c, lane);
        if (s < best_sad) {
          best_sad = s;
          best = c;
          improved = true;
        }
      }
      if (!improved) break;
    }
    // Score LEFT4X4, ABOVE4X4, ZERO4X4, NEW4X4.
    int best_mode = VP8A_SUBMV_ZERO;
    vp8a_mv best_mv = {0, 0}, best_diff = {0, 0};
    double best_j = __longlong_as_double(0x7ff0000000000000LL);
    const vp8a_mv cm[3] = {lmv, amv, vp8a_mv{0, 0}};
    for (int m = 0; m < 3; m++) {
      const double sad = (double)group_sad(P, win, wx0, wy0, mbx, mby, src, row0, col0, gw, gh, cm[m], lane);
      const double mode_bits = submv_ref_bits(t, probs, m);
      const double j = sad + a.lambda * (mode_bits + 0.0);
      if (j < best_j) {
        best_j = j;
        best_mode = m;
        best_mv = cm[m];
        best_diff = vp8a_mv{0, 0};
      }
    }
    const int dr = (int)best.row - bp.row, dc = (int)best.col - bp.col;
    if (dr >= -1023 && dr <= 1023 && dc >= -1023 && dc <= 1023) {
      const double diff_bits = mv_component_bits(t, a.ctx.p[0], dr) + mv_component_bits(t, a.ctx.p[1], dc);
      const double mode_bits = submv_ref_bits(t, probs, VP8A_SUBMV_NEW);
      const double j = (double)best_sad + a.lambda * (mode_bits + diff_bits);
      if (j < best_j) {
        best_j = j;
        best_mode = VP8A_SUBMV_NEW;
        best_mv = best;
        best_diff.row = (int16_t)dr;
        best_diff.col = (int16_t)dc;
      }
    }
    if (!isfinite(best_j)) {
      if (lane == 0) out->valid = 0;
      return;
    }
    const uint32_t gs = group_sad(P, win, wx0, wy0, mbx, mby, src, row0, col0, gw, gh, best_mv, lane);
    for (int b = 0; b < 16; b++)
      if (c_partitions[pid][b] == g) split[b] = best_mv;
    total_sad += gs;
    total_bits += submv_ref_bits(t, probs, best_mode);
    if (best_mode == VP8A_SUBMV_NEW)
      total_bits += mv_component_bits(t, a.ctx.p[0], best_diff.row) + mv_component_bits(t, a.ctx.p[1], best_diff.col);
    modes[g] = (uint8_t)best_mode;
  }
  const double partition_bits = mv_partition_bits(t, pid);
  if (lane == 0) {
    out->j = (double)total_sad + a.lambda * (partition_bits + total_bits);
    for (int i = 0; i < 16; i++) {
      out->split_mvs[i] = split[i];
      out->modes[i] = modes[i];
    }
    out->valid = 1;
  }
}

struct MainOut {
  uint32_t sad_zero, sad_nearest, sad_near;
  vp8a_search_result whole, half, quarter;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__global__ void __launch_bounds__(MAX_REFS* WARPS_PER_REF * 32) analysis_kernel(AnArgs a) {
  __shared__ WarpScratch scratch[MAX_REFS];
  __shared__ __align__(16) uint8_t src[256];
  __shared__ double bit_cost[256];
  __shared__ MainOut mains[MAX_REFS];
  __shared__ SplitOut splits[MAX_REFS][4];
  __shared__ MbInfoDev nb[3];  // above, left, aboveleft
  __shared__ Census cen;
  __shared__ int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ref = warp / WARPS_PER_REF, role = warp % WARPS_PER_REF;  // role 0 = main, 1..4 = split pid
  for (int i = threadIdx.x; i < 256; i += blockDim.x) bit_cost[i] = a.bit_cost[i];
  __syncthreads();
  const MbInfoDev border = {VP8A_REF_INTRA, 0, 0, 0, {0, 0}, {}};

  for (int r = blockIdx.x; r < a.mb_rows; r += gridDim.x) {
    for (int c = 0; c < a.mb_cols; c++) {
      if (threadIdx.x == 0) {
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
            __nanosleep(128);
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
      if (threadIdx.x < 3) {
        const int k = threadIdx.x;
        const int nr = k == 1 ? r : r - 1, nc = k == 0 ? c : c - 1;
        nb[k] = (nr >= 0 && nc >= 0) ? a.infos[(size_t)nr * a.mb_cols + nc] : border;
      }
      for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        const int y = min(r * 16 + (i >> 4), a.fh - 1), x = min(c * 16 + (i & 15), a.fw - 1);
        src[i] = a.fy[(size_t)y * a.fys + x];
      }
      __syncthreads();
      if (threadIdx.x == 0) cen = census(nb[0], nb[1], nb[2], c, r, a.mb_cols, a.mb_rows);
      __syncthreads();
      const int mbx = c * 16, mby = r * 16;
      const vp8a_mv bp = cen.best_predictor;
      const int cx = snap_whole(clamp_component(bp.col)) / 4, cy = snap_whole(clamp_component(bp.row)) / 4;
      const int wx0 = mbx + cx - WIN_LEAD, wy0 = mby + cy - WIN_LEAD;
      if (ref < a.n_refs && role == 0) load_window(a.refs[ref], scratch[ref].win, wx0, wy0, lane);
      __syncthreads();
      if (ref < a.n_refs) {
        const MePlane& P = a.refs[ref];
        WarpScratch& S = scratch[ref];
        if (role == 0) {
          MainOut m;
          m.sad_zero = sad_whole_at(P, S.win, wx0, wy0, mbx, mby, src, lane);
          m.whole = diamond(P, S, wx0, wy0, mbx, mby, bp, 8, src, lane);
          m.half = refine(P, S, wx0, wy0, mbx, mby, m.whole.mv, 2, src, lane);
          m.quarter = refine(P, S, wx0, wy0, mbx, mby, m.half.mv, 1, src, lane);
          m.sad_nearest = sad_at_mv(P, S, wx0, wy0, mbx, mby, cen.nearest.row, cen.nearest.col, src, lane);
          m.sad_near = sad_at_mv(P, S, wx0, wy0, mbx, mby, cen.near_.row, cen.near_.col, src, lane);
          if (lane == 0) mains[ref] = m;
        } else {
          split_partition(a, bit_cost, P, S.win, wx0, wy0, mbx, mby, src, bp, nb[0], nb[1], role - 1,
                          &splits[ref][role - 1], lane);
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        const double* t = bit_cost;
        const double lambda = a.lambda;
        const uint8_t* p = cen.p;
        double best_total = __longlong_as_double(0x7ff0000000000000LL);
        int best_k = -1, best_mode = 0, best_pid = VP8A_PART_NONE;
        vp8a_mv best_mv = {0, 0};
        double best_j = 0.0;
        for (int k = 0; k < a.n_refs; k++) {
          const MainOut& m = mains[k];
          const double bits_zero = bb(t, p[0], 0);
          const double bits_nearest = bb(t, p[0], 1) + bb(t, p[1], 0);
          const double bits_near = bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 0);
          const double bits_new = bb(t, p[0], 1) + bb(t, p[1], 1) + bb(t, p[2], 1) + bb(t, p[3], 0);
          const int dr = (int)m.quarter.mv.row - bp.row, dc = (int)m.quarter.mv.col - bp.col;
          const bool in_range = dr >= -1023 && dr <= 1023 && dc >= -1023 && dc <= 1023;
          const double bits_mv = in_range ? mv_component_bits(t, a.ctx.p[0], dr) + mv_component_bits(t, a.ctx.p[1], dc)
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
          for (int q = 0; q < 4; q++) {
            if (!splits[k][q].valid) continue;
            const double total_j = splits[k][q].j + lambda * bits_split;
            // The stored best already includes bits_split and the
            // comparison adds it again (src/encoder.rs:8679-8683).
            if (!have || total_j < sj + lambda * bits_split) {
              sj = total_j;
              sp = q;
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
          if (total < best_total) {
            best_total = total;
            best_k = k;
            best_mode = mode;
            best_mv = mv;
            best_j = cj;
            best_pid = pid;
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
