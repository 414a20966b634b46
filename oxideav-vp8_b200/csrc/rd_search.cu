// rd_search.cu — the RD-effort inter search of decide_mb_rd
// (src/encoder/inter_search.rs:846-1060) for every MB of a frame.
//
// vp8a_rd_inter_search takes each MB's census neighbours as input, so all
// MBs are independent: one warp per MB, four warps per CTA. Per reference
// the warp runs whole_pixel_search (seeds, then the WIDE 8-point and NARROW
// 4-point descents on SAD + sqrt(lambda) * MV bits, :380-495), then for the
// leader (and, by effort, the runner-up) sub_pixel_refine (shared half-pel
// planes over the staged window plus four quarter-pel six-tap probes,
// :499-552) and the free ZERO / NEAREST / NEAR candidates; the cheapest
// candidate wins with the reference's strict '<'. MV rates are the
// reference's f32 table values (MvCostTable, :166-194): each component's
// f64 bit count rounded to f32, summed in f32, widened. The SAD early exits
// of whole_sad never change an outcome (an exiting candidate is rejected
// either way), so SADs are computed in full.
#include "census.cuh"

namespace {
using namespace vp8a_dev;

struct Shape {
  uint32_t descent_rounds;
  int wide_pattern, half_diagonals, quarter, search_other_refs, refine_runner_up;
  unsigned long long split_gate;
};

// EncodeEffort::inter_shape (src/encoder/inter_search.rs:93-161), the
// fields this search reads.
Shape shape_for(uint32_t effort) {
  switch (effort) {
    case VP8A_EFFORT_FASTEST: return Shape{4, 0, 1, 0, 0, 0, ~0ull};
    case VP8A_EFFORT_FAST: return Shape{8, 1, 1, 1, 1, 0, ~0ull};
    case VP8A_EFFORT_BALANCED: return Shape{16, 1, 1, 1, 1, 1, 4ull};
    default: return Shape{32, 1, 1, 1, 1, 1, 0ull};
  }
}

constexpr int RD_WARPS = 4;
constexpr int MAX_REFS = 3;

struct RdArgs {
  const uint8_t* fy;
  uint64_t fys;
  int fw, fh;
  MePlane refs[MAX_REFS];
  uint8_t ref_ids[MAX_REFS];
  int n_refs;
  int mb_cols, mb_rows;
  vp8a_mv_contexts ctx;
  double lambda_sad;
  uint32_t good_enough;
  Shape shape;
  const double* bit_cost;
  const double* mvbits;  // mv_component_bits per context and value (2 x 2047)
  const MbInfoDev* nb;
  vp8a_rd_inter* out;
};

struct Found {
  vp8a_mv mv;
  uint32_t sad;
  double cost;
};

struct RdCensus {
  vp8a_mv best, nearest, near_;
  double mode_bits[5];
};

// MvCostTable::bits: f32 component costs summed in f32; false when the
// differential leaves [-1023, 1023].
__device__ __forceinline__ bool cost_bits(const double* mvb, vp8a_mv mv, vp8a_mv base, double* out) {
  const int dr = mv.row - base.row, dc = mv.col - base.col;
  if (dr < -1023 || dr > 1023 || dc < -1023 || dc > 1023) return false;
  const float s = (float)mv_bits_lookup(mvb, 0, dr) + (float)mv_bits_lookup(mvb, 1, dc);
  *out = (double)s;
  return true;
}

__device__ __forceinline__ uint32_t whole_sad_g(const MePlane& P, int x, int y, const uint8_t* src, int lane) {
  return sad_global16(P, x, y, src, lane);
}

__global__ void __launch_bounds__(RD_WARPS * 32) rd_search_kernel(RdArgs a) {
  __shared__ WarpScratch scratch[RD_WARPS];
  __shared__ __align__(16) uint8_t srcs[RD_WARPS][256];
  __shared__ double bit_cost[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) bit_cost[i] = a.bit_cost[i];
  __syncthreads();
  const double* t = bit_cost;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int idx = blockIdx.x * RD_WARPS + warp;
  if (idx >= a.mb_cols * a.mb_rows) return;
  const int mb_row = idx / a.mb_cols, mb_col = idx - mb_row * a.mb_cols;
  WarpScratch& S = scratch[warp];
  uint8_t* src = srcs[warp];
  for (int i = lane; i < 256; i += 32) {
    const int y = min(mb_row * 16 + (i >> 4), a.fh - 1), x = min(mb_col * 16 + (i & 15), a.fw - 1);
    src[i] = a.fy[(size_t)y * a.fys + x];
  }
  __syncwarp();
  const MbInfoDev above = a.nb[3 * idx], left = a.nb[3 * idx + 1], al = a.nb[3 * idx + 2];
  const int ox = mb_col * 16, oy = mb_row * 16;
  const int to_left = -((mb_col + 1) << 6), to_right = (a.mb_cols - mb_col) << 6;
  const int to_top = -((mb_row + 1) << 6), to_bottom = (a.mb_rows - mb_row) << 6;
  const int rx0 = max(to_left / 4, -255), rx1 = min(to_right / 4, 255);
  const int ry0 = max(to_top / 4, -255), ry1 = min(to_bottom / 4, 255);
  const uint32_t ge = a.good_enough;
  const double ls = a.lambda_sad;
  // The census does not depend on the reference (default sign bias).
  const Census cn = census(above, left, al, mb_col, mb_row, a.mb_cols, a.mb_rows);
  RdCensus cs;
  cs.best = cn.best_predictor;
  cs.nearest = cn.nearest;
  cs.near_ = cn.near_;
  for (int m = 0; m < 5; m++) {  // the `tree` closure (:905-914)
    double bits = 0.0;
    for (int q = 0; q < m; q++) bits += bb(t, cn.p[q], 1);
    if (m < 4) bits += bb(t, cn.p[m], 0);
    cs.mode_bits[m] = bits;
  }
  vp8a_rd_inter o;
  memset(&o, 0, sizeof o);
  for (int k = 0; k < 3; k++) {
    o.found[k].mv = vp8a_mv{0, 0};
    o.found[k].sad = 0xffffffffu;
  }
  Found found[MAX_REFS];
  double total[MAX_REFS];
  bool have[MAX_REFS] = {false, false, false};
  int leader = 0;
  double leader_cost = __longlong_as_double(0x7ff0000000000000LL);
  const double INF = __longlong_as_double(0x7ff0000000000000LL);

  for (int n = 0; n < a.n_refs; n++) {
    const MePlane& P = a.refs[n];
    const uint8_t id = a.ref_ids[n];
    // whole_pixel_search (:380-495).
    Found best = {{0, 0}, 0xffffffffu, INF};
    auto eval = [&](int px, int py) -> bool {
      vp8a_mv mv;
      mv.row = (int16_t)(py * 4);
      mv.col = (int16_t)(px * 4);
      double bits;
      if (!cost_bits(a.mvbits, mv, cs.best, &bits)) return false;
      const double rate = ls * bits;
      if (rate >= best.cost) return false;
      const uint32_t sad = whole_sad_g(P, ox + px, oy + py, src, lane);
      const double cost = (double)sad + rate;
      if (cost < best.cost) {
        best.mv = mv;
        best.sad = sad;
        best.cost = cost;
        return true;
      }
      return false;
    };
    vp8a_mv seeds[6];
    int len = 0;
    seeds[len++] = vp8a_mv{0, 0};
    seeds[len++] = cs.nearest;
    seeds[len++] = cs.near_;
    seeds[len++] = cs.best;
    if (left.ref_frame == id) seeds[len++] = left.mv;
    if (above.ref_frame == id) seeds[len++] = above.mv;
    int tried_x[8], tried_y[8], ntried = 0;
    for (int sidx = 0; sidx < len; sidx++) {
      const int px = clampi((seeds[sidx].col + 2) >> 2, rx0, rx1);
      const int py = clampi((seeds[sidx].row + 2) >> 2, ry0, ry1);
      bool dup = false;
      for (int q = 0; q < ntried; q++)
        if (tried_x[q] == px && tried_y[q] == py) dup = true;
      if (dup) continue;
      if (ntried < 8) {
        tried_x[ntried] = px;
        tried_y[ntried] = py;
        ntried++;
      }
      eval(px, py);
    }
    const bool descend = n == 0 || a.shape.search_other_refs;
    if (descend && best.sad > ge) {
      if (a.shape.wide_pattern && (unsigned long long)best.sad > 4ull * ge) {
        for (uint32_t it = 0; it < a.shape.descent_rounds; it++) {
          const int cx = best.mv.col / 4, cy = best.mv.row / 4;
          bool improved = false;
          const int wdx[8] = {-2, 2, 0, 0, -1, 1, -1, 1}, wdy[8] = {0, 0, -2, 2, -1, -1, 1, 1};
          for (int q = 0; q < 8; q++) {
            const int px = cx + wdx[q], py = cy + wdy[q];
            if (px >= rx0 && px <= rx1 && py >= ry0 && py <= ry1 && eval(px, py)) improved = true;
          }
          if (!improved || best.sad <= ge) break;
        }
      }
      for (uint32_t it = 0; it < a.shape.descent_rounds; it++) {
        if (best.sad <= ge) break;
        const int cx = best.mv.col / 4, cy = best.mv.row / 4;
        bool improved = false;
        const int ndx[4] = {-1, 1, 0, 0}, ndy[4] = {0, 0, -1, 1};
        for (int q = 0; q < 4; q++) {
          const int px = cx + ndx[q], py = cy + ndy[q];
          if (px >= rx0 && px <= rx1 && py >= ry0 && py <= ry1 && eval(px, py)) improved = true;
        }
        if (!improved) break;
      }
    }
    found[n] = best;
    // ref_frame_tree_bits(ref, 128, 128) (src/encoder.rs:9108).
    const double rbits = id == VP8A_REF_LAST ? bb(t, 128, 0)
                         : id == VP8A_REF_GOLDEN ? bb(t, 128, 1) + bb(t, 128, 0)
                                                 : bb(t, 128, 1) + bb(t, 128, 1);
    total[n] = best.cost + ls * rbits;
    if (total[n] < leader_cost) {
      leader_cost = total[n];
      leader = n;
    }
    have[n] = true;
    o.found[n].mv = best.mv;
    o.found[n].sad = best.sad;
    o.n_searched = (uint8_t)(n + 1);
    if (best.sad <= ge) break;
  }

  bool have_best = false;
  double best_cost = 0.0;
  for (int n = 0; n < a.n_refs; n++) {
    if (!have[n]) continue;
    const bool refine = n == leader || (a.shape.refine_runner_up &&
                                        (a.shape.split_gate == 0ull || total[n] < leader_cost * 1.125));
    if (!refine) continue;
    const MePlane& P = a.refs[n];
    const uint8_t id = a.ref_ids[n];
    const double ref_bits = id == VP8A_REF_LAST ? bb(t, 128, 0)
                            : id == VP8A_REF_GOLDEN ? bb(t, 128, 1) + bb(t, 128, 0)
                                                    : bb(t, 128, 1) + bb(t, 128, 1);
    Found f = found[n];
    if (f.sad > ge / 2) {
      // sub_pixel_refine (:499-552): window around the whole-pel start.
      const int wx0 = ox + f.mv.col / 4 - WIN_LEAD, wy0 = oy + f.mv.row / 4 - WIN_LEAD;
      load_window(P, S.win, wx0, wy0, lane);
      uint32_t hs[8];
      half_plane_sads(S, wx0, wy0, ox, oy, f.mv, src, lane, hs);
      const Found start = f;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const int dy = (k < 3) ? -1 : (k < 5 ? 0 : 1);
        const int dx = (k == 0 || k == 3 || k == 5) ? -1 : ((k == 1 || k == 6) ? 0 : 1);
        if (!a.shape.half_diagonals && dx != 0 && dy != 0) continue;
        vp8a_mv mv;
        mv.row = (int16_t)(start.mv.row + 2 * dy);
        mv.col = (int16_t)(start.mv.col + 2 * dx);
        if (abs((int)mv.row) > 1020 || abs((int)mv.col) > 1020) continue;
        double bits;
        if (cost_bits(a.mvbits, mv, cs.best, &bits)) {
          const double cost = (double)hs[k] + ls * bits;
          if (cost < f.cost) f = Found{mv, hs[k], cost};
        }
      }
      if (a.shape.quarter) {
        const vp8a_mv centre = f.mv;
        const int qdx[4] = {-1, 1, 0, 0}, qdy[4] = {0, 0, -1, 1};
        for (int k = 0; k < 4; k++) {
          vp8a_mv mv;
          mv.row = (int16_t)(centre.row + qdy[k]);
          mv.col = (int16_t)(centre.col + qdx[k]);
          if (abs((int)mv.row) > 1022 || abs((int)mv.col) > 1022) continue;
          const uint32_t sad = sad_at_mv(P, S, wx0, wy0, ox, oy, mv.row, mv.col, src, lane);
          double bits;
          if (cost_bits(a.mvbits, mv, cs.best, &bits)) {
            const double cost = (double)sad + ls * bits;
            if (cost < f.cost) f = Found{mv, sad, cost};
          }
        }
      }
    }
    const vp8a_mv zero = {0, 0};
    int mode;
    double mode_bits;
    if (mv_eq(f.mv, zero)) {
      mode = VP8A_MODE_ZERO;
      mode_bits = cs.mode_bits[0];
    } else if (mv_eq(f.mv, cs.nearest)) {
      mode = VP8A_MODE_NEAREST;
      mode_bits = cs.mode_bits[1];
    } else if (mv_eq(f.mv, cs.near_)) {
      mode = VP8A_MODE_NEAR;
      mode_bits = cs.mode_bits[2];
    } else {
      double diff = 0.0;
      cost_bits(a.mvbits, f.mv, cs.best, &diff);
      mode = VP8A_MODE_NEW;
      mode_bits = cs.mode_bits[3] + diff;
    }
    auto consider = [&](int md, vp8a_mv mv, uint32_t sad, double bits) {
      const double cost = (double)sad + ls * bits;
      if (!have_best || cost < best_cost) {
        have_best = true;
        best_cost = cost;
        o.ref_frame = id;
        o.mode = (uint8_t)md;
        o.mv = mv;
        o.sad = sad;
        o.cost = cost;
        o.bits = bits;
      }
    };
    consider(mode, f.mv, f.sad, ref_bits + mode_bits);
    const vp8a_mv fm[3] = {zero, cs.nearest, cs.near_};
    for (int k = 0; k < 3; k++) {
      if (k == 1 && mv_eq(cs.nearest, zero)) continue;
      if (k == 2 && (mv_eq(cs.near_, zero) || mv_eq(cs.near_, cs.nearest))) continue;
      const vp8a_mv mv = fm[k];
      if (mv_eq(mv, f.mv)) continue;
      const uint32_t sad = ((mv.row & 3) == 0 && (mv.col & 3) == 0)
                               ? whole_sad_g(P, ox + mv.col / 4, oy + mv.row / 4, src, lane)
                               : sad_at_mv(P, S, -(1 << 28), -(1 << 28), ox, oy, mv.row, mv.col, src, lane);
      consider(k, mv, sad, ref_bits + cs.mode_bits[k]);
    }
  }
  o.leader = (uint8_t)leader;
  if (lane == 0) a.out[idx] = o;
}

}  // namespace

extern "C" vp8a_status vp8a_rd_inter_search(vp8a_ctx* ctx, const vp8a_i420* frame, const vp8a_planes* refs,
                                            const uint8_t* ref_ids, uint32_t n_refs,
                                            const vp8a_mv_contexts* mv_contexts, double lambda, uint32_t y1_ac,
                                            uint32_t effort, const vp8a_mb_info* neighbours, vp8a_rd_inter* out) {
  if (!ctx || !frame || !refs || !ref_ids || !neighbours || !out) {
    vp8a::set_error("null argument");
    return VP8A_E_INVALID_ARGUMENT;
  }
  if (frame->width == 0 || frame->height == 0 || frame->width > 0x3FFF || frame->height > 0x3FFF) {
    vp8a::set_error("invalid dimensions");
    return VP8A_E_INVALID_DIMENSIONS;
  }
  if (n_refs == 0 || n_refs > (uint32_t)MAX_REFS || effort > VP8A_EFFORT_THOROUGH) {
    vp8a::set_error("n_refs must be 1..3 and effort a VP8A_EFFORT_* value");
    return VP8A_E_INVALID_ARGUMENT;
  }
  const int mb_cols = (int)((frame->width + 15) / 16), mb_rows = (int)((frame->height + 15) / 16);
  VP8A_CUDA(cudaSetDevice(ctx->device));
  vp8a::Stager st(ctx);
  vp8a_status s;
  uint8_t ids[MAX_REFS];
  if ((s = st.read_to_host(ref_ids, n_refs, ids)) != VP8A_OK) return s;
  for (uint32_t k = 0; k < n_refs; k++) {
    if ((int)refs[k].mb_cols != mb_cols || (int)refs[k].mb_rows != mb_rows) {
      vp8a::set_error("reference planes do not match the frame's MB grid");
      return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
    }
    if (ids[k] < VP8A_REF_LAST || ids[k] > VP8A_REF_ALTREF || !refs[k].y || refs[k].y_stride < (uint64_t)mb_cols * 16) {
      vp8a::set_error("bad reference id, plane or stride");
      return VP8A_E_INVALID_ARGUMENT;
    }
  }
  if (!frame->y || frame->y_stride < frame->width) {
    vp8a::set_error("bad source plane");
    return VP8A_E_INVALID_ARGUMENT;
  }
  RdArgs a{};
  const void* d;
  if ((s = st.in(frame->y, frame->y_stride * (size_t)(frame->height - 1) + frame->width, &d)) != VP8A_OK) return s;
  a.fy = (const uint8_t*)d;
  a.fys = frame->y_stride;
  a.fw = (int)frame->width;
  a.fh = (int)frame->height;
  for (uint32_t k = 0; k < n_refs; k++) {
    const size_t bytes = refs[k].y_stride * (size_t)(mb_rows * 16 - 1) + (size_t)mb_cols * 16;
    if ((s = st.in(refs[k].y, bytes, &d)) != VP8A_OK) return s;
    a.refs[k] = MePlane{(const uint8_t*)d, refs[k].y_stride, mb_cols * 16, mb_rows * 16};
    a.ref_ids[k] = ids[k];
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
  // decide_mb_rd (:850-866): sqrt(lambda), good_enough from y1_ac.
  a.lambda_sad = std::sqrt(lambda);
  const uint32_t qpix = std::max(y1_ac / 8u, 1u);
  a.good_enough = 256u * qpix / 2u;
  a.shape = shape_for(effort);
  a.bit_cost = ctx->d_bit_cost;
  const size_t nmb = (size_t)mb_cols * mb_rows;
  if ((s = st.in(neighbours, sizeof(vp8a_mb_info) * nmb * 3, &d)) != VP8A_OK) return s;
  a.nb = (const MbInfoDev*)d;
  void *dout, *dmvb;
  if ((s = st.out(out, sizeof(vp8a_rd_inter) * nmb, &dout)) != VP8A_OK) return s;
  a.out = (vp8a_rd_inter*)dout;
  if ((s = st.scratch(sizeof(double) * 2 * MV_BITS_SPAN, &dmvb)) != VP8A_OK) return s;
  mv_bits_table_kernel<<<(2 * MV_BITS_SPAN + 255) / 256, 256, 0, ctx->stream>>>(ctx->d_bit_cost, a.ctx,
                                                                               (double*)dmvb);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  a.mvbits = (const double*)dmvb;
  rd_search_kernel<<<vp8a::grid_for(nmb, RD_WARPS), RD_WARPS * 32, 0, ctx->stream>>>(a);
  VP8A_CUDA(cudaGetLastError());
  ctx->launches++;
  return st.finish();
}
