// emit.cpp — the P-frame bitstream writer: the §19.2 inter-frame header,
// the §16/§17 macroblock-mode layer and the §13 residual tokens of
// encode_p_frame_multi_ref_inner_driven (src/encoder.rs:11214-11720 of
// oxideav-vp8), from the analysis decisions and the quantised coefficients
// the device reconstruction produces.
//
// This is host code on purpose: a boolean entropy coder is a serial chain
// (every decision's interval depends on the previous one), which a CPU core
// runs several times faster than one GPU thread, and the writer reads only
// the per-MB decisions and coefficients the device already copied out. The
// token partitions (rows r % n) are independent coders: their tokens are
// coded on one host thread each once the per-block nonzero flags of the
// whole frame (the §13.3 above/left contexts) are known.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/vp8a.h"
#include "coeff_tables.h"

namespace vp8a_emit {
namespace {

// RFC 6386 §7.3 boolean encoder (BoolEncoder, src/encoder.rs:255-500):
// `bottom` holds the low end of the interval with 24 bits of headroom;
// a byte is complete after `pending` more shifts.
struct BoolWriter {
  std::vector<uint8_t> out;
  uint32_t range = 255, bottom = 0;
  int pending = 24;

  void carry() {
    for (size_t i = out.size(); i-- > 0;) {
      if (out[i] != 255) {
        out[i]++;
        return;
      }
      out[i] = 0;
    }
  }
  void put(int prob, bool bit) {
    const uint32_t split = 1 + (((range - 1) * (uint32_t)prob) >> 8);
    // Branch-free choice of the sub-interval: the bit is data, not control.
    const uint32_t m = 0u - (uint32_t)bit;
    bottom += split & m;
    range = split + ((range - 2 * split) & m);
    const int shift = __builtin_clz(range) - 24;  // range in [1, 255]
    range <<= shift;
    if (shift < pending) {
      bottom <<= shift;
      pending -= shift;
      return;
    }
    // The pending byte completes inside this normalisation: its carry bit
    // sits at bit 31 one shift before the byte leaves.
    bottom <<= pending - 1;
    if (bottom & 0x80000000u) carry();
    bottom <<= 1;
    out.push_back((uint8_t)(bottom >> 24));
    bottom &= 0xFFFFFFu;
    const int rest = shift - pending;
    bottom <<= rest;
    pending = 8 - rest;
  }
  void literal(uint32_t v, int bits) {
    while (bits-- > 0) put(128, (v >> bits) & 1);
  }
  void signed_literal(int v, int bits) {
    literal((uint32_t)std::abs(v), bits);
    put(128, v < 0);
  }
  // flush_bool_encoder (RFC 6386 §7.3): settle a carry into the output,
  // then write the four bytes that hold the rest of `bottom`.
  std::vector<uint8_t> finish() {
    const int c = pending;
    uint32_t v = bottom;
    if (v & (1u << (32 - c))) carry();
    v <<= c & 7;
    for (int k = c >> 3; k > 0; k--) v <<= 8;
    for (int k = 0; k < 4; k++) {
      out.push_back((uint8_t)(v >> 24));
      v <<= 8;
    }
    return std::move(out);
  }
};

// ------------------------------------------------------------ §13 tables

const uint8_t kBands[16] = {0, 1, 2, 3, 6, 4, 5, 6, 6, 6, 6, 6, 6, 6, 6, 7};
const uint8_t kZigzag[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};
// DCT_extra probabilities (Pcat1..Pcat6) and the category bases.
const uint8_t kCat1[] = {159}, kCat2[] = {165, 145}, kCat3[] = {173, 148, 140},
              kCat4[] = {176, 155, 140, 135}, kCat5[] = {180, 157, 141, 134, 130},
              kCat6[] = {254, 254, 243, 230, 196, 177, 153, 140, 133, 130, 129};
struct Cat {
  int base, n;
  const uint8_t* p;
};
const Cat kCats[6] = {{5, 1, kCat1}, {7, 2, kCat2}, {11, 3, kCat3}, {19, 4, kCat4}, {35, 5, kCat5}, {67, 11, kCat6}};
// The path of every token through the §13.2 coefficient tree, as
// (node, bit) steps from the root; tokens 0..4 = DCT_0, ONE .. FOUR,
// 5..10 = cat1..cat6, 11 = EOB.
struct Path {
  uint8_t n, node[8], bit[8];
};
const Path kTokenPath[12] = {
    {2, {0, 1}, {1, 0}},                         // DCT_0
    {3, {0, 1, 2}, {1, 1, 0}},                   // ONE
    {5, {0, 1, 2, 3, 4}, {1, 1, 1, 0, 0}},       // TWO
    {6, {0, 1, 2, 3, 4, 5}, {1, 1, 1, 0, 1, 0}}, // THREE
    {6, {0, 1, 2, 3, 4, 5}, {1, 1, 1, 0, 1, 1}}, // FOUR
    {6, {0, 1, 2, 3, 6, 7}, {1, 1, 1, 1, 0, 0}}, // cat1
    {6, {0, 1, 2, 3, 6, 7}, {1, 1, 1, 1, 0, 1}}, // cat2
    {7, {0, 1, 2, 3, 6, 8, 9}, {1, 1, 1, 1, 1, 0, 0}},   // cat3
    {7, {0, 1, 2, 3, 6, 8, 9}, {1, 1, 1, 1, 1, 0, 1}},   // cat4
    {7, {0, 1, 2, 3, 6, 8, 10}, {1, 1, 1, 1, 1, 1, 0}},  // cat5
    {7, {0, 1, 2, 3, 6, 8, 10}, {1, 1, 1, 1, 1, 1, 1}},  // cat6
    {1, {0}, {0}},                                // EOB
};

int token_of(int a) {
  if (a <= 4) return a;
  for (int k = 5; k >= 0; k--)
    if (a >= kCats[k].base) return 5 + k;
  return 0;
}

using Probs = uint8_t[4][8][3][11];

// encode_coeff_block_into (src/encoder.rs:1915): one block's tokens in
// zigzag order from `first`; returns the block's nonzero count.
int code_block(BoolWriter& w, const Probs& probs, int plane, int first, int ctx, const int16_t* raster) {
  int16_t scan[16];
  int last = -1;
  for (int i = 0; i < 16; i++) {
    scan[i] = raster[kZigzag[i]];
    if (i >= first && scan[i] != 0) last = i;
  }
  bool after_zero = false;
  int nonzero = 0;
  for (int i = first; i < 16; i++) {
    const uint8_t* p = probs[plane][kBands[i]][ctx];
    const int a = i > last ? 0 : std::abs((int)scan[i]);
    const int tok = i > last ? 11 : token_of(a);
    const Path& path = kTokenPath[tok];
    for (int s = after_zero ? 1 : 0; s < path.n; s++) w.put(p[path.node[s]], path.bit[s]);
    if (tok == 11) break;
    if (tok >= 5) {
      const Cat& c = kCats[tok - 5];
      const int extra = a - c.base;
      for (int j = 0; j < c.n; j++) w.put(c.p[j], (extra >> (c.n - 1 - j)) & 1);
    }
    if (a != 0) {
      w.put(128, scan[i] < 0);
      nonzero++;
    }
    ctx = a == 0 ? 0 : (a == 1 ? 1 : 2);
    after_zero = tok == 0;
  }
  return nonzero;
}

// ---------------------------------------------------- §16.3 / §17 helpers

const uint8_t kCountsToProbs[6][4] = {{7, 1, 1, 143},    {14, 18, 14, 107}, {135, 64, 57, 68},
                                      {60, 56, 128, 65}, {159, 134, 128, 34}, {234, 188, 128, 28}};
const uint8_t kPartitionMap[4][16] = {{0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1},
                                      {0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1, 1},
                                      {0, 0, 1, 1, 0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 3, 3},
                                      {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}};
const int kPartitionGroups[4] = {2, 2, 4, 16};
const uint8_t kPartitionProbs[3] = {110, 111, 150};
const uint8_t kSubmvProbs[5][3] = {{147, 136, 18}, {106, 145, 1}, {179, 121, 1}, {223, 1, 34}, {208, 1, 1}};
const uint8_t kMvUpdateProbs[2][19] = {
    {237, 246, 253, 253, 254, 254, 254, 254, 254, 254, 254, 254, 254, 254, 250, 250, 252, 254, 254},
    {231, 243, 245, 253, 254, 254, 254, 254, 254, 254, 254, 254, 254, 254, 251, 251, 254, 254, 254}};
const uint8_t kDefaultMvContexts[2][19] = {
    {162, 128, 225, 146, 172, 147, 214, 39, 156, 128, 129, 132, 75, 145, 178, 206, 239, 254, 254},
    {164, 128, 204, 170, 119, 235, 140, 230, 228, 128, 130, 130, 74, 148, 180, 203, 236, 254, 254}};
const int8_t kSmallMvTree[14] = {2, 8, 4, 6, -0, -1, -2, -3, 10, 12, -4, -5, -6, -7};

struct Info {  // MbInfo (src/near_mv.rs:127)
  uint8_t ref = VP8A_REF_INTRA;
  bool split = false;
  vp8a_mv mv{0, 0};
  vp8a_mv smv[16]{};
};

bool eq(vp8a_mv a, vp8a_mv b) { return a.row == b.row && a.col == b.col; }
bool zero(vp8a_mv a) { return a.row == 0 && a.col == 0; }

struct Near {
  vp8a_mv best;
  uint8_t p[4];
};

// find_near_mvs (src/near_mv.rs:310-402, default sign bias), the clamp of
// near.mvs[0] (MvClampRect::for_mb / clamp_mv, :236-283) and mv_ref_probs
// (:404).
Near census(const Info& above, const Info& left, const Info& al, int col, int row, int cols, int rows) {
  vp8a_mv mvs[4] = {};
  int cnt[4] = {0, 0, 0, 0}, k = 0;
  if (above.ref != VP8A_REF_INTRA) {
    if (!zero(above.mv)) mvs[++k] = above.mv;
    cnt[k] += 2;
  }
  if (left.ref != VP8A_REF_INTRA) {
    if (!zero(left.mv)) {
      if (!eq(left.mv, mvs[k])) mvs[++k] = left.mv;
      cnt[k] += 2;
    } else {
      cnt[0] += 2;
    }
  }
  if (al.ref != VP8A_REF_INTRA) {
    if (!zero(al.mv)) {
      if (!eq(al.mv, mvs[k])) mvs[++k] = al.mv;
      cnt[k] += 1;
    } else {
      cnt[0] += 1;
    }
  }
  if (cnt[3] != 0 && eq(mvs[k], mvs[1])) cnt[1] += 1;
  cnt[3] = (above.split + left.split) * 2 + al.split;
  if (cnt[2] > cnt[1]) {
    std::swap(cnt[1], cnt[2]);
    std::swap(mvs[1], mvs[2]);
  }
  if (cnt[1] >= cnt[0]) mvs[0] = mvs[1];
  const int lo_c = -((col + 1) << 6), hi_c = (cols - col) << 6;
  const int lo_r = -((row + 1) << 6), hi_r = (rows - row) << 6;
  Near n;
  n.best.col = (int16_t)std::min(std::max((int)mvs[0].col, lo_c), hi_c);
  n.best.row = (int16_t)std::min(std::max((int)mvs[0].row, lo_r), hi_r);
  for (int i = 0; i < 4; i++) n.p[i] = kCountsToProbs[cnt[i]][i];
  return n;
}

vp8a_mv above_block(const vp8a_mv* cur, const Info& above, int b) {
  if (b >= 4) return cur[b - 4];
  if (above.ref == VP8A_REF_INTRA) return vp8a_mv{0, 0};
  return above.split ? above.smv[b + 12] : above.mv;
}

vp8a_mv left_block(const vp8a_mv* cur, const Info& left, int b) {
  if (b & 3) return cur[b - 1];
  if (left.ref == VP8A_REF_INTRA) return vp8a_mv{0, 0};
  return left.split ? left.smv[b + 3] : left.mv;
}

int submv_context(vp8a_mv l, vp8a_mv a) {  // submv_ref_context (src/near_mv.rs:640)
  if (eq(l, a)) return zero(l) ? 4 : 3;
  if (zero(a)) return 2;
  if (zero(l)) return 1;
  return 0;
}

// write_mv_component (src/motion_vector.rs:292): is_short, short tree or
// long bits (0-2, 9..4, bit 3 only above 15), sign.
void mv_component(BoolWriter& w, const uint8_t* p, int v) {
  const int a = std::abs(v);
  if (a > 7) {
    w.put(p[0], true);
    for (int i = 0; i < 3; i++) w.put(p[9 + i], (a >> i) & 1);
    for (int i = 9; i > 3; i--) w.put(p[9 + i], (a >> i) & 1);
    if (a & 0xFFF0) w.put(p[9 + 3], (a >> 3) & 1);
  } else {
    w.put(p[0], false);
    // the §17.2 small_mvtree, 3 levels deep
    int node = 0;
    for (int depth = 2; depth >= 0; depth--) {
      const int bit = (a >> depth) & 1;
      w.put(p[2 + (node >> 1)], bit);
      node = kSmallMvTree[node + bit];
      if (node <= 0) break;
    }
  }
  if (a != 0) w.put(p[1], v < 0);
}

bool mv_diff(vp8a_mv mv, vp8a_mv best, vp8a_mv* out) {
  const int r = (int)mv.row - best.row, c = (int)mv.col - best.col;
  if (r < -1023 || r > 1023 || c < -1023 || c > 1023) return false;
  out->row = (int16_t)r;
  out->col = (int16_t)c;
  return true;
}

// fit_prob_l8 (src/encoder.rs:9128).
uint8_t fit_prob(uint32_t n_false, uint32_t n_true) {
  const uint32_t total = n_false + n_true;
  if (total == 0) return 128;
  const uint32_t raw = (uint32_t)(((uint64_t)n_false * 256) / total);
  return (uint8_t)std::min<uint32_t>(std::max<uint32_t>(raw, 1), 255);
}

// The MB's coefficient blocks in coding order: Y2 (when the MB has one),
// Y 0..15, U 16..19, V 20..23; per block its plane type, first coefficient
// and raster coefficients (MbCoeffs order y2, y[16], u[4], v[4]).
struct BlockRef {
  int slot_above, slot_left, plane, first;
  const int16_t* c;
};

int mb_blocks(const int16_t* mb, bool has_y2, BlockRef* out) {
  static const uint8_t kLeft[25] = {0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8};
  static const uint8_t kAbove[25] = {0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 4, 5, 4, 5, 6, 7, 6, 7, 8};
  int n = 0;
  if (has_y2) out[n++] = {kAbove[24], kLeft[24], 1, 0, mb};
  for (int b = 0; b < 24; b++) {
    const int plane = b < 16 ? (has_y2 ? 0 : 3) : 2;
    const int first = (b < 16 && has_y2) ? 1 : 0;
    out[n++] = {kAbove[b], kLeft[b], plane, first, mb + 16 + 16 * b};
  }
  return n;
}

// Whether the block has a nonzero coefficient it codes (raster and scan
// order hold the same set past the DC): four 64-bit ORs.
bool block_nonzero(const BlockRef& b) {
  uint64_t w[4];
  std::memcpy(w, b.c, sizeof w);
  if (b.first) w[0] &= ~(uint64_t)0xFFFF;
  return (w[0] | w[1] | w[2] | w[3]) != 0;
}

}  // namespace
}  // namespace vp8a_emit

using namespace vp8a_emit;

extern "C" vp8a_status vp8a_write_inter_frame(const vp8a_frame_header* h, const vp8a_mb_decision* decisions,
                                               const int16_t* coeffs, const int8_t* mb_segment,
                                               const uint8_t* token_prob_updates, uint8_t* out,
                                               uint64_t out_capacity, uint64_t* out_size) {
  if (!h || !decisions || !coeffs || !out_size) return VP8A_E_INVALID_ARGUMENT;
  *out_size = 0;
  if (h->width == 0 || h->width > 0x3FFF || h->height == 0 || h->height > 0x3FFF) return VP8A_E_INVALID_DIMENSIONS;
  if (h->quant.y_ac_qi > 127) return VP8A_E_QUANT_INDEX_OUT_OF_RANGE;
  if (h->loop_filter_level > 63) return VP8A_E_LOOP_FILTER_LEVEL_OUT_OF_RANGE;
  if (h->sharpness_level > 7) return VP8A_E_SHARPNESS_LEVEL_OUT_OF_RANGE;
  const int np = h->n_partitions;
  if (np != 1 && np != 2 && np != 4 && np != 8) return VP8A_E_INVALID_DCT_PARTITION_COUNT;
  if (h->copy_buffer_to_golden > 2 || h->copy_buffer_to_alternate > 2 ||
      (h->refresh_golden_frame && h->copy_buffer_to_golden) ||
      (h->refresh_alternate_frame && h->copy_buffer_to_alternate))
    return VP8A_E_INVALID_COPY_BUFFER_SELECTOR;
  for (int k = 0; k < 4; k++)
    if (std::abs((int)h->lf_ref_delta[k]) > 63 || std::abs((int)h->lf_mode_delta[k]) > 63)
      return VP8A_E_LOOP_FILTER_DELTA_OUT_OF_RANGE;
  const int8_t* qd = &h->quant.y_dc_delta;
  for (int k = 0; k < 5; k++)
    if (qd[k] < -15 || qd[k] > 15) return VP8A_E_INVALID_ARGUMENT;
  if (h->segmentation) {
    if (!mb_segment) return VP8A_E_INVALID_ARGUMENT;
    for (int k = 0; k < 4; k++)
      if (std::abs((int)h->segment_quant[k]) > 127 || std::abs((int)h->segment_lf[k]) > 63)
        return VP8A_E_INVALID_ARGUMENT;
  }
  const int cols = (int)((h->width + 15) / 16), rows = (int)((h->height + 15) / 16);
  const size_t n_mbs = (size_t)cols * rows;

  // Probabilities the tokens are coded against: the §13.5 defaults with the
  // caller's updates laid over them (merge_default_token_probs).
  Probs probs;
  std::memcpy(probs, kDefaultCoeffProbs, sizeof probs);
  if (token_prob_updates) {
    uint8_t* flat = &probs[0][0][0][0];
    for (int i = 0; i < 1056; i++)
      if (token_prob_updates[i]) flat[i] = token_prob_updates[i];
  }

  // Per MB: the wire segment, skip flag (no nonzero block among those the
  // MB codes, src/encoder.rs:8746-8769) and the per-block nonzero flags.
  std::vector<uint8_t> skip(n_mbs), seg(n_mbs, 0);
  std::vector<uint32_t> nzmask(n_mbs);  // bit b: coding-order block b has a coded nonzero
  uint32_t n_skip = 0, n_ref[4] = {0, 0, 0, 0}, seg_count[4] = {0, 0, 0, 0};
  for (size_t i = 0; i < n_mbs; i++) {
    const vp8a_mb_decision& d = decisions[i];
    if (d.ref_frame < VP8A_REF_LAST || d.ref_frame > VP8A_REF_ALTREF || d.mode > VP8A_MODE_SPLIT)
      return VP8A_E_INVALID_ARGUMENT;  // intra MBs are not produced by the device analysis
    if (d.mode == VP8A_MODE_SPLIT && d.partition > VP8A_PART_MV16) return VP8A_E_INVALID_ARGUMENT;
    BlockRef blk[25];
    const int nb = mb_blocks(coeffs + 400 * i, d.mode != VP8A_MODE_SPLIT, blk);
    uint32_t mask = 0;
    for (int b = 0; b < nb; b++) {
      if (!block_nonzero(blk[b])) continue;
      mask |= 1u << b;
      for (int k = blk[b].first; k < 16; k++)
        if (std::abs((int)blk[b].c[k]) > 2114) return VP8A_E_COEFFICIENT_OUT_OF_RANGE;
    }
    nzmask[i] = mask;
    skip[i] = mask == 0;
    n_skip += skip[i];
    n_ref[d.ref_frame]++;
    if (h->segmentation) {
      const int s = mb_segment[i] < 0 ? 0 : mb_segment[i];
      if (s > 3) return VP8A_E_INVALID_ARGUMENT;
      seg[i] = (uint8_t)s;
      seg_count[s]++;
    }
  }

  // ---- §19.2 first partition: the frame header
  BoolWriter hdr;
  uint8_t seg_probs[3] = {0, 0, 0};
  if (h->segmentation) {  // write_update_segmentation (src/encoder.rs:685)
    seg_probs[0] = fit_prob(seg_count[0] + seg_count[1], seg_count[2] + seg_count[3]);
    seg_probs[1] = fit_prob(seg_count[0], seg_count[1]);
    seg_probs[2] = fit_prob(seg_count[2], seg_count[3]);
    hdr.put(128, true);   // segmentation_enabled
    hdr.put(128, true);   // update_mb_segmentation_map
    hdr.put(128, true);   // update_segment_feature_data
    hdr.put(128, false);  // segment_feature_mode: deltas
    for (int k = 0; k < 4; k++) {
      hdr.put(128, true);
      hdr.signed_literal(h->segment_quant[k], 7);
    }
    for (int k = 0; k < 4; k++) {
      hdr.put(128, h->segment_lf_present != 0);
      if (h->segment_lf_present) hdr.signed_literal(h->segment_lf[k], 6);
    }
    for (int k = 0; k < 3; k++) {
      hdr.put(128, true);
      hdr.literal(seg_probs[k], 8);
    }
  } else {
    hdr.put(128, false);
  }
  // write_loop_filter_with_deltas (src/encoder.rs:948)
  hdr.put(128, h->filter_type != 0);
  hdr.literal(h->loop_filter_level, 6);
  hdr.literal(h->sharpness_level, 3);
  hdr.put(128, h->lf_delta_enabled != 0);
  if (h->lf_delta_enabled) {
    hdr.put(128, h->lf_delta_update != 0);
    if (h->lf_delta_update) {
      for (int k = 0; k < 8; k++) {
        const bool sent = k < 4 ? (h->lf_ref_delta_present >> k) & 1 : (h->lf_mode_delta_present >> (k - 4)) & 1;
        const int v = k < 4 ? h->lf_ref_delta[k] : h->lf_mode_delta[k - 4];
        hdr.put(128, sent);
        if (sent) hdr.signed_literal(v, 6);
      }
    }
  }
  hdr.literal(np == 1 ? 0 : (np == 2 ? 1 : (np == 4 ? 2 : 3)), 2);  // write_token_partition_count
  hdr.literal(h->quant.y_ac_qi, 7);                                 // write_quant_indices
  for (int k = 0; k < 5; k++) {
    hdr.put(128, qd[k] != 0);
    if (qd[k]) hdr.signed_literal(qd[k], 4);
  }
  // §9.7 / §9.8 refresh, sign bias, entropy persistence
  hdr.put(128, h->refresh_golden_frame != 0);
  hdr.put(128, h->refresh_alternate_frame != 0);
  if (!h->refresh_golden_frame) hdr.literal(h->copy_buffer_to_golden, 2);
  if (!h->refresh_alternate_frame) hdr.literal(h->copy_buffer_to_alternate, 2);
  hdr.put(128, false);  // sign_bias_golden
  hdr.put(128, false);  // sign_bias_alternate
  hdr.put(128, false);  // refresh_entropy_probs
  hdr.put(128, h->refresh_last != 0);
  // §13.4 token probability updates (write_token_prob_updates :1117)
  {
    const uint8_t* up = &kCoeffUpdateProbs[0][0][0][0];
    for (int i = 0; i < 1056; i++) {
      const bool upd = token_prob_updates && token_prob_updates[i];
      hdr.put(up[i], upd);
      if (upd) hdr.literal(token_prob_updates[i], 8);
    }
  }
  const uint8_t prob_skip = h->fit_skip_prob ? fit_prob((uint32_t)n_mbs - n_skip, n_skip) : 128;
  hdr.put(128, true);  // mb_no_skip_coeff
  hdr.literal(prob_skip, 8);
  const uint8_t prob_intra = h->pick_intra ? fit_prob(0, (uint32_t)n_mbs) : 255;
  const uint8_t prob_last = fit_prob(n_ref[VP8A_REF_LAST], n_ref[VP8A_REF_GOLDEN] + n_ref[VP8A_REF_ALTREF]);
  const uint8_t prob_gf = fit_prob(n_ref[VP8A_REF_GOLDEN], n_ref[VP8A_REF_ALTREF]);
  hdr.literal(prob_intra, 8);
  hdr.literal(prob_last, 8);
  hdr.literal(prob_gf, 8);
  hdr.put(128, false);  // intra_16x16_prob_update_flag
  hdr.put(128, false);  // intra_chroma_prob_update_flag
  for (int c = 0; c < 2; c++)
    for (int k = 0; k < 19; k++) hdr.put(kMvUpdateProbs[c][k], false);

  // ---- §16 / §17 macroblock modes, raster order
  std::vector<Info> above(cols);
  for (int r = 0; r < rows; r++) {
    Info left, al;
    for (int c = 0; c < cols; c++) {
      const size_t i = (size_t)r * cols + c;
      const vp8a_mb_decision& d = decisions[i];
      if (h->segmentation) {  // mb_segment_tree
        hdr.put(seg_probs[0], seg[i] >> 1);
        hdr.put(seg_probs[1 + (seg[i] >> 1)], seg[i] & 1);
      }
      hdr.put(prob_skip, skip[i] != 0);
      hdr.put(prob_intra, true);  // is_inter_mb
      hdr.put(prob_last, d.ref_frame != VP8A_REF_LAST);
      if (d.ref_frame != VP8A_REF_LAST) hdr.put(prob_gf, d.ref_frame == VP8A_REF_ALTREF);
      const Near nr = census(above[c], left, al, c, r, cols, rows);
      // mv_ref_tree: ZERO "0", NEAREST "10", NEAR "110", NEW "1110", SPLIT "1111"
      static const uint8_t kModeLen[5] = {1, 2, 3, 4, 4};
      for (int s = 0; s < kModeLen[d.mode]; s++) hdr.put(nr.p[s], s < d.mode);
      Info cur;
      cur.ref = d.ref_frame;
      cur.mv = d.mv;
      if (d.mode == VP8A_MODE_NEW) {
        vp8a_mv diff;
        if (!mv_diff(d.mv, nr.best, &diff)) return VP8A_E_INVALID_ARGUMENT;
        mv_component(hdr, kDefaultMvContexts[0], diff.row);
        mv_component(hdr, kDefaultMvContexts[1], diff.col);
      } else if (d.mode == VP8A_MODE_SPLIT) {
        const int pid = d.partition;
        // mvpartition_tree: MV16 "0", QUARTERS "10", TOP_BOTTOM "110", LEFT_RIGHT "111"
        const int depth = pid == VP8A_PART_MV16 ? 0 : (pid == VP8A_PART_QUARTERS ? 1 : 2);
        for (int s = 0; s < depth; s++) hdr.put(kPartitionProbs[s], true);
        if (depth < 2) hdr.put(kPartitionProbs[depth], false);
        else hdr.put(kPartitionProbs[2], pid == VP8A_PART_LEFT_RIGHT);
        vp8a_mv running[16] = {};
        for (int g = 0; g < kPartitionGroups[pid]; g++) {
          int anchor = 0;
          while (kPartitionMap[pid][anchor] != g) anchor++;
          const int ctx = submv_context(left_block(running, left, anchor), above_block(running, above[c], anchor));
          const int m = d.submv_modes[g];
          if (m > VP8A_SUBMV_NEW) return VP8A_E_INVALID_ARGUMENT;
          // sub_mv_ref_tree: LEFT "0", ABOVE "10", ZERO "110", NEW "111"
          const uint8_t* p = kSubmvProbs[ctx];
          hdr.put(p[0], m != VP8A_SUBMV_LEFT);
          if (m != VP8A_SUBMV_LEFT) hdr.put(p[1], m != VP8A_SUBMV_ABOVE);
          if (m > VP8A_SUBMV_ABOVE) hdr.put(p[2], m == VP8A_SUBMV_NEW);
          if (m == VP8A_SUBMV_NEW) {
            vp8a_mv diff;
            if (!mv_diff(d.split_mvs[anchor], nr.best, &diff)) return VP8A_E_INVALID_ARGUMENT;
            mv_component(hdr, kDefaultMvContexts[0], diff.row);
            mv_component(hdr, kDefaultMvContexts[1], diff.col);
          }
          for (int b = 0; b < 16; b++)
            if (kPartitionMap[pid][b] == g) running[b] = d.split_mvs[b];
        }
        cur.split = true;
        cur.mv = d.split_mvs[15];
        std::memcpy(cur.smv, d.split_mvs, sizeof cur.smv);
      }
      al = above[c];
      left = cur;
      above[c] = cur;
    }
  }
  const std::vector<uint8_t> first = hdr.finish();
  if (first.size() > 0x7FFFF) return VP8A_E_FIRST_PARTITION_TOO_LARGE;

  // ---- §13 residual tokens. The §13.3 contexts: one above record per
  // column for the whole frame, one left record per row; a skipped MB
  // clears its slots (Y2 only when it has a Y2, clear_skip_ctx
  // src/encoder.rs:7369). The contexts of every MB follow from the
  // nonzero flags alone, so they are resolved first in raster order and
  // each partition then codes its rows on its own thread.
  std::vector<uint8_t> ctx_in(n_mbs * 25 * 2);  // per MB and coding-order block: above, left
  {
    std::vector<uint8_t> above_nz((size_t)cols * 9, 0);
    for (int r = 0; r < rows; r++) {
      uint8_t left_nz[9] = {};
      for (int c = 0; c < cols; c++) {
        const size_t i = (size_t)r * cols + c;
        const bool has_y2 = decisions[i].mode != VP8A_MODE_SPLIT;
        uint8_t* a = &above_nz[(size_t)c * 9];
        BlockRef blk[25];
        const int nb = mb_blocks(coeffs + 400 * i, has_y2, blk);
        if (skip[i]) {
          for (int s = 0; s < 8; s++) a[s] = left_nz[s] = 0;
          if (has_y2) a[8] = left_nz[8] = 0;
          continue;
        }
        for (int b = 0; b < nb; b++) {
          ctx_in[(i * 25 + b) * 2] = a[blk[b].slot_above];
          ctx_in[(i * 25 + b) * 2 + 1] = left_nz[blk[b].slot_left];
          const uint8_t nz = (nzmask[i] >> b) & 1;
          a[blk[b].slot_above] = nz;
          left_nz[blk[b].slot_left] = nz;
        }
      }
    }
  }
  std::vector<std::vector<uint8_t>> parts(np);
  auto code_partition = [&](int p) {
    BoolWriter w;
    for (int r = p; r < rows; r += np)
      for (int c = 0; c < cols; c++) {
        const size_t i = (size_t)r * cols + c;
        if (skip[i]) continue;
        BlockRef blk[25];
        const int nb = mb_blocks(coeffs + 400 * i, decisions[i].mode != VP8A_MODE_SPLIT, blk);
        for (int b = 0; b < nb; b++) {
          const int ctx = ctx_in[(i * 25 + b) * 2] + ctx_in[(i * 25 + b) * 2 + 1];
          if ((nzmask[i] >> b) & 1)
            code_block(w, probs, blk[b].plane, blk[b].first, ctx, blk[b].c);
          else  // an empty block is its EOB alone
            w.put(probs[blk[b].plane][kBands[blk[b].first]][ctx][0], false);
        }
      }
    parts[p] = w.finish();
  };
  if (np == 1 || n_mbs < 4096) {
    for (int p = 0; p < np; p++) code_partition(p);
  } else {
    std::vector<std::thread> th;
    for (int p = 0; p < np; p++) th.emplace_back(code_partition, p);
    for (auto& t : th) t.join();
  }

  // ---- §9.1 frame tag (inter, version 0, shown), first partition, the
  // §9.5 size table (3-byte little-endian sizes of all but the last
  // partition) and the partitions.
  uint64_t total = 3 + first.size() + 3 * (uint64_t)(np - 1);
  for (const auto& p : parts) total += p.size();
  *out_size = total;
  if (!out || out_capacity < total) return VP8A_E_INVALID_ARGUMENT;
  const uint32_t tag = 1u | (0u << 1) | (1u << 4) | ((uint32_t)first.size() << 5);
  uint8_t* o = out;
  *o++ = (uint8_t)tag;
  *o++ = (uint8_t)(tag >> 8);
  *o++ = (uint8_t)(tag >> 16);
  std::memcpy(o, first.data(), first.size());
  o += first.size();
  for (int p = 0; p + 1 < np; p++) {
    const size_t s = parts[p].size();
    *o++ = (uint8_t)s;
    *o++ = (uint8_t)(s >> 8);
    *o++ = (uint8_t)(s >> 16);
  }
  for (const auto& p : parts) {
    if (!p.empty()) std::memcpy(o, p.data(), p.size());
    o += p.size();
  }
  return VP8A_OK;
}
