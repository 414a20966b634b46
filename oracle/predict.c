/*
 * predict.c — oracle restatement of the §18 inter prediction (motion
 * compensation) the encoder builds after its mode decision.
 *
 * TEST INFRASTRUCTURE ONLY (see vp8a_oracle.h). Follows src/motion_comp.rs:
 *   :187-272   stored_luma_mv, avg, chroma_mv, apply_full_pixel
 *   :294-334   SIXTAP_FILTERS, BILINEAR_FILTERS; :370 filter_set_for_version
 *   :396-402   interp
 *   :700-767   sixtap_2d_scalar (4x4 block, 9x9 halo)
 *   :837-880   fetch_luma_mb_halo (21x21); :1018-1057 sixtap_mb_luma_scalar
 *   :1153-1216 fetch_chroma_mb_halo (13x13); :1311-1348 sixtap_mb_chroma_scalar
 *   :1442-1632 fetch_block_whole_pixel, fetch_luma/chroma_mb_whole_pixel
 *   :1633-1718 fetch_block_halo, filter_block_4x4
 *   :1986-2096 predict_inter_mb
 *   :2162-2213 chroma_idx_for_luma_subblock, split_chroma_mvs
 *   :2228-2330 predict_split_mv
 * The whole-MB path is restated in the reference's MB-scale form (one
 * 21x21 luma halo and one 13x13 halo per chroma plane, or the whole-pixel
 * MB copies) and the SPLITMV path in its per-4x4-block form, so the two
 * are independent listings of the same §18.3 arithmetic. The reference's
 * identity elision (sixtap_identity_elide, :960-1016) is byte-exact with
 * the plain two-pass listing by its own tests and is not restated.
 */
#include <string.h>

#include "vp8a_oracle.h"

/* SIXTAP_FILTERS / BILINEAR_FILTERS (src/motion_comp.rs:294-334), RFC 6386
 * §18.3 filters[8][6] and BilinearFilters[8][6]. */
static const int TAPS[2][8][6] = {
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

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int64_t clampl(int64_t v, int64_t lo, int64_t hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

/* stored_luma_mv (src/motion_comp.rs:187): i16 wrapping doubling. */
static inline vp8a_mv stored_luma(vp8a_mv mv) {
  vp8a_mv o;
  o.row = (int16_t)(uint16_t)((uint16_t)mv.row * 2u);
  o.col = (int16_t)(uint16_t)((uint16_t)mv.col * 2u);
  return o;
}

/* avg (src/motion_comp.rs:209): sign-aware divide by 8 with rounding. */
static inline int32_t avg_sum(int32_t s) { return s >= 0 ? (s + 4) >> 3 : -((-s + 4) >> 3); }

/* chroma_mv (src/motion_comp.rs:232): avg of the one vector taken four times. */
vp8a_mv vo_chroma_mv(vp8a_mv luma_eighth) {
  vp8a_mv o;
  o.row = (int16_t)avg_sum(4 * (int32_t)luma_eighth.row);
  o.col = (int16_t)avg_sum(4 * (int32_t)luma_eighth.col);
  return o;
}

/* apply_full_pixel (src/motion_comp.rs:256): x &= ~7, y &= ~7. */
static inline vp8a_mv full_pixel_mv(vp8a_mv mv) {
  vp8a_mv o;
  o.row = (int16_t)(mv.row & ~7);
  o.col = (int16_t)(mv.col & ~7);
  return o;
}

/* interp (src/motion_comp.rs:396-402). */
static inline uint8_t interp(const int* f, const uint8_t* s, size_t step) {
  int a = 0;
  for (int i = 0; i < 6; i++) a += (int)s[i * step] * f[i];
  return (uint8_t)clampi((a + 64) >> 7, 0, 255);
}

/* An edge-clamped n x n fetch whose (0,0) is source (x0, y0): the shared
 * body of fetch_block_halo / fetch_*_mb_halo / fetch_*_whole_pixel
 * (src/motion_comp.rs:1153-1216, :1442-1671). Their in-bounds fast paths
 * are plain row copies of the same positions. */
static void fetch_clamped(const uint8_t* plane, size_t stride, size_t w, size_t h, int64_t x0,
                          int64_t y0, int n, uint8_t* out) {
  for (int r = 0; r < n; r++) {
    int64_t sy = clampl(y0 + r, 0, (int64_t)h - 1);
    for (int c = 0; c < n; c++) {
      int64_t sx = clampl(x0 + c, 0, (int64_t)w - 1);
      out[r * n + c] = plane[(size_t)sy * stride + (size_t)sx];
    }
  }
}

/* sixtap_2d_scalar (src/motion_comp.rs:700-767) generalised over the block
 * width `ow` (4: sixtap_2d, 8: sixtap_mb_chroma_scalar :1311, 16:
 * sixtap_mb_luma_scalar :1018): horizontal pass over all ow+5 halo rows
 * into an 8-bit intermediate, then the vertical pass. */
static void sixtap_block(const uint8_t* halo, int ow, int mx, int my, const int (*filters)[6],
                         uint8_t* out) {
  const int hw = ow + 5;
  uint8_t temp[21 * 16];
  for (int r = 0; r < hw; r++)
    for (int c = 0; c < ow; c++) temp[r * ow + c] = interp(filters[mx], halo + r * hw + c, 1);
  for (int r = 0; r < ow; r++)
    for (int c = 0; c < ow; c++) out[r * ow + c] = interp(filters[my], temp + r * ow + c, ow);
}

void vo_sixtap_2d(const uint8_t* halo81, int mx, int my, int filter_set, uint8_t* out16) {
  sixtap_block(halo81, 4, mx & 7, my & 7, TAPS[filter_set ? 1 : 0], out16);
}

/* One whole-MB-vector plane of predict_inter_mb (src/motion_comp.rs:2034-2094):
 * the n x n block at (bx, by) under the eighth-pel vector `mv`. */
static void predict_plane_mb(const uint8_t* plane, size_t stride, size_t w, size_t h, size_t bx,
                             size_t by, int n, vp8a_mv mv, const int (*filters)[6], uint8_t* out) {
  const int mx = mv.col & 7, my = mv.row & 7;
  const int64_t ox = (int64_t)bx + (mv.col >> 3), oy = (int64_t)by + (mv.row >> 3);
  if (mx == 0 && my == 0) {
    fetch_clamped(plane, stride, w, h, ox, oy, n, out);
  } else {
    uint8_t halo[21 * 21];
    fetch_clamped(plane, stride, w, h, ox - 2, oy - 2, n + 5, halo);
    sixtap_block(halo, n, mx, my, filters, out);
  }
}

/* filter_block_4x4 (src/motion_comp.rs:1693-1718). */
static void filter_block_4x4(const uint8_t* plane, size_t stride, size_t w, size_t h, size_t bx,
                             size_t by, vp8a_mv mv, const int (*filters)[6], uint8_t* out16) {
  predict_plane_mb(plane, stride, w, h, bx, by, 4, mv, filters, out16);
}

/* predict_inter_mb (src/motion_comp.rs:1986-2096). out: ReconstructedMb
 * layout, y[256] then u[64] then v[64]. */
void vo_predict_inter_mb(const vp8a_planes* ref, uint32_t mb_col, uint32_t mb_row, vp8a_mv luma_mv,
                         int full_pixel, int filter_set, uint8_t* out) {
  const int (*filters)[6] = TAPS[filter_set ? 1 : 0];
  vp8a_mv ymv = stored_luma(luma_mv);
  vp8a_mv uvmv = vo_chroma_mv(ymv);
  if (full_pixel) {
    ymv = full_pixel_mv(ymv);
    uvmv = full_pixel_mv(uvmv);
  }
  const size_t lw = (size_t)ref->mb_cols * 16, lh = (size_t)ref->mb_rows * 16;
  const size_t cw = (size_t)ref->mb_cols * 8, ch = (size_t)ref->mb_rows * 8;
  predict_plane_mb(ref->y, ref->y_stride, lw, lh, (size_t)mb_col * 16, (size_t)mb_row * 16, 16, ymv,
                   filters, out);
  predict_plane_mb(ref->u, ref->uv_stride, cw, ch, (size_t)mb_col * 8, (size_t)mb_row * 8, 8, uvmv,
                   filters, out + 256);
  predict_plane_mb(ref->v, ref->uv_stride, cw, ch, (size_t)mb_col * 8, (size_t)mb_row * 8, 8, uvmv,
                   filters, out + 320);
}

/* chroma_idx_for_luma_subblock + split_chroma_mvs (src/motion_comp.rs:2162-2213):
 * the doubled luma components are summed in i32 (no i16 wrap) per chroma
 * sub-block before avg. */
void vo_split_chroma_mvs(const vp8a_mv* split16, vp8a_mv* out4) {
  int32_t sr[4] = {0, 0, 0, 0}, sc[4] = {0, 0, 0, 0};
  for (int b = 0; b < 16; b++) {
    const int c = ((b >> 1) & 1) + ((b >> 2) & 2);
    sr[c] = (int32_t)((uint32_t)sr[c] + (uint32_t)((int32_t)split16[b].row * 2));
    sc[c] = (int32_t)((uint32_t)sc[c] + (uint32_t)((int32_t)split16[b].col * 2));
  }
  for (int c = 0; c < 4; c++) {
    out4[c].row = (int16_t)avg_sum(sr[c]);
    out4[c].col = (int16_t)avg_sum(sc[c]);
  }
}

/* predict_split_mv (src/motion_comp.rs:2228-2330): every luma 4x4 under its
 * own doubled vector, every chroma 4x4 under its split_chroma_mvs average. */
void vo_predict_split_mv(const vp8a_planes* ref, uint32_t mb_col, uint32_t mb_row,
                         const vp8a_mv* split16, int full_pixel, int filter_set, uint8_t* out) {
  const int (*filters)[6] = TAPS[filter_set ? 1 : 0];
  const size_t lw = (size_t)ref->mb_cols * 16, lh = (size_t)ref->mb_rows * 16;
  const size_t cw = (size_t)ref->mb_cols * 8, ch = (size_t)ref->mb_rows * 8;
  uint8_t blk[16];
  for (int sb = 0; sb < 4; sb++)
    for (int sc = 0; sc < 4; sc++) {
      vp8a_mv ymv = stored_luma(split16[sb * 4 + sc]);
      if (full_pixel) ymv = full_pixel_mv(ymv);
      filter_block_4x4(ref->y, ref->y_stride, lw, lh, (size_t)mb_col * 16 + sc * 4,
                       (size_t)mb_row * 16 + sb * 4, ymv, filters, blk);
      for (int r = 0; r < 4; r++) memcpy(out + (sb * 4 + r) * 16 + sc * 4, blk + r * 4, 4);
    }
  vp8a_mv cmv[4];
  vo_split_chroma_mvs(split16, cmv);
  for (int sb = 0; sb < 2; sb++)
    for (int sc = 0; sc < 2; sc++) {
      vp8a_mv uvmv = cmv[sb * 2 + sc];
      if (full_pixel) uvmv = full_pixel_mv(uvmv);
      const size_t bx = (size_t)mb_col * 8 + sc * 4, by = (size_t)mb_row * 8 + sb * 4;
      filter_block_4x4(ref->u, ref->uv_stride, cw, ch, bx, by, uvmv, filters, blk);
      for (int r = 0; r < 4; r++) memcpy(out + 256 + (sb * 4 + r) * 8 + sc * 4, blk + r * 4, 4);
      filter_block_4x4(ref->v, ref->uv_stride, cw, ch, bx, by, uvmv, filters, blk);
      for (int r = 0; r < 4; r++) memcpy(out + 320 + (sb * 4 + r) * 8 + sc * 4, blk + r * 4, 4);
    }
}

/* The prediction pick_mb_for_ref builds for the chosen (mode, mv) of the
 * winning reference (src/encoder.rs:8704-8735): predict_split_mv for SPLIT
 * decisions, predict_inter_mb otherwise, written into the MB-padded output
 * planes. MBs whose reference is VP8A_REF_INTRA or not among ref_ids are
 * left untouched; returns the number of such MBs. */
int vo_predict_inter_frame(const vp8a_planes* refs, const uint8_t* ref_ids, uint32_t n_refs,
                           const vp8a_mb_decision* dec, int full_pixel, int filter_set,
                           vp8a_planes* out) {
  int skipped = 0;
  uint8_t mb[384];
  for (uint32_t row = 0; row < out->mb_rows; row++)
    for (uint32_t col = 0; col < out->mb_cols; col++) {
      const vp8a_mb_decision* d = &dec[(size_t)row * out->mb_cols + col];
      const vp8a_planes* ref = NULL;
      for (uint32_t k = 0; k < n_refs; k++)
        if (d->ref_frame != VP8A_REF_INTRA && ref_ids[k] == d->ref_frame) ref = &refs[k];
      if (!ref) {
        skipped++;
        continue;
      }
      if (d->mode == VP8A_MODE_SPLIT)
        vo_predict_split_mv(ref, col, row, d->split_mvs, full_pixel, filter_set, mb);
      else
        vo_predict_inter_mb(ref, col, row, d->mv, full_pixel, filter_set, mb);
      for (int r = 0; r < 16; r++)
        memcpy(out->y + ((size_t)row * 16 + r) * out->y_stride + (size_t)col * 16, mb + r * 16, 16);
      for (int r = 0; r < 8; r++) {
        memcpy(out->u + ((size_t)row * 8 + r) * out->uv_stride + (size_t)col * 8, mb + 256 + r * 8, 8);
        memcpy(out->v + ((size_t)row * 8 + r) * out->uv_stride + (size_t)col * 8, mb + 320 + r * 8, 8);
      }
    }
  return skipped;
}

/* Batched forms matching the product ABI: item i is the MB at
 * (mb_xy[2i], mb_xy[2i+1]); out gets 384 bytes per item. */
void vo_predict_inter_mb_batch(const vp8a_planes* ref, const uint32_t* mb_xy, const vp8a_mv* mvs,
                               uint32_t n, int full_pixel, int filter_set, uint8_t* out) {
  for (uint32_t i = 0; i < n; i++)
    vo_predict_inter_mb(ref, mb_xy[2 * i], mb_xy[2 * i + 1], mvs[i], full_pixel, filter_set,
                        out + (size_t)i * 384);
}

void vo_predict_split_mv_batch(const vp8a_planes* ref, const uint32_t* mb_xy, const vp8a_mv* mvs16,
                               uint32_t n, int full_pixel, int filter_set, uint8_t* out) {
  for (uint32_t i = 0; i < n; i++)
    vo_predict_split_mv(ref, mb_xy[2 * i], mb_xy[2 * i + 1], mvs16 + (size_t)i * 16, full_pixel,
                        filter_set, out + (size_t)i * 384);
}
