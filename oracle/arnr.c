/*
 * arnr.c — oracle restatement of the ARNR temporal filter.
 *
 * TEST INFRASTRUCTURE ONLY (see vp8a_oracle.h). Follows src/arnr.rs:37-675:
 * refine_search (:264-300) over the edge-clamped block SAD
 * (block_sad_generic :237-258; the early exit never changes the winner and
 * is omitted), weight_table (:307-323), accumulate_luma_block (:337-388),
 * accumulate_chroma_block (:402-459, including its clamped overhang
 * double-accumulation), build_arnr_altref_threaded (:488-650) and
 * resolve_plane (:670-675).
 */
#include <stdlib.h>
#include <string.h>

#include "vp8a_oracle.h"

#define W_MAX 16u
#define BLOCK_SAD_PER_PIXEL_CUTOFF 12u

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* pel (src/arnr.rs:149-153). */
static inline uint8_t pel(const uint8_t* p, size_t stride, int w, int h, int x, int y) {
  return p[(size_t)clampi(y, 0, h - 1) * stride + (size_t)clampi(x, 0, w - 1)];
}

static uint32_t block_sad(const vp8a_i420* src, const vp8a_i420* refp, int bx, int by, int bw,
                          int bh, int mvx, int mvy) {
  int w = (int)src->width, h = (int)src->height;
  uint32_t sad = 0;
  for (int r = 0; r < bh; r++) {
    int sy = by + r;
    for (int c = 0; c < bw; c++) {
      int s = src->y[(size_t)sy * src->y_stride + bx + c];
      int rp = pel(refp->y, refp->y_stride, w, h, bx + c + mvx, sy + mvy);
      int d = s - rp;
      sad += (uint32_t)(d < 0 ? -d : d);
    }
  }
  return sad;
}

void vo_arnr_refine_search(const vp8a_i420* src, const vp8a_i420* refp, uint32_t bx,
                           uint32_t by, uint32_t bw, uint32_t bh, int32_t* mvx, int32_t* mvy,
                           uint32_t* sad_out) {
  int bestx = 0, besty = 0;
  uint32_t best_sad = block_sad(src, refp, bx, by, bw, bh, 0, 0);
  for (int step = 8; step >= 1; step /= 2) {
    int cx = bestx, cy = besty;
    const int d[8][2] = {{-step, -step}, {0, -step}, {step, -step}, {-step, 0},
                         {step, 0},      {-step, step}, {0, step},  {step, step}};
    for (int k = 0; k < 8; k++) {
      int x = cx + d[k][0], y = cy + d[k][1];
      if (abs(x) > 15 || abs(y) > 15) continue;
      uint32_t s = block_sad(src, refp, bx, by, bw, bh, x, y);
      if (s < best_sad) {
        best_sad = s;
        bestx = x;
        besty = y;
      }
    }
  }
  *mvx = bestx;
  *mvy = besty;
  *sad_out = best_sad;
}

typedef struct {
  const vp8a_i420* frames;
  uint32_t center, brows, bcols;
  int32_t* mv; /* 3 per (frame, block): mvx, mvy, sad */
} arnr_search_job;

static void arnr_search_task(void* arg, uint32_t unit) {
  arnr_search_job* j = (arnr_search_job*)arg;
  uint32_t fi = unit / j->brows, brow = unit % j->brows;
  if (fi == j->center) return;
  const vp8a_i420* ctr = &j->frames[j->center];
  uint32_t w = ctr->width, h = ctr->height;
  uint32_t by = brow * 16, bh = (h - by) < 16 ? (h - by) : 16;
  for (uint32_t bcol = 0; bcol < j->bcols; bcol++) {
    uint32_t bx = bcol * 16, bw = (w - bx) < 16 ? (w - bx) : 16;
    int32_t* slot = &j->mv[3 * ((size_t)(fi * j->brows + brow) * j->bcols + bcol)];
    uint32_t sad;
    vo_arnr_refine_search(ctr, &j->frames[fi], bx, by, bw, bh, &slot[0], &slot[1], &sad);
    slot[2] = (int32_t)sad;
  }
}

static void accumulate_plane_block(const uint8_t* ctr, size_t ctr_stride, const uint8_t* f,
                                   size_t f_stride, int pw, int ph, int bx, int by, int bw,
                                   int bh, int mvx, int mvy, const uint32_t* wt, uint32_t* acc,
                                   uint32_t* wsum, int clamp_out) {
  for (int r = 0; r < bh; r++) {
    int yy = by + r;
    if (clamp_out && yy > ph - 1) yy = ph - 1;
    for (int c = 0; c < bw; c++) {
      int xx = bx + c;
      if (clamp_out && xx > pw - 1) xx = pw - 1;
      int ctr_px = ctr[(size_t)yy * ctr_stride + xx];
      int ref_px = pel(f, f_stride, pw, ph, xx + mvx, yy + mvy);
      int d = ref_px - ctr_px;
      uint32_t w = wt[d < 0 ? -d : d];
      acc[(size_t)yy * pw + xx] += w * (uint32_t)ref_px;
      wsum[(size_t)yy * pw + xx] += w;
    }
  }
}

int vo_build_arnr_altref(const vp8a_i420* frames, uint32_t n, uint32_t center,
                         uint32_t strength, uint8_t* y_out, uint8_t* u_out, uint8_t* v_out,
                         uint32_t threads) {
  if (!frames || n == 0 || center >= n || !y_out || !u_out || !v_out)
    return VP8A_E_INVALID_ARGUMENT;
  const vp8a_i420* ctr = &frames[center];
  if (ctr->width == 0 || ctr->height == 0 || ctr->width > 0x3FFF || ctr->height > 0x3FFF)
    return VP8A_E_INVALID_DIMENSIONS;
  for (uint32_t i = 0; i < n; i++)
    if (frames[i].width != ctr->width || frames[i].height != ctr->height)
      return VP8A_E_REFERENCE_DIMENSIONS_MISMATCH;
  int w = (int)ctr->width, h = (int)ctr->height, cw = (w + 1) / 2, ch = (h + 1) / 2;
  /* Centre copy (src/arnr.rs:520-526). */
  for (int r = 0; r < h; r++) memcpy(y_out + (size_t)r * w, ctr->y + (size_t)r * ctr->y_stride, w);
  for (int r = 0; r < ch; r++) {
    memcpy(u_out + (size_t)r * cw, ctr->u + (size_t)r * ctr->uv_stride, cw);
    memcpy(v_out + (size_t)r * cw, ctr->v + (size_t)r * ctr->uv_stride, cw);
  }
  if (strength == 0 || n < 2) return VP8A_OK;
  if (strength > 6) strength = 6;
  uint32_t s_scale = 8u << strength;
  uint32_t wt[256];
  for (int d = 0; d < 256; d++) wt[d] = (W_MAX * s_scale) / (s_scale + (uint32_t)(d * d));

  size_t ny = (size_t)w * h, nc = (size_t)cw * ch;
  uint32_t* acc_y = (uint32_t*)malloc(ny * 4);
  uint32_t* ws_y = (uint32_t*)malloc(ny * 4);
  uint32_t* acc_u = (uint32_t*)malloc(nc * 4);
  uint32_t* ws_u = (uint32_t*)malloc(nc * 4);
  uint32_t* acc_v = (uint32_t*)malloc(nc * 4);
  uint32_t* ws_v = (uint32_t*)malloc(nc * 4);
  uint32_t bcols = (uint32_t)(w + 15) / 16, brows = (uint32_t)(h + 15) / 16;
  int32_t* mv = (int32_t*)calloc((size_t)3 * n * brows * bcols, sizeof(int32_t));
  if (!acc_y || !ws_y || !acc_u || !ws_u || !acc_v || !ws_v || !mv) {
    free(acc_y); free(ws_y); free(acc_u); free(ws_u); free(acc_v); free(ws_v); free(mv);
    return VP8A_E_OUT_OF_MEMORY;
  }
  /* accumulate_center (src/arnr.rs:662). */
  for (size_t i = 0; i < ny; i++) { acc_y[i] = W_MAX * y_out[i]; ws_y[i] = W_MAX; }
  for (size_t i = 0; i < nc; i++) {
    acc_u[i] = W_MAX * u_out[i]; ws_u[i] = W_MAX;
    acc_v[i] = W_MAX * v_out[i]; ws_v[i] = W_MAX;
  }
  arnr_search_job sj = {frames, center, brows, bcols, mv};
  vo_parallel_for(n * brows, threads, arnr_search_task, &sj);

  for (uint32_t fi = 0; fi < n; fi++) {
    if (fi == center) continue;
    const vp8a_i420* f = &frames[fi];
    for (int by = 0; by < h; by += 16) {
      int bh = (h - by) < 16 ? (h - by) : 16;
      for (int bx = 0; bx < w; bx += 16) {
        int bw = (w - bx) < 16 ? (w - bx) : 16;
        const int32_t* a = &mv[3 * ((size_t)(fi * brows + by / 16) * bcols + bx / 16)];
        int mvx = a[0], mvy = a[1];
        uint32_t sad = (uint32_t)a[2];
        if (sad / (uint32_t)(bw * bh) > BLOCK_SAD_PER_PIXEL_CUTOFF) continue;
        accumulate_plane_block(y_out, (size_t)w, f->y, f->y_stride, w, h, bx, by, bw, bh, mvx,
                               mvy, wt, acc_y, ws_y, 0);
        int cmvx = mvx / 2, cmvy = mvy / 2; /* toward zero (src/arnr.rs:622) */
        int cbx = bx / 2, cby = by / 2, cbw = (bw + 1) / 2, cbh = (bh + 1) / 2;
        accumulate_plane_block(u_out, (size_t)cw, f->u, f->uv_stride, cw, ch, cbx, cby, cbw, cbh,
                               cmvx, cmvy, wt, acc_u, ws_u, 1);
        accumulate_plane_block(v_out, (size_t)cw, f->v, f->uv_stride, cw, ch, cbx, cby, cbw, cbh,
                               cmvx, cmvy, wt, acc_v, ws_v, 1);
      }
    }
  }
  for (size_t i = 0; i < ny; i++) y_out[i] = (uint8_t)((acc_y[i] + ws_y[i] / 2) / ws_y[i]);
  for (size_t i = 0; i < nc; i++) {
    u_out[i] = (uint8_t)((acc_u[i] + ws_u[i] / 2) / ws_u[i]);
    v_out[i] = (uint8_t)((acc_v[i] + ws_v[i] / 2) / ws_v[i]);
  }
  free(acc_y); free(ws_y); free(acc_u); free(ws_u); free(acc_v); free(ws_v); free(mv);
  return VP8A_OK;
}
