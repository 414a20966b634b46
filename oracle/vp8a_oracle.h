/*
 * vp8a_oracle.h — CPU restatement of the oxideav-vp8 encoder-analysis path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker the CUDA path is
 * compared against (tests/, __graft_entry__.smoke() and the cpu_baseline leg
 * of bench.py). It is never linked into, loaded by or called from the
 * product library (libvp8a.so).
 *
 * Each function restates one reference function of the Rust crate
 * oxideav-vp8 0.2.9 (cited file:line) as a plain scalar listing, in the same
 * evaluation order, so that its integer results — and, for the f64 RD costs,
 * its IEEE results (built with -ffp-contract=off) — are those of the
 * reference. The Rust toolchain is absent here, so the reference cannot be
 * run; the restatement is pinned instead against the reference's own
 * known-answer unit tests (ported under tests/test_oracle_*.py).
 *
 * Types are shared with the product ABI (include/vp8a.h): plain structs.
 */
#ifndef VP8A_ORACLE_H
#define VP8A_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/vp8a.h"

#ifdef __cplusplus
extern "C" {
#endif

/* §16.3 per-MB census record (MbInfo, src/near_mv.rs:127). */
typedef vp8a_mb_info vo_mb_info;

/* ---- motion search primitives (src/motion_search.rs, src/motion_comp.rs) */
uint32_t vo_block_sad_16x16(const uint8_t* src, const uint8_t* pred);
void vo_fetch_luma_mb_whole_pixel(const uint8_t* plane, size_t stride, size_t w, size_t h,
                                  size_t mb_x, size_t mb_y, vp8a_mv mv_eighth, uint8_t* out256);
void vo_fetch_luma_mb_halo(const uint8_t* plane, size_t stride, size_t w, size_t h,
                           size_t mb_x, size_t mb_y, vp8a_mv mv_eighth, uint8_t* out441);
void vo_sixtap_mb_luma(const uint8_t* halo441, int mx, int my, uint8_t* out256);
uint32_t vo_mb_luma_sad_at_whole_mv(const vp8a_luma_ref* r, size_t mb_col, size_t mb_row,
                                    const uint8_t* src_y, vp8a_mv mv);
uint32_t vo_mb_luma_sad_at_mv(const vp8a_luma_ref* r, size_t mb_col, size_t mb_row,
                              const uint8_t* src_y, vp8a_mv mv);
vp8a_search_result vo_small_diamond_search_luma(const vp8a_luma_ref* r, size_t mb_col,
                                                size_t mb_row, const uint8_t* src_y,
                                                vp8a_mv center, uint32_t max_iters);
vp8a_search_result vo_half_pixel_refine_luma(const vp8a_luma_ref* r, size_t mb_col,
                                             size_t mb_row, const uint8_t* src_y,
                                             vp8a_mv center);
vp8a_search_result vo_quarter_pixel_refine_luma(const vp8a_luma_ref* r, size_t mb_col,
                                                size_t mb_row, const uint8_t* src_y,
                                                vp8a_mv center);

/* Batched forms with the product ABI's argument layout. */
void vo_mb_luma_sad_at_mv_batch(const vp8a_luma_ref* r, const uint8_t* src_mbs,
                                const uint32_t* mb_xy, const vp8a_mv* mvs, uint32_t n,
                                uint32_t* out);
void vo_small_diamond_batch(const vp8a_luma_ref* r, const uint8_t* src_mbs,
                            const uint32_t* mb_xy, const vp8a_mv* centers, uint32_t max_iters,
                            uint32_t n, vp8a_search_result* out);
void vo_half_refine_batch(const vp8a_luma_ref* r, const uint8_t* src_mbs, const uint32_t* mb_xy,
                          const vp8a_mv* centers, uint32_t n, vp8a_search_result* out);
void vo_quarter_refine_batch(const vp8a_luma_ref* r, const uint8_t* src_mbs,
                             const uint32_t* mb_xy, const vp8a_mv* centers, uint32_t n,
                             vp8a_search_result* out);
void vo_motion_descent_batch(const vp8a_luma_ref* r, const uint8_t* src_mbs,
                             const uint32_t* mb_xy, const vp8a_mv* centers, uint32_t max_iters,
                             uint32_t n, vp8a_search_result* whole, vp8a_search_result* half,
                             vp8a_search_result* quarter, uint32_t threads);

/* ---- census, bit costs (src/near_mv.rs, src/motion_vector.rs, src/encoder.rs) */
double vo_bool_bits(uint8_t prob, int value);
double vo_mv_component_bits(const uint8_t* ctx19, int32_t value);
void vo_find_near_mvs(const vo_mb_info* above, const vo_mb_info* left,
                      const vo_mb_info* aboveleft, uint8_t current_ref, vp8a_mv mvs_out[3],
                      int32_t cnt_out[4]);
void vo_default_mv_contexts(vp8a_mv_contexts* out);
void vo_mv_ref_probs(const int32_t cnt[4], uint8_t out[4]);
vp8a_mv vo_clamp_mv_rect(vp8a_mv mv, int mb_col, int mb_row, int mb_cols, int mb_rows);
double vo_rd_lambda(uint32_t y_ac_qi);

/* ---- exhaustive analysis (src/encoder/inter.rs, src/encoder.rs) */
/* extract_mb (src/encoder.rs:5549): edge-replicated 16x16 source luma. */
void vo_extract_mb_luma(const vp8a_i420* f, size_t mb_row, size_t mb_col, uint8_t* out256);
int vo_analyse_inter_frame(const vp8a_i420* frame, const vp8a_planes* refs,
                           const uint8_t* ref_ids, uint32_t n_refs,
                           const vp8a_mv_contexts* mv_contexts, double lambda,
                           vp8a_mb_decision* decisions, vp8a_ref_search* trace,
                           uint32_t threads);
/* vo_analyse_inter_frame with `proposals` (n_refs vectors per MB, raster
 * order) as second NEWMV candidates. */
int vo_analyse_inter_frame_proposals(const vp8a_i420* frame, const vp8a_planes* refs,
                                     const uint8_t* ref_ids, uint32_t n_refs,
                                     const vp8a_mv_contexts* mv_contexts, double lambda,
                                     const vp8a_mv* proposals, vp8a_mb_decision* decisions,
                                     vp8a_ref_search* trace, uint32_t threads);

/* The RD-effort inter search (decide_mb_rd's search part,
 * src/encoder/inter_search.rs:198-552, :846-1060) for every MB given its
 * census neighbours (3 records per MB: above, left, above-left). */
int vo_rd_inter_search(const vp8a_i420* frame, const vp8a_planes* refs, const uint8_t* ref_ids,
                       uint32_t n_refs, const vp8a_mv_contexts* mv_contexts, double lambda,
                       uint32_t y1_ac, uint32_t effort, const vp8a_mb_info* neighbours,
                       vp8a_rd_inter* out, uint32_t threads);

/* ---- ARNR (src/arnr.rs) */
int vo_build_arnr_altref(const vp8a_i420* frames, uint32_t n, uint32_t center,
                         uint32_t strength, uint8_t* y_out, uint8_t* u_out, uint8_t* v_out,
                         uint32_t threads);
/* refine_search of one block (src/arnr.rs:264): returns packed mvx, mvy, sad. */
void vo_arnr_refine_search(const vp8a_i420* src, const vp8a_i420* refp, uint32_t bx,
                           uint32_t by, uint32_t bw, uint32_t bh, int32_t* mvx, int32_t* mvy,
                           uint32_t* sad);

/* ---- §15 loop filter (src/loop_filter.rs) */
void vo_lf_derive(uint8_t level, uint8_t sharpness, int key_frame, uint8_t out4[4]);
int32_t vo_common_adjust(int use_outer_taps, uint8_t* seg4);
void vo_simple_segment(uint8_t edge_limit, uint8_t* seg4);
void vo_subblock_filter(uint8_t hev_threshold, uint8_t interior, uint8_t edge, uint8_t* seg8);
void vo_mb_filter(uint8_t hev_threshold, uint8_t interior, uint8_t edge, uint8_t* seg8);
uint8_t vo_mb_filter_level(const vp8a_filter_config* c, const vp8a_mb_lf_info* mb);
int vo_filter_frame(vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                    const vp8a_filter_config* config);
uint64_t vo_reconstruction_ssd(const vp8a_planes* planes, const vp8a_source* src);
uint64_t vo_score_filter_candidate(const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                                   const vp8a_filter_config* base, const vp8a_source* src,
                                   uint8_t level, uint8_t sharpness, uint32_t every_rows);
void vo_filter_sweep(const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                     const vp8a_filter_config* base, const vp8a_source* src,
                     uint32_t every_rows, uint64_t* ssd_out, uint32_t threads);
void vo_select_filter_params(const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                             const vp8a_filter_config* base, const vp8a_source* src,
                             uint8_t* level, uint8_t* sharp, uint32_t threads);
void vo_select_filter_params_sampled(const vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                                     const vp8a_filter_config* base, const vp8a_source* src,
                                     uint32_t every_rows, uint32_t sweep_sharpness,
                                     uint8_t* level, uint8_t* sharp, uint32_t threads);
/* The reference's selection walks, as pure functions of a 64x8 SSD table
 * (used to check the product's host-side replay). */
void vo_select_from_table_full(const uint64_t* ssd, uint8_t base_sharp, uint8_t* level,
                               uint8_t* sharp);
void vo_select_from_table_sampled(const uint64_t* ssd, uint8_t base_sharp, int sweep,
                                  uint8_t* level, uint8_t* sharp);

/* ---- §18 inter prediction (src/motion_comp.rs; predict.c) */
vp8a_mv vo_chroma_mv(vp8a_mv luma_eighth);
void vo_split_chroma_mvs(const vp8a_mv* split16, vp8a_mv* out4);
void vo_sixtap_2d(const uint8_t* halo81, int mx, int my, int filter_set, uint8_t* out16);
void vo_predict_inter_mb(const vp8a_planes* ref, uint32_t mb_col, uint32_t mb_row, vp8a_mv luma_mv,
                         int full_pixel, int filter_set, uint8_t* out384);
void vo_predict_split_mv(const vp8a_planes* ref, uint32_t mb_col, uint32_t mb_row,
                         const vp8a_mv* split16, int full_pixel, int filter_set, uint8_t* out384);
void vo_predict_inter_mb_batch(const vp8a_planes* ref, const uint32_t* mb_xy, const vp8a_mv* mvs,
                               uint32_t n, int full_pixel, int filter_set, uint8_t* out);
void vo_predict_split_mv_batch(const vp8a_planes* ref, const uint32_t* mb_xy, const vp8a_mv* mvs16,
                               uint32_t n, int full_pixel, int filter_set, uint8_t* out);
int vo_predict_inter_frame(const vp8a_planes* refs, const uint8_t* ref_ids, uint32_t n_refs,
                           const vp8a_mb_decision* dec, int full_pixel, int filter_set,
                           vp8a_planes* out);

/* ---- §14 inter reconstruction, trellis off (src/encoder.rs, src/dequant.rs,
 * src/forward_transform.rs, src/inverse_transform.rs; recon.c) */
void vo_dequant_factors(int32_t q, int32_t ydc, int32_t y2dc, int32_t y2ac, int32_t uvdc,
                        int32_t uvac, int16_t* out);
void vo_segment_factors(const vp8a_quant_indices* qi, int has_segment, int32_t segment_quant,
                        int absolute, int16_t* out);
void vo_forward_dct_4x4(const int16_t* in, int16_t* out);
void vo_forward_wht_4x4(const int16_t* in, int16_t* out);
void vo_inverse_dct_4x4(const int16_t* in, int16_t* out);
void vo_inverse_wht_4x4(const int16_t* in, int16_t* out);
void vo_enc_quantize_block(int16_t* blk, int16_t dc, int16_t ac);
int vo_reconstruct_inter_mb(const uint8_t* src384, uint8_t* pred, const int16_t* f, int split,
                            int16_t* coeffs);
int vo_reconstruct_inter_frame(const vp8a_i420* frame, const vp8a_planes* refs,
                               const uint8_t* ref_ids, uint32_t n_refs,
                               const vp8a_mb_decision* dec, const vp8a_quant_indices* qi,
                               const int8_t* mb_segment, const int16_t* segment_quant,
                               int segment_abs, int full_pixel, int filter_set,
                               vp8a_planes* out, int16_t* coeffs, uint8_t* flags,
                               vp8a_mb_lf_info* lf, uint32_t threads);

/* ---- VP8 decoder restatement (decoder.c) */
typedef struct vo_vp8_decoder vo_vp8_decoder;
/* Caller buffers one decode fills (MB-padded planes of the stream's grid). */
typedef struct vo_vp8_capture {
  uint8_t* refs[3][3];   /* LAST, GOLDEN, ALTREF in force x (y, u, v) */
  uint8_t* pred[3];      /* inter MBs' §18 prediction (intra MBs 0) */
  uint8_t* pre[3];       /* reconstruction before the loop filter */
  uint8_t* post[3];      /* reconstruction after it */
  vp8a_mb_decision* dec; /* per MB: ref_frame (INTRA for intra), mode, mv, split_mvs */
  vp8a_mb_lf_info* lf;
  vp8a_filter_config* cfg;
  int32_t key, version, filtered;
  int32_t mb_cols, mb_rows;  /* set by the caller: the buffers' MB grid */
  int32_t captured;          /* 1 when the last frame's grid matched and was captured */
} vo_vp8_capture;
vo_vp8_decoder* vo_vp8_decoder_new(void);
void vo_vp8_decoder_free(vo_vp8_decoder* d);
void vo_vp8_decoder_capture(vo_vp8_decoder* d, vo_vp8_capture* cap);
int vo_vp8_decoder_prime(vo_vp8_decoder* d, uint32_t width, uint32_t height, const uint8_t* const* refs);
int vo_vp8_decode_frame(vo_vp8_decoder* d, const uint8_t* data, size_t size, uint8_t* out,
                        uint32_t* width, uint32_t* height, int* shown);

/* ---- threading helper */
typedef void (*vo_task_fn)(void* arg, uint32_t index);
void vo_parallel_for(uint32_t n, uint32_t threads, vo_task_fn fn, void* arg);

#ifdef __cplusplus
}
#endif

#endif
