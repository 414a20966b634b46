/*
 * vp8a.h — C ABI of the B200 VP8 encoder-analysis path.
 *
 * This is the drop-in boundary a Rust (or any FFI) caller binds in place of
 * the pure-Rust encoder-analysis functions of oxideav-vp8 0.2.9. Every entry
 * point below cites the reference function it replaces (file:line inside the
 * oxideav-vp8 crate). Signatures use only plain C types: pointers, sizes and
 * the POD structs declared here. No torch or CUDA type crosses the ABI except
 * the opaque `void*` returned by vp8a_ctx_stream().
 *
 * Memory: every buffer argument may live in host memory (pageable or pinned)
 * or in device memory of the context's GPU; the library inspects each pointer.
 * Host buffers are staged through context-owned device buffers and the call
 * returns after its host outputs are written. A call whose buffers are all
 * device memory is asynchronous on the context stream (vp8a_ctx_synchronize
 * waits for it). One context = one GPU + one CUDA stream; a context must not
 * be used from two threads at once (the reference's per-call `threads` budget
 * becomes the GPU's own parallelism).
 *
 * Errors: every function returns a vp8a_status. The codes mirror the
 * reference's EncodeError (src/encoder.rs:69) plus device conditions. Caller
 * bugs the reference panics on (e.g. ARNR centre out of range,
 * src/arnr.rs:494) return VP8A_E_INVALID_ARGUMENT instead of aborting.
 */
#ifndef VP8A_H
#define VP8A_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */

typedef enum vp8a_status {
  VP8A_OK = 0,
  /* EncodeError::InvalidDimensions — width/height 0 or > 0x3FFF. */
  VP8A_E_INVALID_DIMENSIONS = 1,
  /* EncodeError::QuantIndexOutOfRange (> 127). */
  VP8A_E_QUANT_INDEX_OUT_OF_RANGE = 2,
  /* EncodeError::LoopFilterLevelOutOfRange (> 63). */
  VP8A_E_LOOP_FILTER_LEVEL_OUT_OF_RANGE = 3,
  /* EncodeError::SharpnessLevelOutOfRange (> 7). */
  VP8A_E_SHARPNESS_LEVEL_OUT_OF_RANGE = 4,
  /* EncodeError::ReferenceDimensionsMismatch. */
  VP8A_E_REFERENCE_DIMENSIONS_MISMATCH = 5,
  /* A precondition the reference asserts or panics on (null pointer, count
   * mismatch, centre index out of range, MV outside [-1023, 1023]). */
  VP8A_E_INVALID_ARGUMENT = 6,
  /* A CUDA runtime call failed; vp8a_last_error() has the text. */
  VP8A_E_CUDA = 7,
  /* A device-side bounded wait ran out (a wavefront producer never
   * advanced); the context stays usable. */
  VP8A_E_DEVICE_TIMEOUT = 8,
  VP8A_E_OUT_OF_MEMORY = 9,
  VP8A_E_NO_DEVICE = 10,
  /* EncodeError::InvalidDctPartitionCount (not 1, 2, 4 or 8). */
  VP8A_E_INVALID_DCT_PARTITION_COUNT = 11,
  /* EncodeError::FirstPartitionTooLarge (> 0x7FFFF bytes). */
  VP8A_E_FIRST_PARTITION_TOO_LARGE = 12,
  /* EncodeError::Token(CoefficientOutOfRange): |coefficient| > 2114. */
  VP8A_E_COEFFICIENT_OUT_OF_RANGE = 13,
  /* EncodeError::InvalidCopyBufferSelector. */
  VP8A_E_INVALID_COPY_BUFFER_SELECTOR = 14,
  /* EncodeError::LoopFilterDeltaOutOfRange (|delta| > 63). */
  VP8A_E_LOOP_FILTER_DELTA_OUT_OF_RANGE = 15
} vp8a_status;

/* ------------------------------------------------------------------ types */

/* Mv (src/motion_vector.rs:65): quarter-pel luma vector, components in
 * [-1023, 1023] on the wire. */
typedef struct vp8a_mv {
  int16_t row;
  int16_t col;
} vp8a_mv;

/* SearchResult (src/motion_search.rs:248). */
typedef struct vp8a_search_result {
  vp8a_mv mv;
  uint32_t sad;
} vp8a_search_result;

/* LumaRef (src/motion_search.rs:230): a reference luma plane. For encoder
 * searches width/height are the MB-padded plane (mb_cols*16 x mb_rows*16,
 * src/encoder/inter.rs:545-550). Fetches outside replicate the edge pixel. */
typedef struct vp8a_luma_ref {
  const uint8_t* plane;
  uint64_t stride;
  uint32_t width;
  uint32_t height;
} vp8a_luma_ref;

/* I420Frame (src/encoder.rs:5419): visible-size source picture; chroma is
 * ceil(w/2) x ceil(h/2). */
typedef struct vp8a_i420 {
  uint32_t width;
  uint32_t height;
  const uint8_t* y;
  const uint8_t* u;
  const uint8_t* v;
  uint64_t y_stride;
  uint64_t uv_stride;
} vp8a_i420;

/* KeyframePlanes (src/frame.rs:123): MB-padded reconstruction planes,
 * luma (mb_cols*16) x (mb_rows*16), chroma (mb_cols*8) x (mb_rows*8). */
typedef struct vp8a_planes {
  uint8_t* y;
  uint8_t* u;
  uint8_t* v;
  uint64_t y_stride;
  uint64_t uv_stride;
  uint32_t mb_cols;
  uint32_t mb_rows;
} vp8a_planes;

/* RefFrame (src/motion_comp.rs) as used by the census and the §9.4 deltas. */
enum { VP8A_REF_INTRA = 0, VP8A_REF_LAST = 1, VP8A_REF_GOLDEN = 2, VP8A_REF_ALTREF = 3 };

/* InterMode (src/near_mv.rs:68). */
enum { VP8A_MODE_ZERO = 0, VP8A_MODE_NEAREST = 1, VP8A_MODE_NEAR = 2, VP8A_MODE_NEW = 3,
       VP8A_MODE_SPLIT = 4, VP8A_MODE_NONE = 255 };

/* MvPartition (src/near_mv.rs:539), in partition_id order. */
enum { VP8A_PART_TOP_BOTTOM = 0, VP8A_PART_LEFT_RIGHT = 1, VP8A_PART_QUARTERS = 2,
       VP8A_PART_MV16 = 3, VP8A_PART_NONE = 255 };

/* SubMvRefMode (src/near_mv.rs). */
enum { VP8A_SUBMV_LEFT = 0, VP8A_SUBMV_ABOVE = 1, VP8A_SUBMV_ZERO = 2, VP8A_SUBMV_NEW = 3 };

/* MvContexts (src/motion_vector.rs:79): two 19-entry probability vectors,
 * row then column. */
typedef struct vp8a_mv_contexts {
  uint8_t p[2][19];
} vp8a_mv_contexts;

/* The per-MB outcome of the exhaustive inter analysis (MbDecision,
 * src/encoder/inter.rs, with PickedMbForRef's search fields,
 * src/encoder.rs:8470-8514). */
typedef struct vp8a_mb_decision {
  uint8_t ref_frame;   /* VP8A_REF_* of the winning reference */
  uint8_t mode;        /* VP8A_MODE_* */
  uint8_t partition;   /* VP8A_PART_* (SPLIT only) */
  uint8_t reserved;
  vp8a_mv mv;          /* chosen MV (SPLIT: split_mvs[15]) */
  double j;            /* winning per-ref J (without ref_frame_tree bits) */
  double total;        /* j + lambda * ref_frame_tree_bits */
  vp8a_mv split_mvs[16];
  uint8_t submv_modes[16];
} vp8a_mb_decision;

/* Search trace of one (MB, reference) pick (the search part of
 * pick_mb_for_ref, src/encoder.rs:8546-8652). Optional output. */
typedef struct vp8a_ref_search {
  vp8a_mv best_predictor;
  vp8a_mv nearest_mv;
  vp8a_mv near_mv;
  uint32_t sad_zero;
  vp8a_search_result whole;
  vp8a_search_result half;
  vp8a_search_result quarter;
  uint32_t sad_nearest;
  uint32_t sad_near;
  uint8_t chosen_mode;
  uint8_t split_partition;
  uint8_t reserved[2];
  double j;
} vp8a_ref_search;

/* MbInfo (src/near_mv.rs:127): the §16.3 census record one MB leaves for
 * its neighbours. Border / intra MBs have ref_frame = VP8A_REF_INTRA. */
typedef struct vp8a_mb_info {
  uint8_t ref_frame;
  uint8_t is_split;
  uint8_t has_split_mvs;
  uint8_t reserved;
  vp8a_mv mv;
  vp8a_mv split_mvs[16];
} vp8a_mb_info;

/* EncodeEffort (src/encoder/effort.rs), the RD inter search shapes
 * (SearchShape, src/encoder/inter_search.rs:62-162). */
enum { VP8A_EFFORT_FASTEST = 0, VP8A_EFFORT_FAST = 1, VP8A_EFFORT_BALANCED = 2, VP8A_EFFORT_THOROUGH = 3 };

/* The inter candidate decide_mb_rd's search selects for one MB
 * (src/encoder/inter_search.rs:881-1060), before its transform-model,
 * SPLITMV and intra comparisons. */
typedef struct vp8a_rd_inter {
  uint8_t ref_frame;   /* VP8A_REF_* of the winner */
  uint8_t mode;        /* VP8A_MODE_ZERO / NEAREST / NEAR / NEW */
  uint8_t n_searched;  /* references whole-pel searched before the early stop */
  uint8_t leader;      /* index (into refs) of the cheapest whole-pel result */
  vp8a_mv mv;
  uint32_t sad;
  double cost;         /* sad + sqrt(lambda) * bits */
  double bits;         /* ref_frame_tree_bits + mode bits (+ MV differential) */
  vp8a_search_result found[3]; /* whole-pel result per reference, in refs order */
} vp8a_rd_inter;

/* Per-MB side information the §15 pass consults (MacroblockModes +
 * has_coeffs + InterFilterInfo, src/loop_filter.rs:1364-1489). */
typedef struct vp8a_mb_lf_info {
  uint8_t y_mode_is_bpred; /* y_mode == B_PRED (SPLITMV MBs are recorded as B_PRED) */
  uint8_t has_coeffs;      /* mb_has_coeffs (src/loop_filter.rs:1497) */
  uint8_t ref_frame;       /* VP8A_REF_*; VP8A_REF_INTRA for intra MBs */
  uint8_t inter_mode;      /* VP8A_MODE_*; VP8A_MODE_NONE for intra MBs */
  int8_t segment_id;       /* -1 = None */
  uint8_t reserved[3];
} vp8a_mb_lf_info;

/* FrameFilterConfig (src/loop_filter.rs:891). */
typedef struct vp8a_filter_config {
  uint8_t simple;
  uint8_t key_frame;
  uint8_t loop_filter_level;
  uint8_t sharpness_level;
  uint8_t segmentation_enabled;
  uint8_t segment_abs;
  uint8_t delta_enabled;
  uint8_t reserved;
  int16_t segment_lf_level[4];
  int16_t ref_delta_current;
  int16_t bpred_mode_delta;
  int16_t ref_delta_last;
  int16_t ref_delta_golden;
  int16_t ref_delta_altref;
  int16_t zero_mv_mode_delta;
  int16_t other_mv_mode_delta;
  int16_t split_mv_mode_delta;
} vp8a_filter_config;

/* SourcePlanes (src/loop_filter.rs:1916): the visible source window. */
typedef struct vp8a_source {
  uint32_t width;
  uint32_t height;
  const uint8_t* y;
  const uint8_t* u;
  const uint8_t* v;
  uint64_t y_stride;
  uint64_t uv_stride;
} vp8a_source;

/* --------------------------------------------------------------- context */

typedef struct vp8a_ctx vp8a_ctx;

/* Create a context on CUDA device `device` with its own non-blocking stream.
 * Fails with VP8A_E_NO_DEVICE when no GPU is visible: there is no CPU
 * fallback. */
vp8a_status vp8a_ctx_create(int device, vp8a_ctx** out);
vp8a_status vp8a_ctx_destroy(vp8a_ctx* ctx);
/* The context's cudaStream_t, as an opaque pointer. */
void* vp8a_ctx_stream(vp8a_ctx* ctx);
/* Wait for the context stream; returns VP8A_E_DEVICE_TIMEOUT when a bounded
 * device wait of an asynchronous call ran out since the last check. */
vp8a_status vp8a_ctx_synchronize(vp8a_ctx* ctx);
/* Kernel launches issued by this context since creation. */
uint64_t vp8a_ctx_launch_count(const vp8a_ctx* ctx);
/* No counterpart in the reference (its threads join instead of polling).
 * Sets how many times a wavefront wait of the inter analysis (an MB row
 * waiting for the row above it) may poll before it gives up: the call then
 * returns VP8A_E_DEVICE_TIMEOUT, every CTA leaves, and the context stays
 * usable. Default 2^24 polls (seconds). 0 gives up at the first poll that
 * finds the row above behind, which makes the timeout path testable without
 * hanging or faulting anything. Applies to calls issued after it. */
vp8a_status vp8a_ctx_set_wait_limit(vp8a_ctx* ctx, uint64_t polls);
/* No counterpart in the reference (launch shapes of the device kernels).
 * With autotune on (the default) the loop-filter sweep times every launch
 * shape that fits — passes per CTA, threads per CTA, next-MB prefetch — on
 * the first scored sweep of each picture shape and keeps the fastest for
 * that shape in the context (the first call takes longer); off, a cost
 * model picks. Results never depend on the shape. */
vp8a_status vp8a_ctx_set_autotune(vp8a_ctx* ctx, uint32_t on);
/* No counterpart in the reference. On, the inter analysis first builds
 * each reference's 16 quarter-pel sub-pel planes (every §18.3 sample at
 * even eighth-pel fractions, over the MB-padded plane plus a 32-pixel
 * border) in a parallel pass, and its half- and quarter-pel refinements
 * read their predictions from them; off (the default), it synthesises each
 * candidate's prediction inside the wavefront. The results are the same.
 * On costs 16 planes of device scratch per reference and, measured at
 * 1080p, is slower (2.56 against 2.41 ms): an MB's latency is set by its
 * SPLITMV partitions, which run beside the refinements. */
vp8a_status vp8a_ctx_set_subpel_planes(vp8a_ctx* ctx, uint32_t on);
/* TrellisStrength (src/encoder.rs:2669-2711) of this context's inter
 * reconstructions (vp8a_reconstruct_inter_frame[s]): 0 (the default here)
 * quantises by plain rounding, TrellisStrength::OFF; > 0 runs the §13
 * trellis quantiser (trellis_quantize_block, src/encoder.rs:3095) on every
 * block at lambda = rd_lambda(factors) * strength * 0.04 against the §13.5
 * default coefficient probabilities, as the reference's inter path does with
 * KeyframeParams::trellis_strength (whose default is 1.0). Clamped to 0..=8;
 * NaN means 1.0. Applies to calls issued after it. */
vp8a_status vp8a_ctx_set_trellis_strength(vp8a_ctx* ctx, double strength);
/* Forces the loop-filter sweep's launch shape (for tests): `passes` per
 * CTA (1-3; 0 = back to automatic), `threads` per CTA, `prefetch` 0/1. A
 * sweep whose picture the shape does not fit returns
 * VP8A_E_INVALID_ARGUMENT. */
vp8a_status vp8a_ctx_force_sweep_layout(vp8a_ctx* ctx, uint32_t passes, uint32_t threads, uint32_t prefetch);
/* The last sweep's launch shape: out[0] passes per CTA, out[1] threads per
 * CTA, out[2] prefetch, out[3] CTAs per SM (0: rings in global memory). */
vp8a_status vp8a_ctx_last_sweep_layout(const vp8a_ctx* ctx, uint32_t out[4]);
/* Text of the last error on this thread ("" if none). */
const char* vp8a_last_error(void);
/* ABI version of this header (major << 16 | minor). */
uint32_t vp8a_abi_version(void);

/* ------------------------------------------------- motion search (§17/§18) */

/* Batched mb_luma_sad_at_mv (src/motion_search.rs:470) — the §18 six-tap
 * sub-pel SAD; a whole-pel MV takes the copy path, which equals
 * mb_luma_sad_at_whole_mv (src/motion_search.rs:291). Item i scores the
 * source MB src_mbs[256*i] (16x16, stride 16) at MB position
 * (mb_xy[2i], mb_xy[2i+1]) = (mb_col, mb_row) against `ref` at mvs[i]. */
vp8a_status vp8a_mb_luma_sad_at_mv(vp8a_ctx* ctx, const vp8a_luma_ref* ref,
                                   const uint8_t* src_mbs, const uint32_t* mb_xy,
                                   const vp8a_mv* mvs, uint32_t n, uint32_t* sad_out);

/* Batched small_diamond_search_luma (src/motion_search.rs:381). */
vp8a_status vp8a_small_diamond_search_luma(vp8a_ctx* ctx, const vp8a_luma_ref* ref,
                                           const uint8_t* src_mbs, const uint32_t* mb_xy,
                                           const vp8a_mv* centers, uint32_t max_iters,
                                           uint32_t n, vp8a_search_result* out);

/* Batched half_pixel_refine_luma (src/motion_search.rs:564). Centres must
 * be whole-pel and inside [-1023, 1023]. */
vp8a_status vp8a_half_pixel_refine_luma(vp8a_ctx* ctx, const vp8a_luma_ref* ref,
                                        const uint8_t* src_mbs, const uint32_t* mb_xy,
                                        const vp8a_mv* whole_centers, uint32_t n,
                                        vp8a_search_result* out);

/* Batched quarter_pixel_refine_luma (src/motion_search.rs:666). Centres
 * must be half-pel and inside [-1023, 1023]. */
vp8a_status vp8a_quarter_pixel_refine_luma(vp8a_ctx* ctx, const vp8a_luma_ref* ref,
                                           const uint8_t* src_mbs, const uint32_t* mb_xy,
                                           const vp8a_mv* half_centers, uint32_t n,
                                           vp8a_search_result* out);

/* The full descent pick_mb_for_ref runs per (MB, ref)
 * (src/encoder.rs:8576-8596): diamond(center, max_iters) -> half -> quarter,
 * fused in one kernel. Any of the three outputs may be NULL. */
vp8a_status vp8a_motion_descent(vp8a_ctx* ctx, const vp8a_luma_ref* ref,
                                const uint8_t* src_mbs, const uint32_t* mb_xy,
                                const vp8a_mv* centers, uint32_t max_iters, uint32_t n,
                                vp8a_search_result* whole_out, vp8a_search_result* half_out,
                                vp8a_search_result* quarter_out);

/* vp8a_motion_descent for the items whose active[i] is non-zero; the other
 * items' outputs are left as they were. No counterpart in the reference:
 * the learned search's fallback runs the plain descent on the MBs it
 * flags, with the flags kept on the device. */
vp8a_status vp8a_motion_descent_masked(vp8a_ctx* ctx, const vp8a_luma_ref* ref,
                                       const uint8_t* src_mbs, const uint32_t* mb_xy,
                                       const vp8a_mv* centers, uint32_t max_iters, uint32_t n,
                                       const uint8_t* active, vp8a_search_result* whole_out,
                                       vp8a_search_result* half_out,
                                       vp8a_search_result* quarter_out);

/* ------------------------------------- exhaustive inter analysis (§16/§17) */

/* The exhaustive per-MB analysis of a P frame with intra picking off:
 * analyse_inter_frame (src/encoder/inter.rs:263) with
 * decide_mb_exhaustive (src/encoder/inter.rs:537) and pick_mb_for_ref's
 * search and mode decision (src/encoder.rs:8516-8702, SPLITMV
 * src/encoder.rs:7573-8246). `refs[k]` (k < n_refs) are MB-padded
 * reference planes in scoring order with ids `ref_ids[k]` (VP8A_REF_*);
 * `mv_contexts` NULL means the §17.2 defaults; `lambda` is the RD
 * multiplier (rd_lambda, src/encoder.rs:3742): finite and >= 0, else
 * VP8A_E_INVALID_ARGUMENT. Writes mb_cols*mb_rows
 * decisions in raster order; `trace` (optional) receives n_refs entries
 * per MB. The MB-row wavefront runs on the device: MB (r, c) starts once
 * MB (r-1, c) is decided (its census neighbours are the above, left and
 * above-left MBs; the reference's row contract also waits for the
 * above-right MB, which only its intra candidates read). A row's wait for
 * the row above is bounded (vp8a_ctx_set_wait_limit); when it runs out the
 * call returns VP8A_E_DEVICE_TIMEOUT if any buffer was host memory (the call
 * then waits for its kernel anyway), and otherwise stays asynchronous and
 * the next vp8a_ctx_synchronize returns it. */
vp8a_status vp8a_analyse_inter_frame(vp8a_ctx* ctx, const vp8a_i420* frame,
                                     const vp8a_planes* refs, const uint8_t* ref_ids,
                                     uint32_t n_refs, const vp8a_mv_contexts* mv_contexts,
                                     double lambda, vp8a_mb_decision* decisions,
                                     vp8a_ref_search* trace);

/* The RD-effort inter search of decide_mb_rd for every MB of a frame
 * (whole_pixel_search, sub_pixel_refine and the free ZERO/NEAREST/NEAR
 * candidates, src/encoder/inter_search.rs:198-552, :846-1060), given each
 * MB's census neighbours: `neighbours[3*i + k]` is the above (k=0), left
 * (k=1) and above-left (k=2) record of MB i (raster order). `y1_ac` is the
 * luma AC dequantisation factor (good_enough threshold), `effort` one of
 * VP8A_EFFORT_*. Every MB is independent given its neighbours, so all MBs
 * run in parallel. */
vp8a_status vp8a_rd_inter_search(vp8a_ctx* ctx, const vp8a_i420* frame, const vp8a_planes* refs,
                                 const uint8_t* ref_ids, uint32_t n_refs,
                                 const vp8a_mv_contexts* mv_contexts, double lambda,
                                 uint32_t y1_ac, uint32_t effort,
                                 const vp8a_mb_info* neighbours, vp8a_rd_inter* out);

/* rd_lambda (src/encoder.rs:3742) for a luma AC quantiser index 0..=127. */
double vp8a_rd_lambda(uint32_t y_ac_qi);

/* ------------------------------------------- §18 inter prediction (MC) */

/* QuantIndices (src/coded_header.rs:171); an absent delta is 0. */
typedef struct vp8a_quant_indices {
  uint8_t y_ac_qi;
  int8_t y_dc_delta;
  int8_t y2_dc_delta;
  int8_t y2_ac_delta;
  int8_t uv_dc_delta;
  int8_t uv_ac_delta;
  uint8_t reserved[2];
} vp8a_quant_indices;

/* FilterSet (src/motion_comp.rs:344). filter_set_for_version
 * (src/motion_comp.rs:370): frame-tag version 0 uses SIXTAP, any other
 * version BILINEAR. */
enum { VP8A_FILTER_SIXTAP = 0, VP8A_FILTER_BILINEAR = 1 };

/* Batched predict_inter_mb (src/motion_comp.rs:1986): item i predicts the
 * MB at (mb_xy[2i], mb_xy[2i+1]) = (mb_col, mb_row) from `ref` under the
 * quarter-pel luma vector mvs[i]. `full_pixel` is the version-3 full-pel
 * flag (apply_full_pixel, src/motion_comp.rs:256), `filter_set` one of
 * VP8A_FILTER_*. `out` receives 384 bytes per item in ReconstructedMb's
 * layout (src/reconstruct.rs:178): y[256] (16x16 raster), then u[64] and
 * v[64] (8x8 raster). Fetches outside the MB-padded planes replicate the
 * edge pixel, as the reference's do. */
vp8a_status vp8a_predict_inter_mb(vp8a_ctx* ctx, const vp8a_planes* ref, const uint32_t* mb_xy,
                                  const vp8a_mv* mvs, uint32_t n, uint32_t full_pixel,
                                  uint32_t filter_set, uint8_t* out);

/* Batched predict_split_mv (src/motion_comp.rs:2228): as
 * vp8a_predict_inter_mb with 16 quarter-pel vectors per item,
 * split_mvs[16i + b] for luma sub-block b in raster order; chroma takes
 * split_chroma_mvs (src/motion_comp.rs:2175). */
vp8a_status vp8a_predict_split_mv(vp8a_ctx* ctx, const vp8a_planes* ref, const uint32_t* mb_xy,
                                  const vp8a_mv* split_mvs, uint32_t n, uint32_t full_pixel,
                                  uint32_t filter_set, uint8_t* out);

/* The prediction pick_mb_for_ref builds for its chosen mode
 * (src/encoder.rs:8704-8735) for every MB of a frame: predict_split_mv for
 * a VP8A_MODE_SPLIT decision, predict_inter_mb with `mv` otherwise, from
 * the reference of `ref_frame`, written into the MB-padded `out` planes at
 * the MB's position. decisions holds out->mb_cols * out->mb_rows records in
 * raster order (vp8a_analyse_inter_frame's output). `refs[k]` has id
 * `ref_ids[k]` (VP8A_REF_LAST/GOLDEN/ALTREF) and the output's MB grid. MBs
 * whose ref_frame is VP8A_REF_INTRA or has no plane in `refs` keep the
 * pixels `out` already holds. */
vp8a_status vp8a_predict_inter_frame(vp8a_ctx* ctx, const vp8a_planes* refs,
                                     const uint8_t* ref_ids, uint32_t n_refs,
                                     const vp8a_mb_decision* decisions, uint32_t full_pixel,
                                     uint32_t filter_set, vp8a_planes* out);

/* ------------------------------------- §14 inter reconstruction (trellis off) */

/* MbDequantFactors::from_quant_indices / for_segment (src/dequant.rs:169,
 * :201): out = {y1_dc, y1_ac, y2_dc, y2_ac, uv_dc, uv_ac}. With
 * has_segment, the base index is segment_quant (absolute) or y_ac_qi +
 * segment_quant. Host only; no context needed. */
void vp8a_dequant_factors(const vp8a_quant_indices* qi, uint32_t has_segment,
                          int32_t segment_quant, uint32_t absolute, int16_t* out);

/* Per-MB flags of vp8a_reconstruct_inter_frame. */
enum { VP8A_MB_SKIP = 1, VP8A_MB_HAS_COEFFS = 2 };

/* The §18 + §14 step pick_mb_for_ref runs for its chosen mode
 * (src/encoder.rs:8704-8800) with TrellisStrength::OFF (src/encoder.rs:2677),
 * for every MB of a frame: the prediction of vp8a_predict_inter_frame; the
 * residual against the source MB (I420Frame::extract_mb,
 * src/encoder.rs:5549, edge-replicated); forward DCT, Y2 WHT for non-SPLITMV
 * MBs and plain rounding (transform_whole_block_luma_rd :3815,
 * transform_split_mv_mb_rd :8259, transform_chroma_plane_rd :4133,
 * enc_quantize_block :2127); §11.1 skip detection; dequantisation and
 * reconstruct_inter_mb / reconstruct_split_mv_mb (src/motion_comp.rs:2098,
 * :2340). `frame` is the visible source picture; `recon` (MB-padded, the
 * references' grid) receives the reconstruction. Optional outputs:
 * `coeffs`, 400 int16 per MB in MbCoeffs order (src/frame.rs:98: y2[16],
 * y[16][16], u[4][16], v[4][16], raster coefficient order, quantised);
 * `mb_flags`, VP8A_MB_SKIP | VP8A_MB_HAS_COEFFS per MB (mb_has_coeffs,
 * src/loop_filter.rs:1500); `lf_info`, the MB's §15 side information for
 * vp8a_filter_frame / the loop-filter search (SPLITMV recorded as B_PRED,
 * src/loop_filter.rs:1258-1266; segment_id from mb_segment). `mb_segment`
 * (optional, one int8 per MB, -1 = none) selects the factors of segment k
 * from segment_quant[k] (for_segment with `segment_abs`). MBs whose
 * ref_frame is VP8A_REF_INTRA or has no plane in `refs` keep recon's pixels
 * and their lf_info record, and get flags 0 and zero coefficients. */
vp8a_status vp8a_reconstruct_inter_frame(vp8a_ctx* ctx, const vp8a_i420* frame,
                                         const vp8a_planes* refs, const uint8_t* ref_ids,
                                         uint32_t n_refs, const vp8a_mb_decision* decisions,
                                         const vp8a_quant_indices* quant,
                                         const int8_t* mb_segment, const int16_t* segment_quant,
                                         uint32_t segment_abs, uint32_t full_pixel,
                                         uint32_t filter_set, vp8a_planes* recon,
                                         int16_t* coeffs, uint8_t* mb_flags,
                                         vp8a_mb_lf_info* lf_info);

/* ------------------------------------------------------------ ARNR filter */

/* build_arnr_altref (src/arnr.rs:476): temporally filtered altref anchor of
 * `n` frames aligned to frames[center]. Outputs are tightly packed:
 * y_out width*height, u_out/v_out ceil(w/2)*ceil(h/2). `strength` is
 * clamped to 0..=6 (ArnrConfig::new, src/arnr.rs:76). */
vp8a_status vp8a_build_arnr_altref(vp8a_ctx* ctx, const vp8a_i420* frames, uint32_t n,
                                   uint32_t center, uint32_t strength, uint8_t* y_out,
                                   uint8_t* u_out, uint8_t* v_out);

/* build_arnr_altref (src/arnr.rs:476) written straight into MB-padded
 * planes, the KeyframePlanes layout (src/frame.rs:123) an encoder keeps its
 * ALTREF reference in: `out` has mb_cols = ceil(w/16), mb_rows = ceil(h/16)
 * and its own row pitches; the visible anchor is the one
 * vp8a_build_arnr_altref returns, and the padding columns and rows repeat
 * the last visible column and row (the edge replication of an MB-padded
 * reference). The blend kernel writes the padding itself. */
vp8a_status vp8a_build_arnr_altref_planes(vp8a_ctx* ctx, const vp8a_i420* frames, uint32_t n,
                                          uint32_t center, uint32_t strength, const vp8a_planes* out);

/* ------------------------------------------------------- §15 loop filter */

/* filter_inter_frame_flags (src/loop_filter.rs:1364) / filter_frame_flags
 * (src/loop_filter.rs:2506) in place on `planes`. Key frames pass every MB
 * with ref_frame = VP8A_REF_INTRA and config->key_frame = 1. */
vp8a_status vp8a_filter_frame(vp8a_ctx* ctx, vp8a_planes* planes, const vp8a_mb_lf_info* mbs,
                              const vp8a_filter_config* config);

/* reconstruction_ssd (src/loop_filter.rs:1965). */
vp8a_status vp8a_reconstruction_ssd(vp8a_ctx* ctx, const vp8a_planes* planes,
                                    const vp8a_source* src, uint64_t* ssd_out);

/* The whole §9.4 candidate grid: ssd_out[level * 8 + sharpness] is
 * score_filter_candidate (src/loop_filter.rs:2062) for every level 0..=63
 * and sharpness 0..=7 (level 0 is the unfiltered SSD for every sharpness).
 * `every_rows` = 0 scores whole frames; > 0 scores the two-MB-row bands of
 * select_filter_params_sampled (src/loop_filter.rs:2288). */
vp8a_status vp8a_filter_sweep(vp8a_ctx* ctx, const vp8a_planes* planes,
                              const vp8a_mb_lf_info* mbs, const vp8a_filter_config* base,
                              const vp8a_source* src, uint32_t every_rows, uint64_t* ssd_out);

/* No counterpart in the reference. vp8a_filter_sweep for callers that may
 * not allocate device memory once they are running — for instance a host
 * that hands the library a pre-sized memory pool, or a real-time encoder
 * loop where an allocation can stall or fail. It computes exactly what
 * vp8a_filter_sweep computes and allocates nothing: no cudaMalloc, no
 * cudaFree, no staging buffers. Therefore:
 *  - every buffer (the planes, `mbs`, the source planes and the 512-entry
 *    `ssd_out`) must already be device memory of the context's GPU
 *    (VP8A_E_INVALID_ARGUMENT otherwise);
 *  - its scratch (candidate list and step schedule) is one fixed array of
 *    about 72 KiB compiled into the library, which every GPU that loads the
 *    library holds until the process exits; it bounds the picture to at most
 *    256 x 136 MBs (4096 x 2176 pixels), larger grids return
 *    VP8A_E_INVALID_DIMENSIONS;
 *  - the scratch is shared by every call on a device and keeps the last
 *    call's contents (each call rewrites all it reads), so calls whose work
 *    overlaps on the GPU — from different contexts or streams — race; keep
 *    them ordered on one stream;
 *  - the first call on each device looks the scratch's device address up
 *    (cudaGetSymbolAddress); make that first call before any stream
 *    capture.
 * All its work is queued on the context stream (vp8a_ctx_synchronize waits
 * for it). */
vp8a_status vp8a_filter_sweep_noalloc(vp8a_ctx* ctx, const vp8a_planes* planes,
                                      const vp8a_mb_lf_info* mbs, const vp8a_filter_config* base,
                                      const vp8a_source* src, uint32_t every_rows,
                                      uint64_t* ssd_out);

/* vp8a_filter_sweep restricted to level 0 and levels lo_level..hi_level
 * (every sharpness): ssd_out[level * 8 + sharpness] is written for those
 * and UINT64_MAX elsewhere, so the reference's selection walk over the
 * table stays inside the window. No counterpart in the reference: the
 * learned proposal's loop-filter window. */
vp8a_status vp8a_filter_sweep_window(vp8a_ctx* ctx, const vp8a_planes* planes,
                                     const vp8a_mb_lf_info* mbs, const vp8a_filter_config* base,
                                     const vp8a_source* src, uint32_t lo_level, uint32_t hi_level,
                                     uint64_t* ssd_out);

/* select_filter_params (src/loop_filter.rs:2047): the reference's coarse
 * grid + refine + sharpness search, replayed over the device sweep. */
vp8a_status vp8a_select_filter_params(vp8a_ctx* ctx, const vp8a_planes* planes,
                                      const vp8a_mb_lf_info* mbs,
                                      const vp8a_filter_config* base, const vp8a_source* src,
                                      uint8_t* level_out, uint8_t* sharpness_out);

/* FilterSampling::for_key_frame (src/loop_filter.rs:2266): the band
 * spacing and sharpness sweep the key-frame encoder's sampled loop-filter
 * pick uses (src/encoder.rs:6643-6651). Host only; no context needed. */
void vp8a_key_frame_sampling(uint32_t mb_rows, uint32_t* every_rows, uint32_t* sweep_sharpness);

/* select_filter_params_sampled (src/loop_filter.rs:2288) with
 * FilterSampling { every_rows, sweep_sharpness }. */
vp8a_status vp8a_select_filter_params_sampled(vp8a_ctx* ctx, const vp8a_planes* planes,
                                              const vp8a_mb_lf_info* mbs,
                                              const vp8a_filter_config* base,
                                              const vp8a_source* src, uint32_t every_rows,
                                              uint32_t sweep_sharpness, uint8_t* level_out,
                                              uint8_t* sharpness_out);

/* ---------------------------------------------------- batched work lists
 *
 * The reference encodes each stream with its own encoder object
 * (Vp8AltrefStreamEncoder::push_frame, src/stream.rs:2750, one
 * encode_p_frame_multi_ref_auto_loop_filter per frame, src/encoder.rs:9373)
 * and has no batched form. The *_frames / *_altrefs / *_sweeps entry points
 * below take a work list of independent jobs of uneven sizes (many streams'
 * frames) and run every job of one stage in one persistent launch; each
 * job's results are the ones the single-job call gives. At most
 * VP8A_MAX_BATCH_JOBS jobs per call. */
#define VP8A_MAX_BATCH_JOBS 1024u

/* No counterpart in the reference: vp8a_analyse_inter_frame with one
 * proposed vector per (MB, reference) — `proposals` holds n_refs vectors
 * per MB in raster order, e.g. the learned proposal's refined seeds — as a
 * second NEWMV candidate beside the searched one: its exact SAD is computed
 * here and it costs what a searched vector costs (SAD + lambda * (NEWMV
 * mode bits + differential bits)); it replaces the searched vector when
 * strictly cheaper. A zero vector or one beyond +-1023 quarter-pels is not
 * a candidate. Everything else is vp8a_analyse_inter_frame's decision. */
vp8a_status vp8a_analyse_inter_frame_proposals(vp8a_ctx* ctx, const vp8a_i420* frame,
                                               const vp8a_planes* refs, const uint8_t* ref_ids,
                                               uint32_t n_refs, const vp8a_mv_contexts* mv_contexts,
                                               double lambda, const vp8a_mv* proposals,
                                               vp8a_mb_decision* decisions, vp8a_ref_search* trace);

/* One vp8a_analyse_inter_frame call's arguments. */
typedef struct vp8a_analysis_job {
  vp8a_i420 frame;
  const vp8a_planes* refs;              /* n_refs MB-padded references */
  const uint8_t* ref_ids;               /* n_refs VP8A_REF_* */
  uint32_t n_refs;                      /* 1..3 */
  const vp8a_mv_contexts* mv_contexts;  /* NULL = the §17.2 defaults */
  double lambda;
  vp8a_mb_decision* decisions;          /* mb_cols*mb_rows, raster order */
  vp8a_ref_search* trace;               /* optional: n_refs per MB */
} vp8a_analysis_job;

/* vp8a_analyse_inter_frame for every job: the MB rows of all jobs with the
 * same reference count form one work list over one persistent launch (each
 * job keeps its own row-to-row wavefront; jobs with the longest wavefront
 * start first). */
vp8a_status vp8a_analyse_inter_frames(vp8a_ctx* ctx, const vp8a_analysis_job* jobs, uint32_t n_jobs);

/* No counterpart in the reference: vp8a_analyse_inter_frames with
 * vp8a_analyse_inter_frame_proposals' second NEWMV candidate per job.
 * proposals[j] holds job j's n_refs vectors per MB (raster order), or is
 * NULL for a job without proposals. */
vp8a_status vp8a_analyse_inter_frames_proposals(vp8a_ctx* ctx, const vp8a_analysis_job* jobs, uint32_t n_jobs,
                                                const vp8a_mv* const* proposals);

/* One vp8a_build_arnr_altref call's arguments. */
typedef struct vp8a_arnr_job {
  const vp8a_i420* frames;  /* n frames of one size */
  uint32_t n;
  uint32_t center;
  uint32_t strength;
  uint8_t* y_out;
  uint8_t* u_out;
  uint8_t* v_out;
} vp8a_arnr_job;

/* vp8a_build_arnr_altref for every job: one search launch over every
 * job's (frame, strip of blocks) and one blend launch over every job's
 * blocks. */
vp8a_status vp8a_build_arnr_altrefs(vp8a_ctx* ctx, const vp8a_arnr_job* jobs, uint32_t n_jobs);

/* One vp8a_build_arnr_altref_planes call's arguments. */
typedef struct vp8a_arnr_planes_job {
  const vp8a_i420* frames;  /* n frames of one size */
  uint32_t n;
  uint32_t center;
  uint32_t strength;
  vp8a_planes out;          /* MB-padded output planes (written) */
} vp8a_arnr_planes_job;

/* vp8a_build_arnr_altref_planes for every job (launches as
 * vp8a_build_arnr_altrefs). */
vp8a_status vp8a_build_arnr_altrefs_planes(vp8a_ctx* ctx, const vp8a_arnr_planes_job* jobs, uint32_t n_jobs);

/* One vp8a_reconstruct_inter_frame call's arguments (`recon` is written). */
typedef struct vp8a_recon_job {
  vp8a_i420 frame;
  const vp8a_planes* refs;
  const uint8_t* ref_ids;
  uint32_t n_refs;
  uint32_t segment_abs;
  const vp8a_mb_decision* decisions;
  vp8a_quant_indices quant;
  const int8_t* mb_segment;
  const int16_t* segment_quant;
  uint32_t full_pixel;
  uint32_t filter_set;
  vp8a_planes recon;
  int16_t* coeffs;
  uint8_t* mb_flags;
  vp8a_mb_lf_info* lf_info;
} vp8a_recon_job;

/* vp8a_reconstruct_inter_frame for every job: one prediction launch and one
 * reconstruction launch over every job's MBs. */
vp8a_status vp8a_reconstruct_inter_frames(vp8a_ctx* ctx, const vp8a_recon_job* jobs, uint32_t n_jobs);

/* One vp8a_filter_sweep call's arguments. */
typedef struct vp8a_sweep_job {
  vp8a_planes planes;
  const vp8a_mb_lf_info* mbs;
  vp8a_filter_config base;
  vp8a_source src;
  uint32_t every_rows;
  uint64_t* ssd_out;  /* 512 entries, level * 8 + sharpness */
} vp8a_sweep_job;

/* vp8a_filter_sweep for every job: the (job, candidate) pairs of all jobs
 * in one launch when every job's slot rings fit in shared memory (the
 * larger pictures otherwise run as their own launches). */
vp8a_status vp8a_filter_sweeps(vp8a_ctx* ctx, const vp8a_sweep_job* jobs, uint32_t n_jobs);

/* select_filter_params (src/loop_filter.rs:2047) for every job: the
 * reference's walk — the coarse grid 0, 4, ..., 60, 63 at the base
 * sharpness, the +-3 refine around its winner, the other sharpness values
 * at a non-zero chosen level — with each stage of all jobs in one batched
 * sweep launch. Whole frames only (every_rows 0); the jobs' ssd_out is not
 * used (the walk keeps its tables in scratch). level_out[j] and
 * sharpness_out[j] (host memory) receive job j's pair. */
vp8a_status vp8a_select_filter_params_batch(vp8a_ctx* ctx, const vp8a_sweep_job* jobs, uint32_t n_jobs,
                                            uint8_t* level_out, uint8_t* sharpness_out);

/* ------------------------------------------- learned motion proposal
 *
 * No counterpart in the reference: the learned proposal the survey builds
 * beside the plain search. A 4-layer 3x3 conv net (32 channels, BF16
 * weights and activations, FP32 accumulation on the tensor cores) maps an
 * MB's coarse cost volume against a reference (2 x 32 x 32: at each of a
 * 32 x 32 grid of whole-pel vectors 2 px apart, cell (i, j) = (2 (i - 16),
 * 2 (j - 16)) px, the half-resolution SAD of the MB and the reference's
 * texture) to scores over that grid; its best cells seed an exact local
 * search with the plain search's SAD kernels. All buffers are
 * device memory of the context's GPU; all calls are stream-ordered on the
 * context stream and allocate nothing. Activations are NHWC [n][32][32][C]
 * BF16 (uint16 bit patterns); weights [cout][9][cin] with tap
 * (dy + 1) * 3 + (dx + 1). */

/* The net's input for n MBs: item i is the MB at mb_xy[2i], mb_xy[2i+1]
 * (column, row); out = [n][32][32][2] BF16: (32 - the mean absolute
 * difference of the 2x2-averaged MB and reference block at the cell's
 * vector) / 32, and (the averaged reference at the block's centre - 128) /
 * 64. `src` and `ref` are visible luma planes of one size; `out` is
 * 16-byte aligned. */
vp8a_status vp8a_lp_windows(vp8a_ctx* ctx, const vp8a_luma_ref* src, const vp8a_luma_ref* ref,
                            const uint32_t* mb_xy, uint32_t n, uint16_t* out);

/* The exact whole-pel search around the net's seeds for n MBs: item i is
 * the MB at mb_xy[2i], mb_xy[2i+1] (column, row) with its 16x16 source
 * src_mbs[i] (256 bytes) and k seed cells seeds[i*k .. i*k+k-1] (cell c
 * stands for the vector ((c / 32 - 16) * 2, (c % 32 - 16) * 2) px). Every
 * vector within +-radius px of each seed is scored (whole-pel SAD against
 * the edge-clamped `ref`); out[i] = the first smallest in seed, row,
 * column order (vector in quarter-pels, SAD). 1 <= k <= 4, radius <= 4,
 * k * (2 radius + 1)^2 <= 128. */
vp8a_status vp8a_lp_seeded_search(vp8a_ctx* ctx, const vp8a_luma_ref* ref, const uint8_t* src_mbs,
                                  const uint32_t* mb_xy, const int32_t* seeds, uint32_t k, uint32_t radius,
                                  uint32_t n, vp8a_search_result* out);

/* The whole net (2 -> 32 -> 32 -> 32 -> 1, ReLU between) for n images in
 * one launch, activations kept on chip: x = [n][32][32][2] BF16, weights
 * and FP32 biases as for vp8a_lp_conv_forward's four layers. cells[i*k ..]
 * receives image i's k highest-scoring cells, best first (the first cell
 * among equal scores), 1 <= k <= 16; `logits` (optional, [n][1024] FP32)
 * the scores. The same sums as the layer-by-layer calls in another FP32
 * accumulation order. */
vp8a_status vp8a_lp_net_propose(vp8a_ctx* ctx, const uint16_t* x, uint32_t n, const uint16_t* w1,
                                const float* b1, const uint16_t* w2, const float* b2, const uint16_t* w3,
                                const float* b3, const uint16_t* w4, const float* b4, uint32_t k,
                                int32_t* cells, float* logits);

/* One conv layer (cin -> cout in {2->32, 32->32, 32->1}) over n images,
 * + bias, ReLU when `relu`; output BF16 `y` or FP32 `y_f32` (one of them). */
vp8a_status vp8a_lp_conv_forward(vp8a_ctx* ctx, const uint16_t* x, uint32_t cin, const uint16_t* w,
                                 const float* bias, uint32_t cout, uint32_t n, uint32_t relu,
                                 uint16_t* y, float* y_f32);

/* Its gradients: `dw` (cout*9*cin) and `db` (cout) FP32 are accumulated
 * into (zero them first); `dx` (optional, BF16) = the gradient w.r.t. x,
 * multiplied by (x > 0) when `x_relu` (x came out of a ReLU). */
vp8a_status vp8a_lp_conv_backward(vp8a_ctx* ctx, const uint16_t* x, uint32_t cin, const uint16_t* w,
                                  uint32_t cout, uint32_t n, const uint16_t* dy, uint32_t x_relu,
                                  uint16_t* dx, float* dw, float* db);

/* Softmax over each item's 1024 scores; with `labels` (cell index, < 0 =
 * none): the summed cross-entropy added to `loss`, d(scores) =
 * (softmax - onehot) / n into `dlogits` (BF16) and the label's probability
 * into `label_prob` (each optional). */
vp8a_status vp8a_lp_softmax_ce(vp8a_ctx* ctx, const float* logits, const int32_t* labels, uint32_t n,
                               uint16_t* dlogits, float* loss, float* label_prob);

/* Channel sums of n images' activations ([n][32][32][c] BF16, c divides
 * 256, at most 64) added into sums[c] (FP32). */
vp8a_status vp8a_lp_pool(vp8a_ctx* ctx, const uint16_t* x, uint32_t c, uint32_t n, float* sums);

/* The loop-filter level head: features f = sums / count (c of them),
 * scores z = w f + b over `levels` levels ([levels][c] weights), written to
 * `logits` (optional); with label >= 0 the cross-entropy is added to `loss`
 * (optional) and its gradients to dw, db. */
vp8a_status vp8a_lp_lf_head(vp8a_ctx* ctx, const float* sums, float count, uint32_t c, const float* w,
                            const float* b, uint32_t levels, int32_t label, float* logits, float* dw,
                            float* db, float* loss);

/* One Adam step (bias-corrected for `step` >= 1) on FP32 master weights;
 * writes their BF16 copies. */
vp8a_status vp8a_lp_adam(vp8a_ctx* ctx, float* w, const float* grad, float* m, float* v, uint32_t n,
                         float lr, float beta1, float beta2, float eps, uint32_t step, uint16_t* w_bf16);

/* ------------------------------------------- P-frame bitstream (§19.2) */

/* The frame-level choices an inter frame's header carries: KeyframeParams
 * (y_ac_qi, filter_type, levels, nbr_of_dct_partitions), RefreshControls
 * (src/encoder.rs:9174), LoopFilterDeltas (:771) and the segmentation layer
 * (InterSegmentationConfig) of encode_p_frame_multi_ref_inner_driven
 * (src/encoder.rs:10739). */
typedef struct vp8a_frame_header {
  uint32_t width;                   /* visible size, 1..0x3FFF */
  uint32_t height;
  vp8a_quant_indices quant;         /* y_ac_qi; a delta of 0 is not sent */
  uint8_t filter_type;              /* 0 = normal (§15.3), 1 = simple (§15.2) */
  uint8_t loop_filter_level;        /* 0..63 */
  uint8_t sharpness_level;          /* 0..7 */
  uint8_t n_partitions;             /* token partitions: 1, 2, 4 or 8 */
  uint8_t refresh_golden_frame;
  uint8_t refresh_alternate_frame;
  uint8_t copy_buffer_to_golden;    /* 0..2, sent when !refresh_golden_frame */
  uint8_t copy_buffer_to_alternate; /* 0..2, sent when !refresh_alternate_frame */
  uint8_t refresh_last;
  uint8_t pick_intra;               /* 1: prob_intra fitted to the MB counts (the
                                       auto-LF entry point); 0: prob_intra 255 */
  uint8_t fit_skip_prob;            /* 1: prob_skip_false fitted to the skips (the
                                       reduced search); 0: 128 (exhaustive) */
  uint8_t lf_delta_enabled;         /* loop_filter_adj_enable */
  uint8_t lf_delta_update;          /* mode_ref_lf_delta_update */
  uint8_t lf_ref_delta_present;     /* bit k: ref_frame_delta[k] is sent */
  uint8_t lf_mode_delta_present;    /* bit k: mode_delta[k] is sent */
  int8_t lf_ref_delta[4];           /* INTRA, LAST, GOLDEN, ALTREF; |v| <= 63 */
  int8_t lf_mode_delta[4];          /* B_PRED, ZEROMV, other MV, SPLITMV */
  uint8_t segmentation;             /* 1: update_segmentation with the MB map */
  uint8_t segment_lf_present;       /* 1: the per-segment filter deltas are sent */
  int8_t segment_quant[4];          /* §10 quantiser deltas per segment */
  int8_t segment_lf[4];             /* §10 filter-level deltas per segment */
  uint8_t reserved[2];
} vp8a_frame_header;

/* The inter-frame bitstream encode_p_frame_multi_ref_inner_driven writes
 * (src/encoder.rs:11214-11720): the §9.1 frame tag, the first partition
 * (§19.2 header; per MB the segment id, mb_skip_coeff, is_inter_mb, the
 * §16.2 ref_frame and mv_ref_tree walk against the §16.3 census
 * probabilities, NEWMV and NEW4X4 §17.2 differentials against the default
 * MV contexts, SPLITMV partition and sub_mv_ref modes) and the §13 token
 * partitions (MB row r in partition r % n, encode_coeff_block_into
 * src/encoder.rs:1915, skipped MBs clear their contexts,
 * clear_skip_ctx :7369). `decisions` are the analysis's (inter MBs only),
 * `coeffs` the quantised coefficients of vp8a_reconstruct_inter_frame (400
 * per MB, MbCoeffs order), `mb_segment` one id per MB when the header
 * enables segmentation (-1 = segment 0), `token_prob_updates` NULL or 1056
 * entries in [4][8][3][11] order (0 = keep the §13.5 default, else the new
 * probability, sent as a §13.4 update and coded against). mb_skip_coeff is
 * derived from the coefficients as the reference does (src/encoder.rs:8746).
 * Writes the frame to `out` and its size to `out_size`; when `out` is NULL
 * or `out_capacity` is short, returns VP8A_E_INVALID_ARGUMENT with
 * `out_size` set to the size needed. Host memory only; runs on the host
 * (the boolean coder is a serial chain) with one thread per token
 * partition, and needs no context. */
vp8a_status vp8a_write_inter_frame(const vp8a_frame_header* header,
                                   const vp8a_mb_decision* decisions, const int16_t* coeffs,
                                   const int8_t* mb_segment, const uint8_t* token_prob_updates,
                                   uint8_t* out, uint64_t out_capacity, uint64_t* out_size);

#ifdef __cplusplus
}
#endif

#endif /* VP8A_H */
