"""Python mirror of the reference's encoder-analysis entry points.

Each function keeps the name and argument meaning of the oxideav-vp8
function it replaces (cited) and calls the matching C-ABI entry point of
libvp8a.so, which runs CUDA kernels on the context's GPU. Inputs may be
numpy arrays (host) or torch CUDA tensors (device); outputs are numpy unless
an `out=` buffer is given. Errors raise Vp8aError carrying the vp8a_status,
the counterpart of the reference's EncodeError.
"""
import ctypes as C

import numpy as np

from . import abi
from .frames import i420, luma_ref, planes, ptr, source
from .lib import check, load


class Context:
    """One GPU + one CUDA stream (vp8a_ctx_create)."""

    def __init__(self, device=0):
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.vp8a_ctx_create(device, C.byref(h)), "vp8a_ctx_create")
        self.handle = h.value
        self.device = device

    def close(self):
        if self.handle:
            self._lib.vp8a_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self):
        return self._lib.vp8a_ctx_stream(self.handle)

    @property
    def launches(self):
        return int(self._lib.vp8a_ctx_launch_count(self.handle))

    def synchronize(self):
        check(self._lib.vp8a_ctx_synchronize(self.handle), "vp8a_ctx_synchronize")

    def set_trellis_strength(self, strength):
        """TrellisStrength of this context's reconstructions (0 = plain rounding)."""
        check(self._lib.vp8a_ctx_set_trellis_strength(self.handle, float(strength)), "vp8a_ctx_set_trellis_strength")

    def set_subpel_planes(self, on):
        """Precomputed sub-pel planes for the analysis refinements (default on)."""
        check(self._lib.vp8a_ctx_set_subpel_planes(self.handle, int(bool(on))), "vp8a_ctx_set_subpel_planes")

    def set_autotune(self, on):
        """Measured (True, the default) or modelled launch shapes."""
        check(self._lib.vp8a_ctx_set_autotune(self.handle, int(bool(on))), "vp8a_ctx_set_autotune")

    def force_sweep_layout(self, passes, threads=0, prefetch=0):
        """Force the loop-filter sweep's launch shape (passes 0 = automatic)."""
        check(self._lib.vp8a_ctx_force_sweep_layout(self.handle, passes, threads, prefetch),
              "vp8a_ctx_force_sweep_layout")

    def last_sweep_layout(self):
        """(passes per CTA, threads per CTA, prefetch, CTAs per SM) of the last sweep."""
        out = (C.c_uint32 * 4)()
        check(self._lib.vp8a_ctx_last_sweep_layout(self.handle, out), "vp8a_ctx_last_sweep_layout")
        return tuple(int(x) for x in out)

    def set_wait_limit(self, polls):
        """Poll budget of the analysis wavefront waits (default 2**24)."""
        check(self._lib.vp8a_ctx_set_wait_limit(self.handle, int(polls)), "vp8a_ctx_set_wait_limit")


def _mvs(a):
    a = np.ascontiguousarray(a)
    if a.dtype != abi.MV_DTYPE:
        a = np.ascontiguousarray(a.astype(np.int16).reshape(-1, 2)).view(abi.MV_DTYPE).reshape(-1)
    return a


def _xy(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32).reshape(-1, 2))


def _src(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint8).reshape(-1, 256))
    return a


def mb_luma_sad_at_mv(ctx, ref_plane, src_mbs, mb_xy, mvs, width=None, height=None):
    """mb_luma_sad_at_mv (src/motion_search.rs:470) over a batch."""
    r = luma_ref(ref_plane, width, height)
    src, xy, mv = _src(src_mbs), _xy(mb_xy), _mvs(mvs)
    n = len(mv)
    out = np.zeros(n, np.uint32)
    check(ctx._lib.vp8a_mb_luma_sad_at_mv(ctx.handle, C.byref(r), ptr(src), ptr(xy), ptr(mv), n, ptr(out)),
          "vp8a_mb_luma_sad_at_mv")
    return out


def small_diamond_search_luma(ctx, ref_plane, src_mbs, mb_xy, centers, max_iters, width=None, height=None):
    """small_diamond_search_luma (src/motion_search.rs:381) over a batch."""
    r = luma_ref(ref_plane, width, height)
    src, xy, c = _src(src_mbs), _xy(mb_xy), _mvs(centers)
    out = np.zeros(len(c), abi.SEARCH_RESULT_DTYPE)
    check(ctx._lib.vp8a_small_diamond_search_luma(ctx.handle, C.byref(r), ptr(src), ptr(xy), ptr(c), max_iters,
                                                  len(c), ptr(out)), "vp8a_small_diamond_search_luma")
    return out


def half_pixel_refine_luma(ctx, ref_plane, src_mbs, mb_xy, centers, width=None, height=None):
    """half_pixel_refine_luma (src/motion_search.rs:564) over a batch."""
    r = luma_ref(ref_plane, width, height)
    src, xy, c = _src(src_mbs), _xy(mb_xy), _mvs(centers)
    out = np.zeros(len(c), abi.SEARCH_RESULT_DTYPE)
    check(ctx._lib.vp8a_half_pixel_refine_luma(ctx.handle, C.byref(r), ptr(src), ptr(xy), ptr(c), len(c), ptr(out)),
          "vp8a_half_pixel_refine_luma")
    return out


def quarter_pixel_refine_luma(ctx, ref_plane, src_mbs, mb_xy, centers, width=None, height=None):
    """quarter_pixel_refine_luma (src/motion_search.rs:666) over a batch."""
    r = luma_ref(ref_plane, width, height)
    src, xy, c = _src(src_mbs), _xy(mb_xy), _mvs(centers)
    out = np.zeros(len(c), abi.SEARCH_RESULT_DTYPE)
    check(ctx._lib.vp8a_quarter_pixel_refine_luma(ctx.handle, C.byref(r), ptr(src), ptr(xy), ptr(c), len(c),
                                                  ptr(out)), "vp8a_quarter_pixel_refine_luma")
    return out


def motion_descent(ctx, ref_plane, src_mbs, mb_xy, centers, max_iters=8, width=None, height=None):
    """Diamond -> half -> quarter as pick_mb_for_ref runs it
    (src/encoder.rs:8576-8596). Returns (whole, half, quarter)."""
    r = luma_ref(ref_plane, width, height)
    src, xy, c = _src(src_mbs), _xy(mb_xy), _mvs(centers)
    n = len(c)
    w, h, q = (np.zeros(n, abi.SEARCH_RESULT_DTYPE) for _ in range(3))
    check(ctx._lib.vp8a_motion_descent(ctx.handle, C.byref(r), ptr(src), ptr(xy), ptr(c), max_iters, n, ptr(w),
                                       ptr(h), ptr(q)), "vp8a_motion_descent")
    return w, h, q


def rd_lambda(y_ac_qi):
    """rd_lambda (src/encoder.rs:3742) for a luma AC quantiser index."""
    return load().vp8a_rd_lambda(y_ac_qi)


def analyse_inter_frame(ctx, frame, refs, ref_ids, lam, mv_contexts=None, trace=False, proposals=None):
    """The exhaustive inter analysis (analyse_inter_frame,
    src/encoder/inter.rs:263, intra picking off). `frame` = (y, u, v)
    visible planes; `refs` = list of MB-padded (y, u, v). Returns the
    decisions as a (mb_rows, mb_cols) structured array (and the per-ref
    search trace when `trace`). `proposals` (optional: n_refs MV_DTYPE
    vectors per MB, raster order, numpy or a device tensor) adds each as a
    second NEWMV candidate (vp8a_analyse_inter_frame_proposals)."""
    f = i420(*frame)
    prs = [planes(*p) for p in refs]
    parr = (abi.Planes * len(prs))(*prs)
    ids = np.ascontiguousarray(np.asarray(ref_ids, np.uint8))
    mbr, mbc = (f.height + 15) // 16, (f.width + 15) // 16
    dec = np.zeros(mbr * mbc, abi.MB_DECISION_DTYPE)
    tr = np.zeros(mbr * mbc * len(prs), abi.REF_SEARCH_DTYPE) if trace else None
    ctxs = mv_contexts if mv_contexts is not None else abi.default_mv_contexts()
    if proposals is None:
        check(ctx._lib.vp8a_analyse_inter_frame(ctx.handle, C.byref(f), C.cast(parr, C.c_void_p), ptr(ids), len(prs),
                                                C.byref(ctxs), lam, ptr(dec), ptr(tr)), "vp8a_analyse_inter_frame")
    else:
        pr = proposals if hasattr(proposals, "data_ptr") else np.ascontiguousarray(proposals, abi.MV_DTYPE)
        check(ctx._lib.vp8a_analyse_inter_frame_proposals(ctx.handle, C.byref(f), C.cast(parr, C.c_void_p), ptr(ids),
                                                          len(prs), C.byref(ctxs), lam, ptr(pr), ptr(dec), ptr(tr)),
              "vp8a_analyse_inter_frame_proposals")
    dec = dec.reshape(mbr, mbc)
    if trace:
        return dec, tr.reshape(mbr, mbc, len(prs))
    return dec


def rd_inter_search(ctx, frame, refs, ref_ids, lam, y1_ac, effort, neighbours, mv_contexts=None):
    """decide_mb_rd's inter search (src/encoder/inter_search.rs:846-1060)
    for every MB given its census neighbours (3 vp8a_mb_info records per MB:
    above, left, above-left). Returns a (mb_rows, mb_cols) RD_INTER_DTYPE
    array."""
    f = i420(*frame)
    prs = [planes(*p) for p in refs]
    parr = (abi.Planes * len(prs))(*prs)
    ids = np.ascontiguousarray(np.asarray(ref_ids, np.uint8))
    nb = np.ascontiguousarray(neighbours, abi.MB_INFO_DTYPE)
    mbr, mbc = (f.height + 15) // 16, (f.width + 15) // 16
    out = np.zeros(mbr * mbc, abi.RD_INTER_DTYPE)
    ctxs = mv_contexts if mv_contexts is not None else abi.default_mv_contexts()
    check(ctx._lib.vp8a_rd_inter_search(ctx.handle, C.byref(f), C.cast(parr, C.c_void_p), ptr(ids), len(prs),
                                        C.byref(ctxs), lam, y1_ac, effort, ptr(nb), ptr(out)), "vp8a_rd_inter_search")
    return out.reshape(mbr, mbc)


def neighbours_from_decisions(dec):
    """The (above, left, above-left) census records of every MB, built from
    a frame's decisions the way analyse_row forwards them
    (src/encoder/inter.rs:458-480); border slots are intra records."""
    d = np.asarray(dec)
    mbr, mbc = d.shape
    info = np.zeros((mbr + 1, mbc + 1), abi.MB_INFO_DTYPE)
    inner = info[1:, 1:]
    inner["ref_frame"] = d["ref_frame"]
    inner["mv"] = d["mv"]
    split = d["mode"] == abi.MODE_SPLIT
    inner["is_split"] = split
    inner["has_split_mvs"] = split
    inner["split_mvs"] = np.where(split[..., None], d["split_mvs"], np.zeros_like(d["split_mvs"]))
    nb = np.zeros((mbr, mbc, 3), abi.MB_INFO_DTYPE)
    nb[:, :, 0] = info[:-1, 1:]
    nb[:, :, 1] = info[1:, :-1]
    nb[:, :, 2] = info[:-1, :-1]
    return np.ascontiguousarray(nb.reshape(-1))


def filter_set_for_version(version):
    """filter_set_for_version (src/motion_comp.rs:370): version 0 selects
    the six-tap set, any other version the bilinear set."""
    return abi.FILTER_SIXTAP if version == 0 else abi.FILTER_BILINEAR


def _contig(a):
    return a if hasattr(a, "data_ptr") else np.ascontiguousarray(a)


def predict_inter_mb(ctx, ref, mb_xy, mvs, full_pixel=False, filter_set=abi.FILTER_SIXTAP, out=None):
    """predict_inter_mb (src/motion_comp.rs:1986) over a batch: item i is the
    MB at mb_xy[i] = (mb_col, mb_row) under the quarter-pel vector mvs[i].
    `ref` = MB-padded (y, u, v). Returns (n, 384) uint8 ReconstructedMb
    records: y[256], u[64], v[64] in raster order."""
    p = planes(*ref)
    xy, mv = _xy(mb_xy), _mvs(mvs)
    n = len(mv)
    o = np.zeros((n, 384), np.uint8) if out is None else out
    check(ctx._lib.vp8a_predict_inter_mb(ctx.handle, C.byref(p), ptr(xy), ptr(mv), n, int(bool(full_pixel)),
                                         filter_set, ptr(o)), "vp8a_predict_inter_mb")
    return o


def predict_split_mv(ctx, ref, mb_xy, split_mvs, full_pixel=False, filter_set=abi.FILTER_SIXTAP, out=None):
    """predict_split_mv (src/motion_comp.rs:2228) over a batch: 16
    quarter-pel vectors per item (raster sub-block order)."""
    p = planes(*ref)
    xy, mv = _xy(mb_xy), _mvs(split_mvs)
    n = len(mv) // 16
    assert len(mv) == 16 * n and len(xy) == n, "need 16 vectors and one position per MB"
    o = np.zeros((n, 384), np.uint8) if out is None else out
    check(ctx._lib.vp8a_predict_split_mv(ctx.handle, C.byref(p), ptr(xy), ptr(mv), n, int(bool(full_pixel)),
                                         filter_set, ptr(o)), "vp8a_predict_split_mv")
    return o


def predict_inter_frame(ctx, refs, ref_ids, decisions, out, full_pixel=False, filter_set=abi.FILTER_SIXTAP):
    """The prediction pick_mb_for_ref builds for each MB's chosen mode
    (src/encoder.rs:8704-8735), written into the MB-padded planes `out` =
    (y, u, v) in place; MBs without an inter reference keep their pixels.
    `decisions` is vp8a_analyse_inter_frame's output (any shape, raster
    order). Returns `out`."""
    prs = [planes(*p) for p in refs]
    parr = (abi.Planes * len(prs))(*prs)
    ids = np.ascontiguousarray(np.asarray(ref_ids, np.uint8))
    dec = _contig(decisions)
    op = planes(*out)
    check(ctx._lib.vp8a_predict_inter_frame(ctx.handle, C.cast(parr, C.c_void_p), ptr(ids), len(prs), ptr(dec),
                                            int(bool(full_pixel)), filter_set, C.byref(op)),
          "vp8a_predict_inter_frame")
    return out


def dequant_factors(quant, segment_quant=None, absolute=False):
    """MbDequantFactors::from_quant_indices / for_segment (src/dequant.rs:169,
    :201): (y1_dc, y1_ac, y2_dc, y2_ac, uv_dc, uv_ac)."""
    out = np.zeros(6, np.int16)
    load().vp8a_dequant_factors(C.byref(quant), segment_quant is not None, segment_quant or 0, int(bool(absolute)),
                                ptr(out))
    return tuple(int(x) for x in out)


def write_inter_frame(header, decisions, coeffs, mb_segment=None, token_prob_updates=None):
    """The inter-frame bitstream of encode_p_frame_multi_ref_inner_driven
    (src/encoder.rs:11214-11720) as bytes: `header` an abi.FrameHeader,
    `decisions` the analysis's MB_DECISION_DTYPE records (raster order),
    `coeffs` (n_mbs, 400) int16 quantised coefficients as
    reconstruct_inter_frame returns them, `mb_segment` one int8 per MB when
    the header enables segmentation, `token_prob_updates` None or 1056
    probabilities in [4][8][3][11] order (0 = keep the default). Host
    memory; no context needed."""
    lib = load()
    dec = np.ascontiguousarray(decisions).reshape(-1)
    cf = np.ascontiguousarray(coeffs, np.int16)
    if cf.size != dec.size * 400:
        raise ValueError("coeffs must hold 400 int16 per MB")
    seg = None if mb_segment is None else np.ascontiguousarray(np.asarray(mb_segment, np.int8).reshape(-1))
    upd = None
    if token_prob_updates is not None:
        upd = np.ascontiguousarray(np.asarray(token_prob_updates, np.uint8).reshape(-1))
        if upd.size != 1056:
            raise ValueError("token_prob_updates must hold 1056 entries")
    size = C.c_uint64(0)
    cap = 1024 + 600 * dec.size
    while True:
        out = np.zeros(cap, np.uint8)
        st = lib.vp8a_write_inter_frame(C.byref(header), ptr(dec), ptr(cf), ptr(seg), ptr(upd), ptr(out), cap,
                                        C.byref(size))
        if st == abi.E_INVALID_ARGUMENT and size.value > cap:
            cap = size.value
            continue
        check(st, "vp8a_write_inter_frame")
        return out[:size.value].tobytes()


def encode_p_frame(ctx, frame, refs, ref_ids, y_ac_qi, loop_filter_level=0, sharpness_level=0, simple=False,
                   n_partitions=1, auto_lf=True, refresh_last=True, proposals=None):
    """encode_p_frame_multi_ref_auto_loop_filter (src/encoder.rs:9373) with
    intra picking off and the trellis off: the exhaustive analysis, the §14
    reconstruction of the chosen modes, the §9.4 (level, sharpness) search
    (select_filter_params, when `auto_lf`), the §15 filter pass and the
    bitstream. `frame` = visible (y, u, v); `refs` = MB-padded (y, u, v)
    with ids `ref_ids` (VP8A_REF_*). Returns (frame bytes, the filtered
    reconstruction as MB-padded (y, u, v), details dict with the decisions,
    coefficients, flags, the loop-filter records and the chosen level and
    sharpness). `proposals` (optional) are second NEWMV candidates for the
    analysis (vp8a_analyse_inter_frame_proposals)."""
    dec = analyse_inter_frame(ctx, frame, refs, ref_ids, rd_lambda(y_ac_qi), proposals=proposals).reshape(-1)
    quant = abi.quant_indices(y_ac_qi)
    recon = tuple(np.zeros_like(p) for p in refs[0])
    lf = np.zeros(dec.size, abi.MB_LF_INFO_DTYPE)
    cf, fl = reconstruct_inter_frame(ctx, frame, refs, ref_ids, dec, quant, recon, lf_info=lf)
    level, sharp = loop_filter_level, sharpness_level
    if auto_lf:
        base = abi.filter_config(level=0, sharpness=sharpness_level, simple=simple)
        level, sharp = select_filter_params(ctx, recon, lf, base, frame)
    cfg = abi.filter_config(level=level, sharpness=sharp, simple=simple)
    out = filter_frame(ctx, recon, lf, cfg) if level else recon
    hdr = abi.frame_header(frame[0].shape[1], frame[0].shape[0], quant, n_partitions=n_partitions,
                           refresh_last=refresh_last, filter_type=int(simple), loop_filter_level=level,
                           sharpness_level=sharp)
    bits = write_inter_frame(hdr, dec, cf)
    return bits, out, dict(decisions=dec, coeffs=cf, flags=fl, lf_info=lf, recon=recon, level=level,
                           sharpness=sharp)


def reconstruct_inter_frame(ctx, frame, refs, ref_ids, decisions, quant, recon, mb_segment=None,
                            segment_quant=None, segment_abs=False, full_pixel=False, filter_set=abi.FILTER_SIXTAP,
                            coeffs=True, flags=True, lf_info=None):
    """pick_mb_for_ref's §18 prediction + §14 transform / quantise /
    reconstruct for every MB's chosen mode with the trellis off
    (src/encoder.rs:8704-8800). `frame` = visible (y, u, v); `recon` =
    MB-padded (y, u, v) written in place; `quant` an abi.QuantIndices.
    Returns (coeffs (n_mbs, 400) int16 in MbCoeffs order or None,
    flags (n_mbs,) uint8 of abi.MB_SKIP | abi.MB_HAS_COEFFS or None);
    `lf_info` (optional MB_LF_INFO_DTYPE buffer) receives each inter MB's
    §15 side information for the loop-filter calls."""
    f = i420(*frame)
    prs = [planes(*p) for p in refs]
    parr = (abi.Planes * len(prs))(*prs)
    ids = np.ascontiguousarray(np.asarray(ref_ids, np.uint8))
    dec = _contig(decisions)
    op = planes(*recon)
    n = op.mb_cols * op.mb_rows
    cf = np.zeros((n, 400), np.int16) if coeffs is True else coeffs
    fl = np.zeros(n, np.uint8) if flags is True else flags
    seg = None if mb_segment is None else _contig(mb_segment if hasattr(mb_segment, "data_ptr")
                                                  else np.asarray(mb_segment, np.int8))
    sq = None if segment_quant is None else np.ascontiguousarray(np.asarray(segment_quant, np.int16).reshape(4))
    check(ctx._lib.vp8a_reconstruct_inter_frame(ctx.handle, C.byref(f), C.cast(parr, C.c_void_p), ptr(ids), len(prs),
                                                ptr(dec), C.byref(quant), ptr(seg), ptr(sq), int(bool(segment_abs)),
                                                int(bool(full_pixel)), filter_set, C.byref(op), ptr(cf), ptr(fl),
                                                ptr(lf_info)),
          "vp8a_reconstruct_inter_frame")
    return cf, fl


def build_arnr_altref(ctx, frames, center, strength=3):
    """build_arnr_altref (src/arnr.rs:476). `frames` = list of (y, u, v).
    Returns the packed (y, u, v) anchor."""
    recs = [i420(*f) for f in frames]
    arr = (abi.I420 * len(recs))(*recs)
    # Output size follows the centre frame; an out-of-range centre is
    # rejected by the library (VP8A_E_INVALID_ARGUMENT).
    shape_src = frames[center] if 0 <= center < len(frames) else frames[0]
    h, w = shape_src[0].shape[0], shape_src[0].shape[1]
    ch, cw = (h + 1) // 2, (w + 1) // 2
    y = np.zeros((h, w), np.uint8)
    u = np.zeros((ch, cw), np.uint8)
    v = np.zeros((ch, cw), np.uint8)
    check(ctx._lib.vp8a_build_arnr_altref(ctx.handle, C.cast(arr, C.c_void_p), len(recs), center, strength, ptr(y),
                                          ptr(u), ptr(v)), "vp8a_build_arnr_altref")
    return y, u, v


def build_arnr_altref_planes(ctx, frames, center, strength=3, out=None):
    """build_arnr_altref (src/arnr.rs:476) into MB-padded planes
    (vp8a_build_arnr_altref_planes): the anchor with its padding
    edge-replicated, the layout of a reference. `out` = MB-padded (y, u, v)
    to write (numpy or torch CUDA), else new numpy planes. Returns `out`."""
    recs = [i420(*f) for f in frames]
    arr = (abi.I420 * len(recs))(*recs)
    shape_src = frames[center] if 0 <= center < len(frames) else frames[0]
    h, w = shape_src[0].shape[0], shape_src[0].shape[1]
    if out is None:
        mbr, mbc = (h + 15) // 16, (w + 15) // 16
        out = (np.zeros((mbr * 16, mbc * 16), np.uint8), np.zeros((mbr * 8, mbc * 8), np.uint8),
               np.zeros((mbr * 8, mbc * 8), np.uint8))
    p = planes(*out)
    check(ctx._lib.vp8a_build_arnr_altref_planes(ctx.handle, C.cast(arr, C.c_void_p), len(recs), center, strength,
                                                 C.byref(p)), "vp8a_build_arnr_altref_planes")
    return out


def filter_frame(ctx, recon, mbs, config):
    """filter_inter_frame_flags / filter_frame_flags
    (src/loop_filter.rs:1364, :2506) on a copy of `recon` (MB-padded
    (y, u, v)); returns the filtered planes."""
    y, u, v = (np.array(p, np.uint8, copy=True) for p in recon)
    p = planes(y, u, v)
    m = np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
    check(ctx._lib.vp8a_filter_frame(ctx.handle, C.byref(p), ptr(m), C.byref(config)), "vp8a_filter_frame")
    return y, u, v


def reconstruction_ssd(ctx, recon, src):
    """reconstruction_ssd (src/loop_filter.rs:1965)."""
    p, s = planes(*recon), source(*src)
    out = np.zeros(1, np.uint64)
    check(ctx._lib.vp8a_reconstruction_ssd(ctx.handle, C.byref(p), C.byref(s), ptr(out)), "vp8a_reconstruction_ssd")
    return int(out[0])


def filter_sweep(ctx, recon, mbs, base, src, every_rows=0):
    """score_filter_candidate (src/loop_filter.rs:2062) for every (level,
    sharpness); returns a (64, 8) uint64 table."""
    p, s = planes(*recon), source(*src)
    m = np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
    out = np.zeros(512, np.uint64)
    check(ctx._lib.vp8a_filter_sweep(ctx.handle, C.byref(p), ptr(m), C.byref(base), C.byref(s), every_rows,
                                     ptr(out)), "vp8a_filter_sweep")
    return out.reshape(64, 8)


def filter_sweep_window(ctx, recon, mbs, base, src, lo_level, hi_level):
    """vp8a_filter_sweep_window: the sweep table for level 0 and levels
    lo..hi only (UINT64_MAX elsewhere); a (64, 8) uint64 table."""
    p, s = planes(*recon), source(*src)
    m = np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
    out = np.zeros(512, np.uint64)
    check(ctx._lib.vp8a_filter_sweep_window(ctx.handle, C.byref(p), ptr(m), C.byref(base), C.byref(s), lo_level,
                                            hi_level, ptr(out)), "vp8a_filter_sweep_window")
    return out.reshape(64, 8)


def select_filter_params(ctx, recon, mbs, base, src):
    """select_filter_params (src/loop_filter.rs:2047) -> (level, sharpness)."""
    p, s = planes(*recon), source(*src)
    m = np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
    lv, sh = C.c_uint8(), C.c_uint8()
    check(ctx._lib.vp8a_select_filter_params(ctx.handle, C.byref(p), ptr(m), C.byref(base), C.byref(s),
                                             C.byref(lv), C.byref(sh)), "vp8a_select_filter_params")
    return lv.value, sh.value


def select_filter_params_sampled(ctx, recon, mbs, base, src, every_rows, sweep_sharpness):
    """select_filter_params_sampled (src/loop_filter.rs:2288)."""
    p, s = planes(*recon), source(*src)
    m = np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
    lv, sh = C.c_uint8(), C.c_uint8()
    check(ctx._lib.vp8a_select_filter_params_sampled(ctx.handle, C.byref(p), ptr(m), C.byref(base), C.byref(s),
                                                     every_rows, int(bool(sweep_sharpness)), C.byref(lv),
                                                     C.byref(sh)), "vp8a_select_filter_params_sampled")
    return lv.value, sh.value


def key_frame_sampling(mb_rows):
    """FilterSampling::for_key_frame (src/loop_filter.rs:2266) ->
    (every_rows, sweep_sharpness), from the library's own helper."""
    er, sw = C.c_uint32(), C.c_uint32()
    load().vp8a_key_frame_sampling(int(mb_rows), C.byref(er), C.byref(sw))
    return er.value, bool(sw.value)


def select_filter_params_key_frame(ctx, recon, mbs, base, src, sampled=True):
    """The key-frame encoder's loop-filter pick (src/encoder.rs:6638-6655):
    the sampled search with FilterSampling::for_key_frame, or the full
    search. `base` is the key frame's FrameFilterConfig (key_frame set)
    and `mbs` its intra MB side information."""
    if not sampled:
        return select_filter_params(ctx, recon, mbs, base, src)
    er, sw = key_frame_sampling(recon[0].shape[0] // 16)
    return select_filter_params_sampled(ctx, recon, mbs, base, src, er, sw)


def lf_info_from_decisions(dec, has_coeffs=None):
    """Per-MB §15 side information from inter decisions: SPLITMV MBs are
    recorded as B_PRED (src/loop_filter.rs:1258-1266)."""
    d = np.asarray(dec).reshape(-1)
    m = np.zeros(len(d), abi.MB_LF_INFO_DTYPE)
    m["ref_frame"] = d["ref_frame"]
    m["inter_mode"] = d["mode"]
    m["y_mode_is_bpred"] = (d["mode"] == abi.MODE_SPLIT).astype(np.uint8)
    m["segment_id"] = -1
    if has_coeffs is not None:
        m["has_coeffs"] = np.asarray(has_coeffs, np.uint8).reshape(-1)
    return m


# ------------------------------------------------------ batched work lists
#
# Each *_frames / *_altrefs / *_sweeps call runs a list of independent jobs
# (many streams' frames, of uneven sizes) as one launch per stage; every
# job's results equal the single-job call's.


def _batch(ctx, fn, jobs, where):
    arr = (type(jobs[0]) * len(jobs))(*jobs) if jobs else None
    check(getattr(ctx._lib, fn)(ctx.handle, C.cast(arr, C.c_void_p) if arr is not None else None, len(jobs)), where)


def analyse_inter_frames(ctx, jobs):
    """vp8a_analyse_inter_frames: `jobs` = list of dicts with the arguments
    of analyse_inter_frame (frame, refs, ref_ids, lam, optional
    mv_contexts, optional proposals: n_refs MV_DTYPE vectors per MB, numpy
    or a device tensor; any job with proposals makes the call
    vp8a_analyse_inter_frames_proposals). Returns each job's (mb_rows,
    mb_cols) decisions."""
    keep, cj, outs, props = [], [], [], []
    for j in jobs:
        f = i420(*j["frame"])
        prs = [planes(*p) for p in j["refs"]]
        parr = (abi.Planes * len(prs))(*prs)
        ids = np.ascontiguousarray(np.asarray(j["ref_ids"], np.uint8))
        ctxs = j.get("mv_contexts") or abi.default_mv_contexts()
        mbr, mbc = (f.height + 15) // 16, (f.width + 15) // 16
        dec = np.zeros(mbr * mbc, abi.MB_DECISION_DTYPE)
        keep += [parr, ids, ctxs]
        cj.append(abi.AnalysisJob(f, C.cast(parr, C.c_void_p), ptr(ids), len(prs), C.cast(C.pointer(ctxs), C.c_void_p),
                                  j["lam"], ptr(dec), None))
        outs.append(dec.reshape(mbr, mbc))
        pr = j.get("proposals")
        if pr is not None and not hasattr(pr, "data_ptr"):
            pr = np.ascontiguousarray(pr, abi.MV_DTYPE)
        keep.append(pr)
        props.append(None if pr is None else (pr.data_ptr() if hasattr(pr, "data_ptr") else pr.ctypes.data))
    if any(p is not None for p in props):
        arr = (abi.AnalysisJob * len(cj))(*cj)
        parr_ = (C.c_void_p * len(props))(*props)
        check(ctx._lib.vp8a_analyse_inter_frames_proposals(ctx.handle, C.cast(arr, C.c_void_p), len(cj),
                                                           C.cast(parr_, C.c_void_p)),
              "vp8a_analyse_inter_frames_proposals")
    else:
        _batch(ctx, "vp8a_analyse_inter_frames", cj, "vp8a_analyse_inter_frames")
    return outs


def build_arnr_altrefs(ctx, jobs):
    """vp8a_build_arnr_altrefs: `jobs` = list of (frames, center, strength)
    with frames a list of (y, u, v). Returns each job's packed (y, u, v)."""
    keep, cj, outs = [], [], []
    for frames, center, strength in jobs:
        recs = [i420(*f) for f in frames]
        arr = (abi.I420 * len(recs))(*recs)
        h, w = frames[0][0].shape[:2]
        ch, cw = (h + 1) // 2, (w + 1) // 2
        y, u, v = np.zeros((h, w), np.uint8), np.zeros((ch, cw), np.uint8), np.zeros((ch, cw), np.uint8)
        keep.append(arr)
        cj.append(abi.ArnrJob(C.cast(arr, C.c_void_p), len(recs), center, strength, ptr(y), ptr(u), ptr(v)))
        outs.append((y, u, v))
    _batch(ctx, "vp8a_build_arnr_altrefs", cj, "vp8a_build_arnr_altrefs")
    return outs


def build_arnr_altrefs_planes(ctx, jobs):
    """vp8a_build_arnr_altrefs_planes: `jobs` = list of (frames, center,
    strength). Returns each job's MB-padded (y, u, v) anchor."""
    keep, cj, outs = [], [], []
    for frames, center, strength in jobs:
        recs = [i420(*f) for f in frames]
        arr = (abi.I420 * len(recs))(*recs)
        h, w = frames[0][0].shape[:2]
        mbr, mbc = (h + 15) // 16, (w + 15) // 16
        out = (np.zeros((mbr * 16, mbc * 16), np.uint8), np.zeros((mbr * 8, mbc * 8), np.uint8),
               np.zeros((mbr * 8, mbc * 8), np.uint8))
        keep.append(arr)
        cj.append(abi.ArnrPlanesJob(C.cast(arr, C.c_void_p), len(recs), center, strength, planes(*out)))
        outs.append(out)
    _batch(ctx, "vp8a_build_arnr_altrefs_planes", cj, "vp8a_build_arnr_altrefs_planes")
    return outs


def reconstruct_inter_frames(ctx, jobs):
    """vp8a_reconstruct_inter_frames: `jobs` = list of dicts with the
    arguments of reconstruct_inter_frame (frame, refs, ref_ids, decisions,
    quant, recon, optional mb_segment, segment_quant, segment_abs,
    full_pixel, filter_set, lf_info). `recon` is written in place. Returns
    each job's (coeffs, flags)."""
    keep, cj, outs = [], [], []
    for j in jobs:
        f = i420(*j["frame"])
        prs = [planes(*p) for p in j["refs"]]
        parr = (abi.Planes * len(prs))(*prs)
        ids = np.ascontiguousarray(np.asarray(j["ref_ids"], np.uint8))
        dec = _contig(j["decisions"])
        op = planes(*j["recon"])
        n = op.mb_cols * op.mb_rows
        cf, fl = np.zeros((n, 400), np.int16), np.zeros(n, np.uint8)
        seg = j.get("mb_segment")
        seg = None if seg is None else np.ascontiguousarray(np.asarray(seg, np.int8))
        sq = j.get("segment_quant")
        sq = None if sq is None else np.ascontiguousarray(np.asarray(sq, np.int16).reshape(4))
        keep += [parr, ids, dec, seg, sq]
        cj.append(abi.ReconJob(f, C.cast(parr, C.c_void_p), ptr(ids), len(prs), int(bool(j.get("segment_abs"))),
                               ptr(dec), j["quant"], ptr(seg), ptr(sq), int(bool(j.get("full_pixel"))),
                               j.get("filter_set", abi.FILTER_SIXTAP), op, ptr(cf), ptr(fl), ptr(j.get("lf_info"))))
        outs.append((cf, fl))
    _batch(ctx, "vp8a_reconstruct_inter_frames", cj, "vp8a_reconstruct_inter_frames")
    return outs


def filter_sweeps(ctx, jobs):
    """vp8a_filter_sweeps: `jobs` = list of (recon, mbs, base, src[,
    every_rows]). Returns each job's (64, 8) uint64 table."""
    keep, cj, outs = [], [], []
    for j in jobs:
        recon, mbs, base, src = j[:4]
        every = j[4] if len(j) > 4 else 0
        m = np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
        out = np.zeros(512, np.uint64)
        keep.append(m)
        cj.append(abi.SweepJob(planes(*recon), ptr(m), base, source(*src), every, ptr(out)))
        outs.append(out.reshape(64, 8))
    _batch(ctx, "vp8a_filter_sweeps", cj, "vp8a_filter_sweeps")
    return outs


def select_filter_params_batch(ctx, jobs):
    """vp8a_select_filter_params_batch: select_filter_params
    (src/loop_filter.rs:2047) for every job of `jobs` = list of (recon, mbs,
    base, src); each stage of the walk runs all jobs in one launch. Returns
    each job's (level, sharpness)."""
    keep, cj = [], []
    for recon, mbs, base, src in jobs:
        m = mbs if hasattr(mbs, "data_ptr") else np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
        keep.append(m)
        cj.append(abi.SweepJob(planes(*recon), ptr(m), base, source(*src), 0, None))
    arr = (abi.SweepJob * len(cj))(*cj)
    lv = np.zeros(len(cj), np.uint8)
    sh = np.zeros(len(cj), np.uint8)
    check(ctx._lib.vp8a_select_filter_params_batch(ctx.handle, C.cast(arr, C.c_void_p), len(cj), ptr(lv), ptr(sh)),
          "vp8a_select_filter_params_batch")
    return [(int(a), int(b)) for a, b in zip(lv, sh)]
