"""Python face of the oracle (liboracle.so) — TEST INFRASTRUCTURE ONLY.

The oracle is the CPU restatement of the reference's encoder-analysis path
(see vp8a_oracle.h). Only tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py use it, as the checker or as the
timed CPU baseline; the product (libvp8a.so, package vp8a) never loads it.

Function names and argument meanings match the product API in vp8a.api
(without the GPU context), so a parity test calls both the same way.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG_DIR = os.path.join(ROOT, "oxideav-vp8_b200")
if PKG_DIR not in sys.path:
    sys.path.insert(0, PKG_DIR)

from vp8a import abi  # noqa: E402  (ABI record layouts only)
from vp8a.frames import i420, luma_ref, planes, ptr, source  # noqa: E402

LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None
P = C.c_void_p
U32 = C.c_uint32


def build(force=False):
    """Compile liboracle.so with the Makefile beside this file."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "-B" if force else "liboracle.so"], check=True, capture_output=True)
    else:
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    sig = {
        "vo_block_sad_16x16": (U32, [P, P]),
        "vo_mb_luma_sad_at_mv_batch": (None, [C.POINTER(abi.LumaRef), P, P, P, U32, P]),
        "vo_small_diamond_batch": (None, [C.POINTER(abi.LumaRef), P, P, P, U32, U32, P]),
        "vo_half_refine_batch": (None, [C.POINTER(abi.LumaRef), P, P, P, U32, P]),
        "vo_quarter_refine_batch": (None, [C.POINTER(abi.LumaRef), P, P, P, U32, P]),
        "vo_motion_descent_batch": (None, [C.POINTER(abi.LumaRef), P, P, P, U32, U32, P, P, P, U32]),
        "vo_sixtap_mb_luma": (None, [P, C.c_int, C.c_int, P]),
        "vo_bool_bits": (C.c_double, [C.c_uint8, C.c_int]),
        "vo_mv_component_bits": (C.c_double, [P, C.c_int32]),
        "vo_rd_lambda": (C.c_double, [U32]),
        "vo_analyse_inter_frame": (C.c_int, [C.POINTER(abi.I420), P, P, U32, C.POINTER(abi.MvContexts),
                                             C.c_double, P, P, U32]),
        "vo_analyse_inter_frame_proposals": (C.c_int, [C.POINTER(abi.I420), P, P, U32, C.POINTER(abi.MvContexts),
                                                       C.c_double, P, P, P, U32]),
        "vo_build_arnr_altref": (C.c_int, [P, U32, U32, U32, P, P, P, U32]),
        "vo_lf_derive": (None, [C.c_uint8, C.c_uint8, C.c_int, P]),
        "vo_common_adjust": (C.c_int32, [C.c_int, P]),
        "vo_simple_segment": (None, [C.c_uint8, P]),
        "vo_subblock_filter": (None, [C.c_uint8, C.c_uint8, C.c_uint8, P]),
        "vo_mb_filter": (None, [C.c_uint8, C.c_uint8, C.c_uint8, P]),
        "vo_mb_filter_level": (C.c_uint8, [C.POINTER(abi.FilterConfig), P]),
        "vo_filter_frame": (C.c_int, [C.POINTER(abi.Planes), P, C.POINTER(abi.FilterConfig)]),
        "vo_reconstruction_ssd": (C.c_uint64, [C.POINTER(abi.Planes), C.POINTER(abi.Source)]),
        "vo_score_filter_candidate": (C.c_uint64, [C.POINTER(abi.Planes), P, C.POINTER(abi.FilterConfig),
                                                   C.POINTER(abi.Source), C.c_uint8, C.c_uint8, U32]),
        "vo_filter_sweep": (None, [C.POINTER(abi.Planes), P, C.POINTER(abi.FilterConfig), C.POINTER(abi.Source),
                                   U32, P, U32]),
        "vo_select_filter_params": (None, [C.POINTER(abi.Planes), P, C.POINTER(abi.FilterConfig),
                                           C.POINTER(abi.Source), P, P, U32]),
        "vo_select_filter_params_sampled": (None, [C.POINTER(abi.Planes), P, C.POINTER(abi.FilterConfig),
                                                   C.POINTER(abi.Source), U32, U32, P, P, U32]),
        "vo_select_from_table_full": (None, [P, C.c_uint8, P, P]),
        "vo_select_from_table_sampled": (None, [P, C.c_uint8, C.c_int, P, P]),
        "vo_type_size": (C.c_size_t, [C.c_int]),
        "vo_chroma_mv": (abi.Mv, [abi.Mv]),
        "vo_split_chroma_mvs": (None, [P, P]),
        "vo_sixtap_2d": (None, [P, C.c_int, C.c_int, C.c_int, P]),
        "vo_predict_inter_mb_batch": (None, [C.POINTER(abi.Planes), P, P, U32, C.c_int, C.c_int, P]),
        "vo_predict_split_mv_batch": (None, [C.POINTER(abi.Planes), P, P, U32, C.c_int, C.c_int, P]),
        "vo_predict_inter_frame": (C.c_int, [P, P, U32, P, C.c_int, C.c_int, C.POINTER(abi.Planes)]),
        "vo_dequant_factors": (None, [C.c_int32] * 6 + [P]),
        "vo_vp8_decoder_new": (P, []),
        "vo_vp8_decoder_free": (None, [P]),
        "vo_vp8_decoder_capture": (None, [P, P]),
        "vo_vp8_decoder_prime": (C.c_int, [P, U32, U32, P]),
        "vo_vp8_decode_frame": (C.c_int, [P, P, C.c_size_t, P, C.POINTER(U32), C.POINTER(U32),
                                          C.POINTER(C.c_int)]),
        "vo_segment_factors": (None, [C.POINTER(abi.QuantIndices), C.c_int, C.c_int32, C.c_int, P]),
        "vo_forward_dct_4x4": (None, [P, P]),
        "vo_forward_wht_4x4": (None, [P, P]),
        "vo_inverse_dct_4x4": (None, [P, P]),
        "vo_inverse_wht_4x4": (None, [P, P]),
        "vo_enc_quantize_block": (None, [P, C.c_int16, C.c_int16]),
        "vo_reconstruct_inter_mb": (C.c_int, [P, P, P, C.c_int, P]),
        "vo_reconstruct_inter_mb_trellis": (C.c_int, [P, P, P, C.c_int, P, C.c_double]),
        "vo_reconstruct_inter_frame": (C.c_int, [C.POINTER(abi.I420), P, P, U32, P, C.POINTER(abi.QuantIndices), P, P,
                                                 C.c_int, C.c_int, C.c_int, C.POINTER(abi.Planes), P, P, P, U32]),
        "vo_reconstruct_inter_frame_trellis": (C.c_int, [C.POINTER(abi.I420), P, P, U32, P,
                                                         C.POINTER(abi.QuantIndices), P, P, C.c_int, C.c_int, C.c_int,
                                                         C.POINTER(abi.Planes), P, P, P, C.c_double, U32]),
        "vo_trellis_quantize_block": (None, [P, C.c_int16, C.c_int16, C.c_int, C.c_int, C.c_int, C.c_double]),
        "vo_coeff_token_bits": (C.c_double, [C.c_int, C.c_int, C.c_int, C.c_int, U32]),
        "vo_eob_token_bits": (C.c_double, [C.c_int, C.c_int, C.c_int]),
        "vo_trellis_lambda": (C.c_double, [C.c_int16, C.c_double]),
        "vo_idct_basis_norm_sq": (P, []),
        "vo_rd_inter_search": (C.c_int, [C.POINTER(abi.I420), P, P, U32, C.POINTER(abi.MvContexts), C.c_double,
                                         U32, U32, P, P, U32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _mvs(a):
    a = np.ascontiguousarray(a)
    if a.dtype != abi.MV_DTYPE:
        a = np.ascontiguousarray(a.astype(np.int16).reshape(-1, 2)).view(abi.MV_DTYPE).reshape(-1)
    return a


def _xy(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32).reshape(-1, 2))


def _src(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint8).reshape(-1, 256))


def type_sizes():
    lib = load()
    names = ["vp8a_mv", "vp8a_search_result", "vp8a_luma_ref", "vp8a_i420", "vp8a_planes", "vp8a_mv_contexts",
             "vp8a_mb_decision", "vp8a_ref_search", "vp8a_mb_lf_info", "vp8a_filter_config", "vp8a_source",
             "vp8a_mb_info", "vp8a_rd_inter", "vp8a_quant_indices", "vp8a_analysis_job", "vp8a_arnr_job",
             "vp8a_recon_job", "vp8a_sweep_job", "vp8a_frame_header", "vp8a_arnr_planes_job"]
    return {n: int(lib.vo_type_size(i)) for i, n in enumerate(names)}


def block_sad_16x16(src, pred):
    s = np.ascontiguousarray(src, np.uint8)
    p = np.ascontiguousarray(pred, np.uint8)
    return int(load().vo_block_sad_16x16(ptr(s), ptr(p)))


def sixtap_mb_luma(halo441, mx, my):
    h = np.ascontiguousarray(halo441, np.uint8).reshape(-1)
    out = np.zeros(256, np.uint8)
    load().vo_sixtap_mb_luma(ptr(h), mx, my, ptr(out))
    return out.reshape(16, 16)


def mb_luma_sad_at_mv(ref_plane, src_mbs, mb_xy, mvs, width=None, height=None):
    r = luma_ref(ref_plane, width, height)
    src, xy, mv = _src(src_mbs), _xy(mb_xy), _mvs(mvs)
    out = np.zeros(len(mv), np.uint32)
    load().vo_mb_luma_sad_at_mv_batch(C.byref(r), ptr(src), ptr(xy), ptr(mv), len(mv), ptr(out))
    return out


def small_diamond_search_luma(ref_plane, src_mbs, mb_xy, centers, max_iters, width=None, height=None):
    r = luma_ref(ref_plane, width, height)
    src, xy, c = _src(src_mbs), _xy(mb_xy), _mvs(centers)
    out = np.zeros(len(c), abi.SEARCH_RESULT_DTYPE)
    load().vo_small_diamond_batch(C.byref(r), ptr(src), ptr(xy), ptr(c), max_iters, len(c), ptr(out))
    return out


def half_pixel_refine_luma(ref_plane, src_mbs, mb_xy, centers, width=None, height=None):
    r = luma_ref(ref_plane, width, height)
    src, xy, c = _src(src_mbs), _xy(mb_xy), _mvs(centers)
    out = np.zeros(len(c), abi.SEARCH_RESULT_DTYPE)
    load().vo_half_refine_batch(C.byref(r), ptr(src), ptr(xy), ptr(c), len(c), ptr(out))
    return out


def quarter_pixel_refine_luma(ref_plane, src_mbs, mb_xy, centers, width=None, height=None):
    r = luma_ref(ref_plane, width, height)
    src, xy, c = _src(src_mbs), _xy(mb_xy), _mvs(centers)
    out = np.zeros(len(c), abi.SEARCH_RESULT_DTYPE)
    load().vo_quarter_refine_batch(C.byref(r), ptr(src), ptr(xy), ptr(c), len(c), ptr(out))
    return out


def motion_descent(ref_plane, src_mbs, mb_xy, centers, max_iters=8, width=None, height=None, threads=1):
    r = luma_ref(ref_plane, width, height)
    src, xy, c = _src(src_mbs), _xy(mb_xy), _mvs(centers)
    n = len(c)
    w, h, q = (np.zeros(n, abi.SEARCH_RESULT_DTYPE) for _ in range(3))
    load().vo_motion_descent_batch(C.byref(r), ptr(src), ptr(xy), ptr(c), max_iters, n, ptr(w), ptr(h), ptr(q),
                                   threads)
    return w, h, q


def bool_bits(prob, value):
    return load().vo_bool_bits(prob, int(bool(value)))


def mv_component_bits(ctx19, value):
    p = np.ascontiguousarray(ctx19, np.uint8)
    return load().vo_mv_component_bits(ptr(p), value)


def rd_lambda(qi):
    return load().vo_rd_lambda(qi)


def _check(status, where):
    if status != 0:
        raise RuntimeError(f"{where}: {abi.STATUS_NAMES.get(status, status)}")


def analyse_inter_frame(frame, refs, ref_ids, lam, mv_contexts=None, trace=False, threads=1, proposals=None):
    """The exhaustive analysis; `proposals` (optional, (mb_rows * mb_cols,
    n_refs) MV_DTYPE) adds one proposed NEWMV vector per MB and reference."""
    f = i420(*frame)
    prs = [planes(*p) for p in refs]
    parr = (abi.Planes * len(prs))(*prs)
    ids = np.ascontiguousarray(np.asarray(ref_ids, np.uint8))
    mbr, mbc = (f.height + 15) // 16, (f.width + 15) // 16
    dec = np.zeros(mbr * mbc, abi.MB_DECISION_DTYPE)
    tr = np.zeros(mbr * mbc * len(prs), abi.REF_SEARCH_DTYPE) if trace else None
    ctxs = mv_contexts if mv_contexts is not None else abi.default_mv_contexts()
    if proposals is None:
        st = load().vo_analyse_inter_frame(C.byref(f), C.cast(parr, C.c_void_p), ptr(ids), len(prs), C.byref(ctxs),
                                           lam, ptr(dec), ptr(tr), threads)
    else:
        pr = np.ascontiguousarray(proposals, abi.MV_DTYPE).reshape(-1)
        assert pr.size == mbr * mbc * len(prs)
        st = load().vo_analyse_inter_frame_proposals(C.byref(f), C.cast(parr, C.c_void_p), ptr(ids), len(prs),
                                                     C.byref(ctxs), lam, ptr(pr), ptr(dec), ptr(tr), threads)
    _check(st, "vo_analyse_inter_frame")
    dec = dec.reshape(mbr, mbc)
    if trace:
        return dec, tr.reshape(mbr, mbc, len(prs))
    return dec


def build_arnr_altref(frames, center, strength=3, threads=1):
    recs = [i420(*f) for f in frames]
    arr = (abi.I420 * len(recs))(*recs)
    h, w = frames[center][0].shape
    ch, cw = (h + 1) // 2, (w + 1) // 2
    y = np.zeros((h, w), np.uint8)
    u = np.zeros((ch, cw), np.uint8)
    v = np.zeros((ch, cw), np.uint8)
    st = load().vo_build_arnr_altref(C.cast(arr, C.c_void_p), len(recs), center, strength, ptr(y), ptr(u), ptr(v),
                                     threads)
    _check(st, "vo_build_arnr_altref")
    return y, u, v


def lf_derive(level, sharpness, key_frame):
    out = np.zeros(4, np.uint8)
    load().vo_lf_derive(level, sharpness, int(bool(key_frame)), ptr(out))
    return tuple(int(v) for v in out)  # interior, hev, mbedge, subedge


def common_adjust(use_outer_taps, seg4):
    s = np.ascontiguousarray(seg4, np.uint8).copy()
    a = load().vo_common_adjust(int(bool(use_outer_taps)), ptr(s))
    return int(a), s


def simple_segment(edge_limit, seg4):
    s = np.ascontiguousarray(seg4, np.uint8).copy()
    load().vo_simple_segment(edge_limit, ptr(s))
    return s


def subblock_filter(hev, interior, edge, seg8):
    s = np.ascontiguousarray(seg8, np.uint8).copy()
    load().vo_subblock_filter(hev, interior, edge, ptr(s))
    return s


def mb_filter(hev, interior, edge, seg8):
    s = np.ascontiguousarray(seg8, np.uint8).copy()
    load().vo_mb_filter(hev, interior, edge, ptr(s))
    return s


def mb_filter_level(config, mb):
    m = np.ascontiguousarray(np.asarray(mb, abi.MB_LF_INFO_DTYPE).reshape(1))
    return int(load().vo_mb_filter_level(C.byref(config), ptr(m)))


def filter_frame(recon, mbs, config):
    y, u, v = (np.array(p, np.uint8, copy=True) for p in recon)
    p = planes(y, u, v)
    m = np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
    _check(load().vo_filter_frame(C.byref(p), ptr(m), C.byref(config)), "vo_filter_frame")
    return y, u, v


def reconstruction_ssd(recon, src):
    return int(load().vo_reconstruction_ssd(C.byref(planes(*recon)), C.byref(source(*src))))


def score_filter_candidate(recon, mbs, base, src, level, sharpness, every_rows=0):
    m = np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
    return int(load().vo_score_filter_candidate(C.byref(planes(*recon)), ptr(m), C.byref(base),
                                                C.byref(source(*src)), level, sharpness, every_rows))


def filter_sweep(recon, mbs, base, src, every_rows=0, threads=1):
    m = np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
    out = np.zeros(512, np.uint64)
    load().vo_filter_sweep(C.byref(planes(*recon)), ptr(m), C.byref(base), C.byref(source(*src)), every_rows,
                           ptr(out), threads)
    return out.reshape(64, 8)


def select_filter_params(recon, mbs, base, src, threads=1):
    m = np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
    lv, sh = C.c_uint8(), C.c_uint8()
    load().vo_select_filter_params(C.byref(planes(*recon)), ptr(m), C.byref(base), C.byref(source(*src)),
                                   C.byref(lv), C.byref(sh), threads)
    return lv.value, sh.value


def key_frame_sampling(mb_rows):
    """FilterSampling::for_key_frame (src/loop_filter.rs:2266-2272):
    bands = clamp(mb_rows / 32, 3, 6); every_rows = max(mb_rows / bands, 2);
    the sharpness sweep on."""
    bands = min(max(mb_rows // 32, 3), 6)
    return max(mb_rows // bands, 2), True


def select_filter_params_sampled(recon, mbs, base, src, every_rows, sweep_sharpness, threads=1):
    m = np.ascontiguousarray(mbs, abi.MB_LF_INFO_DTYPE)
    lv, sh = C.c_uint8(), C.c_uint8()
    load().vo_select_filter_params_sampled(C.byref(planes(*recon)), ptr(m), C.byref(base), C.byref(source(*src)),
                                           every_rows, int(bool(sweep_sharpness)), C.byref(lv), C.byref(sh), threads)
    return lv.value, sh.value


def select_from_table(table, base_sharp, sampled=False, sweep=True):
    t = np.ascontiguousarray(np.asarray(table, np.uint64).reshape(512))
    lv, sh = C.c_uint8(), C.c_uint8()
    if sampled:
        load().vo_select_from_table_sampled(ptr(t), base_sharp, int(bool(sweep)), C.byref(lv), C.byref(sh))
    else:
        load().vo_select_from_table_full(ptr(t), base_sharp, C.byref(lv), C.byref(sh))
    return lv.value, sh.value


class MbInfo(C.Structure):
    """vo_mb_info (MbInfo, src/near_mv.rs:127)."""

    _fields_ = [("ref_frame", C.c_uint8), ("is_split", C.c_uint8), ("has_split_mvs", C.c_uint8),
                ("reserved", C.c_uint8), ("mv", abi.Mv), ("split_mvs", abi.Mv * 16)]


def mb_info(ref_frame=0, mv=(0, 0), is_split=False, split_mvs=None):
    m = MbInfo()
    m.ref_frame = ref_frame
    m.mv.row, m.mv.col = mv
    m.is_split = int(bool(is_split))
    if split_mvs is not None:
        m.has_split_mvs = 1
        for i, (r, c) in enumerate(split_mvs):
            m.split_mvs[i].row, m.split_mvs[i].col = r, c
    return m


def find_near_mvs(above, left, aboveleft, current_ref=1):
    lib = load()
    fn = lib.vo_find_near_mvs
    fn.restype = None
    fn.argtypes = [C.POINTER(MbInfo)] * 3 + [C.c_uint8, P, P]
    mvs = np.zeros(3, abi.MV_DTYPE)
    cnt = np.zeros(4, np.int32)
    fn(C.byref(above), C.byref(left), C.byref(aboveleft), current_ref, ptr(mvs), ptr(cnt))
    return [(int(m["row"]), int(m["col"])) for m in mvs], [int(c) for c in cnt]


def neighbours_from_decisions(dec):
    """The (above, left, above-left) census records of every MB, built from
    a frame's decisions the way analyse_row forwards them
    (src/encoder/inter.rs:458-480); border slots are intra records."""
    d = np.asarray(dec)
    mbr, mbc = d.shape
    info = np.zeros((mbr + 1, mbc + 1), abi.MB_INFO_DTYPE)  # row/col 0 = border
    inner = info[1:, 1:]
    inner["ref_frame"] = d["ref_frame"]
    inner["mv"] = d["mv"]
    split = d["mode"] == abi.MODE_SPLIT
    inner["is_split"] = split
    inner["has_split_mvs"] = split
    inner["split_mvs"] = np.where(split[..., None], d["split_mvs"], np.zeros_like(d["split_mvs"]))
    nb = np.zeros((mbr, mbc, 3), abi.MB_INFO_DTYPE)
    nb[:, :, 0] = info[:-1, 1:]   # above
    nb[:, :, 1] = info[1:, :-1]   # left
    nb[:, :, 2] = info[:-1, :-1]  # above-left
    return np.ascontiguousarray(nb.reshape(-1))


def rd_inter_search(frame, refs, ref_ids, lam, y1_ac, effort, neighbours, mv_contexts=None, threads=1):
    f = i420(*frame)
    prs = [planes(*p) for p in refs]
    parr = (abi.Planes * len(prs))(*prs)
    ids = np.ascontiguousarray(np.asarray(ref_ids, np.uint8))
    nb = np.ascontiguousarray(neighbours, abi.MB_INFO_DTYPE)
    mbr, mbc = (f.height + 15) // 16, (f.width + 15) // 16
    out = np.zeros(mbr * mbc, abi.RD_INTER_DTYPE)
    ctxs = mv_contexts if mv_contexts is not None else abi.default_mv_contexts()
    st = load().vo_rd_inter_search(C.byref(f), C.cast(parr, C.c_void_p), ptr(ids), len(prs), C.byref(ctxs), lam,
                                   y1_ac, effort, ptr(nb), ptr(out), threads)
    _check(st, "vo_rd_inter_search")
    return out.reshape(mbr, mbc)


# ---- §18 inter prediction (predict.c) -----------------------------------

def chroma_mv(row, col):
    """chroma_mv (src/motion_comp.rs:232) of an eighth-pel luma vector."""
    m = load().vo_chroma_mv(abi.Mv(row, col))
    return (m.row, m.col)


def split_chroma_mvs(split_mvs):
    """split_chroma_mvs (src/motion_comp.rs:2175): 16 quarter-pel vectors ->
    4 eighth-pel chroma vectors, as an (4, 2) int array (row, col)."""
    mv = _mvs(split_mvs)
    assert len(mv) == 16
    out = np.zeros(4, abi.MV_DTYPE)
    load().vo_split_chroma_mvs(ptr(mv), ptr(out))
    return np.stack([out["row"], out["col"]], axis=1).astype(np.int32)


def sixtap_2d(halo81, mx, my, filter_set=abi.FILTER_SIXTAP):
    """sixtap_2d (src/motion_comp.rs:680) of a 9x9 halo, block origin (2, 2)."""
    h = np.ascontiguousarray(np.asarray(halo81, np.uint8).reshape(81))
    out = np.zeros(16, np.uint8)
    load().vo_sixtap_2d(ptr(h), mx, my, filter_set, ptr(out))
    return out.reshape(4, 4)


def predict_inter_mb(ref, mb_xy, mvs, full_pixel=False, filter_set=abi.FILTER_SIXTAP):
    """predict_inter_mb (src/motion_comp.rs:1986) over a batch; (n, 384)."""
    p = planes(*ref)
    xy, mv = _xy(mb_xy), _mvs(mvs)
    out = np.zeros((len(mv), 384), np.uint8)
    load().vo_predict_inter_mb_batch(C.byref(p), ptr(xy), ptr(mv), len(mv), int(bool(full_pixel)), filter_set,
                                     ptr(out))
    return out


def predict_split_mv(ref, mb_xy, split_mvs, full_pixel=False, filter_set=abi.FILTER_SIXTAP):
    """predict_split_mv (src/motion_comp.rs:2228) over a batch; (n, 384)."""
    p = planes(*ref)
    xy, mv = _xy(mb_xy), _mvs(split_mvs)
    n = len(mv) // 16
    out = np.zeros((n, 384), np.uint8)
    load().vo_predict_split_mv_batch(C.byref(p), ptr(xy), ptr(mv), n, int(bool(full_pixel)), filter_set, ptr(out))
    return out


def predict_inter_frame(refs, ref_ids, decisions, out, full_pixel=False, filter_set=abi.FILTER_SIXTAP):
    """The per-MB prediction of pick_mb_for_ref's chosen mode
    (src/encoder.rs:8704-8735) into the MB-padded planes `out` in place.
    Returns the number of MBs left untouched (no inter reference)."""
    prs = [planes(*p) for p in refs]
    parr = (abi.Planes * len(prs))(*prs)
    ids = np.ascontiguousarray(np.asarray(ref_ids, np.uint8))
    dec = np.ascontiguousarray(decisions).reshape(-1)
    op = planes(*out)
    return load().vo_predict_inter_frame(C.cast(parr, C.c_void_p), ptr(ids), len(prs), ptr(dec),
                                         int(bool(full_pixel)), filter_set, C.byref(op))


# ---- §14 inter reconstruction, trellis off (recon.c) ---------------------

def dequant_factors(q, ydc=0, y2dc=0, y2ac=0, uvdc=0, uvac=0):
    """MbDequantFactors::from_base_and_deltas (src/dequant.rs:118):
    (y1_dc, y1_ac, y2_dc, y2_ac, uv_dc, uv_ac)."""
    out = np.zeros(6, np.int16)
    load().vo_dequant_factors(q, ydc, y2dc, y2ac, uvdc, uvac, ptr(out))
    return tuple(int(x) for x in out)


def segment_factors(qi, segment_quant=None, absolute=False):
    """from_quant_indices / for_segment (src/dequant.rs:169, :201)."""
    out = np.zeros(6, np.int16)
    load().vo_segment_factors(C.byref(qi), segment_quant is not None, segment_quant or 0, int(absolute), ptr(out))
    return tuple(int(x) for x in out)


def _blk(fn, block):
    a = np.ascontiguousarray(np.asarray(block, np.int16).reshape(16))
    out = np.zeros(16, np.int16)
    fn(ptr(a), ptr(out))
    return out


def forward_dct_4x4(block):
    return _blk(load().vo_forward_dct_4x4, block)


def forward_wht_4x4(block):
    return _blk(load().vo_forward_wht_4x4, block)


def inverse_dct_4x4(block):
    return _blk(load().vo_inverse_dct_4x4, block)


def inverse_wht_4x4(block):
    return _blk(load().vo_inverse_wht_4x4, block)


def enc_quantize_block(block, dc, ac):
    a = np.ascontiguousarray(np.asarray(block, np.int16).reshape(16)).copy()
    load().vo_enc_quantize_block(ptr(a), dc, ac)
    return a


def reconstruct_inter_mb(src384, pred384, factors, split, tlambda=0.0):
    """The §14 half of the chosen-mode step for one MB (with the §13
    trellis at `tlambda` when > 0): returns (recon 384 B, quantised coeffs
    (400,) int16, flags)."""
    src = np.ascontiguousarray(np.asarray(src384, np.uint8).reshape(384))
    rec = np.ascontiguousarray(np.asarray(pred384, np.uint8).reshape(384)).copy()
    f = np.ascontiguousarray(np.asarray(factors, np.int16).reshape(6))
    cf = np.zeros(400, np.int16)
    fl = load().vo_reconstruct_inter_mb_trellis(ptr(src), ptr(rec), ptr(f), int(bool(split)), ptr(cf), tlambda)
    return rec, cf, fl


def trellis_quantize_block(block, dc, ac, first_coeff, plane, lam, entry_ctx3=0):
    """trellis_quantize_block (src/encoder.rs:3095) on one raster block;
    returns the chosen levels (16,) int16."""
    b = np.ascontiguousarray(np.asarray(block, np.int16).reshape(16)).copy()
    load().vo_trellis_quantize_block(ptr(b), dc, ac, first_coeff, entry_ctx3, plane, lam)
    return b


def coeff_token_bits(plane, i, ctx3, prev_was_zero, level):
    return load().vo_coeff_token_bits(plane, i, ctx3, int(bool(prev_was_zero)), level)


def eob_token_bits(plane, i, ctx3):
    return load().vo_eob_token_bits(plane, i, ctx3)


def trellis_lambda(y1_ac, strength):
    return load().vo_trellis_lambda(y1_ac, strength)


def idct_basis_norm_sq():
    p = load().vo_idct_basis_norm_sq()
    return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(16,)).copy()


def reconstruct_inter_frame(frame, refs, ref_ids, decisions, quant, out, mb_segment=None, segment_quant=None,
                            segment_abs=False, full_pixel=False, filter_set=abi.FILTER_SIXTAP, lf_info=None,
                            threads=1, trellis_strength=0.0):
    """pick_mb_for_ref's chosen-mode §18 + §14 step (with the §13 trellis at
    TrellisStrength `trellis_strength`; 0 = off) for a frame into the
    MB-padded planes `out` in place. Returns
    (coeffs (mb_rows*mb_cols, 400) int16, flags (mb_rows*mb_cols,) uint8,
    number of MBs left untouched); `lf_info` (optional MB_LF_INFO_DTYPE
    array) receives the §15 side information."""
    f = i420(*frame)
    prs = [planes(*p) for p in refs]
    parr = (abi.Planes * len(prs))(*prs)
    ids = np.ascontiguousarray(np.asarray(ref_ids, np.uint8))
    dec = np.ascontiguousarray(decisions).reshape(-1)
    op = planes(*out)
    n = op.mb_cols * op.mb_rows
    cf = np.zeros((n, 400), np.int16)
    fl = np.zeros(n, np.uint8)
    seg = None if mb_segment is None else np.ascontiguousarray(np.asarray(mb_segment, np.int8).reshape(-1))
    sq = None if segment_quant is None else np.ascontiguousarray(np.asarray(segment_quant, np.int16).reshape(4))
    skipped = load().vo_reconstruct_inter_frame_trellis(C.byref(f), C.cast(parr, C.c_void_p), ptr(ids), len(prs),
                                                        ptr(dec), C.byref(quant), ptr(seg), ptr(sq),
                                                        int(bool(segment_abs)), int(bool(full_pixel)), filter_set,
                                                        C.byref(op), ptr(cf), ptr(fl), ptr(lf_info),
                                                        float(trellis_strength), threads)
    return cf, fl, skipped


# ---- VP8 decoder restatement (decoder.c) ---------------------------------

def ivf_frames(data):
    """The frame payloads of an IVF file (32-byte header, then 12-byte frame
    headers: 4-byte little-endian size + 8-byte timestamp)."""
    assert data[:4] == b"DKIF", "not an IVF file"
    hdr = int.from_bytes(data[6:8], "little")
    pos, out = hdr, []
    while pos + 12 <= len(data):
        n = int.from_bytes(data[pos:pos + 4], "little")
        out.append(bytes(data[pos + 12:pos + 12 + n]))
        pos += 12 + n
    return out


class Vp8Decoder:
    """Vp8DecoderState (src/state.rs): decode frames in order; each call
    returns the visible I420 picture as (y, u, v) arrays."""

    def __init__(self):
        self.lib = load()
        self.h = self.lib.vo_vp8_decoder_new()

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.vo_vp8_decoder_free(self.h)
            self.h = None

    def decode_into(self, frame, max_pixels=1 << 24):
        buf = np.frombuffer(frame, np.uint8)
        out = np.zeros(max_pixels * 3 // 2 + 16, np.uint8)
        w, h, shown = U32(), U32(), C.c_int()
        st = self.lib.vo_vp8_decode_frame(self.h, ptr(buf), len(buf), ptr(out), C.byref(w), C.byref(h),
                                          C.byref(shown))
        if st != 0:
            raise RuntimeError(f"vo_vp8_decode_frame: {st}")
        w, h = w.value, h.value
        cw, ch = (w + 1) // 2, (h + 1) // 2
        y = out[:w * h].reshape(h, w).copy()
        u = out[w * h:w * h + cw * ch].reshape(ch, cw).copy()
        v = out[w * h + cw * ch:w * h + 2 * cw * ch].reshape(ch, cw).copy()
        return (y, u, v), bool(shown.value)


def decode_ivf(data):
    """Every frame of an IVF stream through the restated decoder, as a list
    of ((y, u, v), shown)."""
    dec = Vp8Decoder()
    return [dec.decode_into(f) for f in ivf_frames(data)]


class _Capture(C.Structure):
    _fields_ = [("refs", (P * 3) * 3), ("pred", P * 3), ("pre", P * 3), ("post", P * 3), ("dec", P), ("lf", P),
                ("cfg", C.POINTER(abi.FilterConfig)), ("key", C.c_int32), ("version", C.c_int32),
                ("filtered", C.c_int32), ("mb_cols", C.c_int32), ("mb_rows", C.c_int32), ("captured", C.c_int32)]


class CapturingDecoder(Vp8Decoder):
    """A decoder of width x height frames that records each decoded frame's
    intermediate state (MB-padded planes as (y, u, v)): `refs` (LAST,
    GOLDEN, ALTREF in force), `pred` (inter MBs' prediction, intra MBs 0),
    `dec` (MB_DECISION_DTYPE; ref_frame INTRA for intra MBs), `pre` /
    `post` (reconstruction before / after the loop filter), `lf`
    (MB_LF_INFO_DTYPE), `cfg` (abi.FilterConfig), `key`, `version`,
    `filtered`, and the visible `picture`."""

    def __init__(self, width, height):
        super().__init__()
        self.width, self.height = width, height
        mbc, mbr = (width + 15) // 16, (height + 15) // 16
        shapes = [(mbr * 16, mbc * 16), (mbr * 8, mbc * 8), (mbr * 8, mbc * 8)]
        new = lambda: [np.zeros(s, np.uint8) for s in shapes]  # noqa: E731
        self.refs, self.pred, self.pre, self.post = [new() for _ in range(3)], new(), new(), new()
        self.dec = np.zeros(mbc * mbr, abi.MB_DECISION_DTYPE)
        self.lf = np.zeros(mbc * mbr, abi.MB_LF_INFO_DTYPE)
        self.cfg = abi.FilterConfig()
        cap = self.cap = _Capture()
        for s in range(3):
            for p in range(3):
                cap.refs[s][p] = ptr(self.refs[s][p])
        for p in range(3):
            cap.pred[p], cap.pre[p], cap.post[p] = ptr(self.pred[p]), ptr(self.pre[p]), ptr(self.post[p])
        cap.dec, cap.lf, cap.cfg = ptr(self.dec), ptr(self.lf), C.pointer(self.cfg)
        cap.mb_cols, cap.mb_rows = mbc, mbr
        self.lib.vo_vp8_decoder_capture(self.h, C.byref(cap))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.vo_vp8_decoder_capture(self.h, None)
        super().__del__()

    def prime(self, refs):
        """Install `refs` (LAST, GOLDEN, ALTREF as MB-padded (y, u, v)) with
        a key frame's default entropy state (vo_vp8_decoder_prime)."""
        planes = [np.ascontiguousarray(p, np.uint8) for r in refs for p in r]
        arr = (P * 9)(*[ptr(p) for p in planes])
        if self.lib.vo_vp8_decoder_prime(self.h, self.width, self.height, arr) != 0:
            raise RuntimeError("vo_vp8_decoder_prime failed")

    def decode(self, frame):
        self.cap.captured = 0
        picture, shown = self.decode_into(frame)
        if not self.cap.captured:
            raise ValueError("frame size differs from the decoder's; capture needs a fixed size")
        return {"refs": [tuple(p.copy() for p in r) for r in self.refs], "pred": tuple(p.copy() for p in self.pred),
                "pre": tuple(p.copy() for p in self.pre), "post": tuple(p.copy() for p in self.post),
                "dec": self.dec.copy(), "lf": self.lf.copy(), "cfg": abi.FilterConfig.from_buffer_copy(self.cfg),
                "key": bool(self.cap.key), "version": int(self.cap.version), "filtered": bool(self.cap.filtered),
                "picture": picture, "shown": shown}


def decode_ivf_captured(data):
    """Decode an IVF stream with the restated decoder, yielding per frame
    the state CapturingDecoder.decode records."""
    w, h = int.from_bytes(data[12:14], "little"), int.from_bytes(data[14:16], "little")
    dec = CapturingDecoder(w, h)
    for frame in ivf_frames(data):
        yield dec.decode(frame)
