"""Loader and prototypes for libvp8a.so, the B200 encoder-analysis library.

The shared library is built in-tree (vp8a/build.py) next to this file. It is
the only implementation: there is no CPU fallback, so a missing or unloadable
library raises, and a process without a GPU gets VP8A_E_NO_DEVICE from
vp8a_ctx_create.
"""
import ctypes as C
import os

from . import abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libvp8a.so")

# Every entry point declared in include/vp8a.h, with its argtypes/restype.
P = C.c_void_p
U32 = C.c_uint32
PROTOTYPES = {
    "vp8a_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "vp8a_ctx_destroy": (C.c_int, [P]),
    "vp8a_ctx_stream": (P, [P]),
    "vp8a_ctx_synchronize": (C.c_int, [P]),
    "vp8a_ctx_launch_count": (C.c_uint64, [P]),
    "vp8a_ctx_set_wait_limit": (C.c_int, [P, C.c_uint64]),
    "vp8a_ctx_set_autotune": (C.c_int, [P, U32]),
    "vp8a_select_filter_params_batch": (C.c_int, [P, P, U32, P, P]),
    "vp8a_ctx_set_subpel_planes": (C.c_int, [P, U32]),
    "vp8a_ctx_set_trellis_strength": (C.c_int, [P, C.c_double]),
    "vp8a_ctx_force_sweep_layout": (C.c_int, [P, U32, U32, U32]),
    "vp8a_ctx_last_sweep_layout": (C.c_int, [P, P]),
    "vp8a_last_error": (C.c_char_p, []),
    "vp8a_abi_version": (U32, []),
    "vp8a_mb_luma_sad_at_mv": (C.c_int, [P, C.POINTER(abi.LumaRef), P, P, P, U32, P]),
    "vp8a_small_diamond_search_luma": (C.c_int, [P, C.POINTER(abi.LumaRef), P, P, P, U32, U32, P]),
    "vp8a_half_pixel_refine_luma": (C.c_int, [P, C.POINTER(abi.LumaRef), P, P, P, U32, P]),
    "vp8a_quarter_pixel_refine_luma": (C.c_int, [P, C.POINTER(abi.LumaRef), P, P, P, U32, P]),
    "vp8a_motion_descent": (C.c_int, [P, C.POINTER(abi.LumaRef), P, P, P, U32, U32, P, P, P]),
    "vp8a_analyse_inter_frame": (
        C.c_int,
        [P, C.POINTER(abi.I420), P, P, U32, C.POINTER(abi.MvContexts), C.c_double, P, P],
    ),
    "vp8a_analyse_inter_frame_proposals": (
        C.c_int,
        [P, C.POINTER(abi.I420), P, P, U32, C.POINTER(abi.MvContexts), C.c_double, P, P, P],
    ),
    "vp8a_rd_lambda": (C.c_double, [U32]),
    "vp8a_analyse_inter_frames": (C.c_int, [P, P, U32]),
    "vp8a_analyse_inter_frames_proposals": (C.c_int, [P, P, U32, P]),
    "vp8a_build_arnr_altrefs": (C.c_int, [P, P, U32]),
    "vp8a_build_arnr_altrefs_planes": (C.c_int, [P, P, U32]),
    "vp8a_reconstruct_inter_frames": (C.c_int, [P, P, U32]),
    "vp8a_filter_sweeps": (C.c_int, [P, P, U32]),
    "vp8a_lp_net_propose": (C.c_int, [P, P, U32, P, P, P, P, P, P, P, P, U32, P, P]),
    "vp8a_motion_descent_masked": (C.c_int, [P, P, P, P, P, U32, U32, P, P, P, P]),
    "vp8a_lp_seeded_search": (C.c_int, [P, P, P, P, P, U32, U32, U32, P]),
    "vp8a_lp_windows": (C.c_int, [P, C.POINTER(abi.LumaRef), C.POINTER(abi.LumaRef), P, U32, P]),
    "vp8a_lp_conv_forward": (C.c_int, [P, P, U32, P, P, U32, U32, U32, P, P]),
    "vp8a_lp_conv_backward": (C.c_int, [P, P, U32, P, U32, U32, P, U32, P, P, P]),
    "vp8a_lp_softmax_ce": (C.c_int, [P, P, P, U32, P, P, P]),
    "vp8a_lp_adam": (C.c_int, [P, P, P, P, P, U32, C.c_float, C.c_float, C.c_float, C.c_float, U32, P]),
    "vp8a_lp_pool": (C.c_int, [P, P, U32, U32, P]),
    "vp8a_lp_lf_head": (C.c_int, [P, P, C.c_float, U32, P, P, U32, C.c_int32, P, P, P, P]),
    "vp8a_filter_sweep_window": (C.c_int, [P, P, P, P, P, U32, U32, P]),
    "vp8a_rd_inter_search": (
        C.c_int,
        [P, C.POINTER(abi.I420), P, P, U32, C.POINTER(abi.MvContexts), C.c_double, U32, U32, P, P],
    ),
    "vp8a_predict_inter_mb": (C.c_int, [P, C.POINTER(abi.Planes), P, P, U32, U32, U32, P]),
    "vp8a_predict_split_mv": (C.c_int, [P, C.POINTER(abi.Planes), P, P, U32, U32, U32, P]),
    "vp8a_predict_inter_frame": (C.c_int, [P, P, P, U32, P, U32, U32, C.POINTER(abi.Planes)]),
    "vp8a_dequant_factors": (None, [C.POINTER(abi.QuantIndices), U32, C.c_int32, U32, P]),
    "vp8a_write_inter_frame": (C.c_int, [C.POINTER(abi.FrameHeader), P, P, P, P, P, C.c_uint64,
                                         C.POINTER(C.c_uint64)]),
    "vp8a_reconstruct_inter_frame": (
        C.c_int,
        [P, C.POINTER(abi.I420), P, P, U32, P, C.POINTER(abi.QuantIndices), P, P, U32, U32, U32,
         C.POINTER(abi.Planes), P, P, P],
    ),
    "vp8a_build_arnr_altref": (C.c_int, [P, P, U32, U32, U32, P, P, P]),
    "vp8a_build_arnr_altref_planes": (C.c_int, [P, P, U32, U32, U32, C.POINTER(abi.Planes)]),
    "vp8a_filter_frame": (C.c_int, [P, C.POINTER(abi.Planes), P, C.POINTER(abi.FilterConfig)]),
    "vp8a_reconstruction_ssd": (C.c_int, [P, C.POINTER(abi.Planes), C.POINTER(abi.Source), P]),
    "vp8a_filter_sweep": (
        C.c_int,
        [P, C.POINTER(abi.Planes), P, C.POINTER(abi.FilterConfig), C.POINTER(abi.Source), U32, P],
    ),
    "vp8a_filter_sweep_noalloc": (
        C.c_int,
        [P, C.POINTER(abi.Planes), P, C.POINTER(abi.FilterConfig), C.POINTER(abi.Source), U32, P],
    ),
    "vp8a_select_filter_params": (
        C.c_int,
        [P, C.POINTER(abi.Planes), P, C.POINTER(abi.FilterConfig), C.POINTER(abi.Source), P, P],
    ),
    "vp8a_key_frame_sampling": (None, [U32, C.POINTER(U32), C.POINTER(U32)]),
    "vp8a_select_filter_params_sampled": (
        C.c_int,
        [P, C.POINTER(abi.Planes), P, C.POINTER(abi.FilterConfig), C.POINTER(abi.Source), U32, U32, P, P],
    ),
}

_lib = None


def load():
    """Load libvp8a.so (once) and attach prototypes. Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libvp8a.so not found at {LIB_PATH}; build it with "
            "`python oxideav-vp8_b200/vp8a/build.py` (there is no CPU fallback)"
        )
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class Vp8aError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        msg = load().vp8a_last_error().decode(errors="replace")
        super().__init__(f"{where}: {abi.STATUS_NAMES.get(status, status)} ({msg})")


def check(status, where=""):
    if status != abi.OK:
        raise Vp8aError(status, where)
    return status
