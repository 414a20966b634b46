"""vp8a — B200-native encoder-analysis path of the OxideAV VP8 encoder.

Motion search (§17/§18), ARNR altref synthesis and the §15 loop-filter
(level, sharpness) search as hand-written sm_100a CUDA kernels behind the
C ABI in include/vp8a.h; this package is the Python mirror of that ABI.
"""
from . import abi, synth
from .api import (
    Context,
    analyse_inter_frame,
    build_arnr_altref,
    filter_frame,
    filter_set_for_version,
    filter_sweep,
    half_pixel_refine_luma,
    key_frame_sampling,
    lf_info_from_decisions,
    mb_luma_sad_at_mv,
    motion_descent,
    neighbours_from_decisions,
    predict_inter_frame,
    predict_inter_mb,
    predict_split_mv,
    rd_inter_search,
    quarter_pixel_refine_luma,
    rd_lambda,
    reconstruction_ssd,
    select_filter_params,
    select_filter_params_key_frame,
    select_filter_params_sampled,
    small_diamond_search_luma,
)
from .frames import i420, luma_ref, pad_to_mb, planes, source
from .lib import LIB_PATH, PROTOTYPES, Vp8aError, load

__all__ = [
    "abi",
    "synth",
    "Context",
    "Vp8aError",
    "load",
    "LIB_PATH",
    "PROTOTYPES",
    "analyse_inter_frame",
    "build_arnr_altref",
    "filter_frame",
    "filter_set_for_version",
    "filter_sweep",
    "half_pixel_refine_luma",
    "key_frame_sampling",
    "lf_info_from_decisions",
    "mb_luma_sad_at_mv",
    "neighbours_from_decisions",
    "predict_inter_frame",
    "predict_inter_mb",
    "predict_split_mv",
    "rd_inter_search",
    "motion_descent",
    "quarter_pixel_refine_luma",
    "rd_lambda",
    "reconstruction_ssd",
    "select_filter_params",
    "select_filter_params_key_frame",
    "select_filter_params_sampled",
    "small_diamond_search_luma",
    "i420",
    "luma_ref",
    "pad_to_mb",
    "planes",
    "source",
]
