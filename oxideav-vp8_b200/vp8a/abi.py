"""ctypes / numpy mirrors of the POD types declared in include/vp8a.h.

The C header is the contract; these definitions repeat its layouts so that
Python callers (and the tests) can pass numpy arrays or torch tensors of
these records straight through the C ABI. `check_layouts()` asserts the
sizes against the C compiler's view (exported by the library itself).
"""
import ctypes as C

import numpy as np

# vp8a_status (include/vp8a.h)
OK = 0
E_INVALID_DIMENSIONS = 1
E_QUANT_INDEX_OUT_OF_RANGE = 2
E_LOOP_FILTER_LEVEL_OUT_OF_RANGE = 3
E_SHARPNESS_LEVEL_OUT_OF_RANGE = 4
E_REFERENCE_DIMENSIONS_MISMATCH = 5
E_INVALID_ARGUMENT = 6
E_CUDA = 7
E_DEVICE_TIMEOUT = 8
E_OUT_OF_MEMORY = 9
E_NO_DEVICE = 10
E_INVALID_DCT_PARTITION_COUNT = 11
E_FIRST_PARTITION_TOO_LARGE = 12
E_COEFFICIENT_OUT_OF_RANGE = 13
E_INVALID_COPY_BUFFER_SELECTOR = 14
E_LOOP_FILTER_DELTA_OUT_OF_RANGE = 15

STATUS_NAMES = {
    0: "OK",
    1: "InvalidDimensions",
    2: "QuantIndexOutOfRange",
    3: "LoopFilterLevelOutOfRange",
    4: "SharpnessLevelOutOfRange",
    5: "ReferenceDimensionsMismatch",
    6: "InvalidArgument",
    7: "Cuda",
    8: "DeviceTimeout",
    9: "OutOfMemory",
    10: "NoDevice",
    11: "InvalidDctPartitionCount",
    12: "FirstPartitionTooLarge",
    13: "CoefficientOutOfRange",
    14: "InvalidCopyBufferSelector",
    15: "LoopFilterDeltaOutOfRange",
}

REF_INTRA, REF_LAST, REF_GOLDEN, REF_ALTREF = 0, 1, 2, 3
MODE_ZERO, MODE_NEAREST, MODE_NEAR, MODE_NEW, MODE_SPLIT, MODE_NONE = 0, 1, 2, 3, 4, 255
FILTER_SIXTAP, FILTER_BILINEAR = 0, 1
PART_TOP_BOTTOM, PART_LEFT_RIGHT, PART_QUARTERS, PART_MV16, PART_NONE = 0, 1, 2, 3, 255


class Mv(C.Structure):
    _fields_ = [("row", C.c_int16), ("col", C.c_int16)]


class SearchResult(C.Structure):
    _fields_ = [("mv", Mv), ("sad", C.c_uint32)]


class LumaRef(C.Structure):
    _fields_ = [("plane", C.c_void_p), ("stride", C.c_uint64), ("width", C.c_uint32), ("height", C.c_uint32)]


class I420(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("y", C.c_void_p),
        ("u", C.c_void_p),
        ("v", C.c_void_p),
        ("y_stride", C.c_uint64),
        ("uv_stride", C.c_uint64),
    ]


class Planes(C.Structure):
    _fields_ = [
        ("y", C.c_void_p),
        ("u", C.c_void_p),
        ("v", C.c_void_p),
        ("y_stride", C.c_uint64),
        ("uv_stride", C.c_uint64),
        ("mb_cols", C.c_uint32),
        ("mb_rows", C.c_uint32),
    ]


class MvContexts(C.Structure):
    _fields_ = [("p", (C.c_uint8 * 19) * 2)]


class FilterConfig(C.Structure):
    _fields_ = [
        ("simple", C.c_uint8),
        ("key_frame", C.c_uint8),
        ("loop_filter_level", C.c_uint8),
        ("sharpness_level", C.c_uint8),
        ("segmentation_enabled", C.c_uint8),
        ("segment_abs", C.c_uint8),
        ("delta_enabled", C.c_uint8),
        ("reserved", C.c_uint8),
        ("segment_lf_level", C.c_int16 * 4),
        ("ref_delta_current", C.c_int16),
        ("bpred_mode_delta", C.c_int16),
        ("ref_delta_last", C.c_int16),
        ("ref_delta_golden", C.c_int16),
        ("ref_delta_altref", C.c_int16),
        ("zero_mv_mode_delta", C.c_int16),
        ("other_mv_mode_delta", C.c_int16),
        ("split_mv_mode_delta", C.c_int16),
    ]


class QuantIndices(C.Structure):
    """vp8a_quant_indices (QuantIndices, src/coded_header.rs:171); 0 = no delta."""

    _fields_ = [("y_ac_qi", C.c_uint8), ("y_dc_delta", C.c_int8), ("y2_dc_delta", C.c_int8),
                ("y2_ac_delta", C.c_int8), ("uv_dc_delta", C.c_int8), ("uv_ac_delta", C.c_int8),
                ("reserved", C.c_uint8 * 2)]


def quant_indices(y_ac_qi, y_dc=0, y2_dc=0, y2_ac=0, uv_dc=0, uv_ac=0):
    return QuantIndices(y_ac_qi, y_dc, y2_dc, y2_ac, uv_dc, uv_ac)


MB_SKIP, MB_HAS_COEFFS = 1, 2


class FrameHeader(C.Structure):
    """vp8a_frame_header: the frame-level choices of an inter frame's
    header (KeyframeParams, RefreshControls src/encoder.rs:9174,
    LoopFilterDeltas :771, the segmentation layer)."""

    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("quant", QuantIndices),
        ("filter_type", C.c_uint8),
        ("loop_filter_level", C.c_uint8),
        ("sharpness_level", C.c_uint8),
        ("n_partitions", C.c_uint8),
        ("refresh_golden_frame", C.c_uint8),
        ("refresh_alternate_frame", C.c_uint8),
        ("copy_buffer_to_golden", C.c_uint8),
        ("copy_buffer_to_alternate", C.c_uint8),
        ("refresh_last", C.c_uint8),
        ("pick_intra", C.c_uint8),
        ("fit_skip_prob", C.c_uint8),
        ("lf_delta_enabled", C.c_uint8),
        ("lf_delta_update", C.c_uint8),
        ("lf_ref_delta_present", C.c_uint8),
        ("lf_mode_delta_present", C.c_uint8),
        ("lf_ref_delta", C.c_int8 * 4),
        ("lf_mode_delta", C.c_int8 * 4),
        ("segmentation", C.c_uint8),
        ("segment_lf_present", C.c_uint8),
        ("segment_quant", C.c_int8 * 4),
        ("segment_lf", C.c_int8 * 4),
        ("reserved", C.c_uint8 * 2),
    ]


def frame_header(width, height, quant, n_partitions=1, refresh_last=True, pick_intra=True, **kw):
    """A vp8a_frame_header with the defaults of the auto-LF P-frame entry
    point (encode_p_frame_multi_ref_auto_loop_filter, src/encoder.rs:9373:
    RefreshControls::default, no deltas, intra picking on) and keyword
    overrides; list-valued fields take sequences."""
    h = FrameHeader()
    h.width, h.height, h.quant = width, height, quant
    h.n_partitions, h.refresh_last, h.pick_intra = n_partitions, int(refresh_last), int(pick_intra)
    for k, v in kw.items():
        if isinstance(v, (list, tuple)):
            arr = getattr(h, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(h, k, int(v))
    return h


class Source(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("y", C.c_void_p),
        ("u", C.c_void_p),
        ("v", C.c_void_p),
        ("y_stride", C.c_uint64),
        ("uv_stride", C.c_uint64),
    ]


MAX_BATCH_JOBS = 1024


class AnalysisJob(C.Structure):
    """vp8a_analysis_job: one vp8a_analyse_inter_frame call of a batch."""

    _fields_ = [("frame", I420), ("refs", C.c_void_p), ("ref_ids", C.c_void_p), ("n_refs", C.c_uint32),
                ("mv_contexts", C.c_void_p), ("lam", C.c_double), ("decisions", C.c_void_p),
                ("trace", C.c_void_p)]


class ArnrJob(C.Structure):
    """vp8a_arnr_job: one vp8a_build_arnr_altref call of a batch."""

    _fields_ = [("frames", C.c_void_p), ("n", C.c_uint32), ("center", C.c_uint32), ("strength", C.c_uint32),
                ("y_out", C.c_void_p), ("u_out", C.c_void_p), ("v_out", C.c_void_p)]


class ArnrPlanesJob(C.Structure):
    """vp8a_arnr_planes_job: one vp8a_build_arnr_altref_planes call of a batch."""

    _fields_ = [("frames", C.c_void_p), ("n", C.c_uint32), ("center", C.c_uint32), ("strength", C.c_uint32),
                ("out", Planes)]


class ReconJob(C.Structure):
    """vp8a_recon_job: one vp8a_reconstruct_inter_frame call of a batch."""

    _fields_ = [("frame", I420), ("refs", C.c_void_p), ("ref_ids", C.c_void_p), ("n_refs", C.c_uint32),
                ("segment_abs", C.c_uint32), ("decisions", C.c_void_p), ("quant", QuantIndices),
                ("mb_segment", C.c_void_p), ("segment_quant", C.c_void_p), ("full_pixel", C.c_uint32),
                ("filter_set", C.c_uint32), ("recon", Planes), ("coeffs", C.c_void_p), ("mb_flags", C.c_void_p),
                ("lf_info", C.c_void_p)]


class SweepJob(C.Structure):
    """vp8a_sweep_job: one vp8a_filter_sweep call of a batch."""

    _fields_ = [("planes", Planes), ("mbs", C.c_void_p), ("base", FilterConfig), ("src", Source),
                ("every_rows", C.c_uint32), ("ssd_out", C.c_void_p)]


MV_DTYPE = np.dtype([("row", "<i2"), ("col", "<i2")])
SEARCH_RESULT_DTYPE = np.dtype([("mv", MV_DTYPE), ("sad", "<u4")])
MB_DECISION_DTYPE = np.dtype(
    [
        ("ref_frame", "u1"),
        ("mode", "u1"),
        ("partition", "u1"),
        ("reserved", "u1"),
        ("mv", MV_DTYPE),
        ("j", "<f8"),
        ("total", "<f8"),
        ("split_mvs", MV_DTYPE, (16,)),
        ("submv_modes", "u1", (16,)),
    ],
    align=True,
)
REF_SEARCH_DTYPE = np.dtype(
    [
        ("best_predictor", MV_DTYPE),
        ("nearest_mv", MV_DTYPE),
        ("near_mv", MV_DTYPE),
        ("sad_zero", "<u4"),
        ("whole", SEARCH_RESULT_DTYPE),
        ("half", SEARCH_RESULT_DTYPE),
        ("quarter", SEARCH_RESULT_DTYPE),
        ("sad_nearest", "<u4"),
        ("sad_near", "<u4"),
        ("chosen_mode", "u1"),
        ("split_partition", "u1"),
        ("reserved", "u1", (2,)),
        ("j", "<f8"),
    ],
    align=True,
)
MB_INFO_DTYPE = np.dtype(
    [
        ("ref_frame", "u1"),
        ("is_split", "u1"),
        ("has_split_mvs", "u1"),
        ("reserved", "u1"),
        ("mv", MV_DTYPE),
        ("split_mvs", MV_DTYPE, (16,)),
    ]
)
RD_INTER_DTYPE = np.dtype(
    [
        ("ref_frame", "u1"),
        ("mode", "u1"),
        ("n_searched", "u1"),
        ("leader", "u1"),
        ("mv", MV_DTYPE),
        ("sad", "<u4"),
        ("cost", "<f8"),
        ("bits", "<f8"),
        ("found", SEARCH_RESULT_DTYPE, (3,)),
    ],
    align=True,
)
EFFORT_FASTEST, EFFORT_FAST, EFFORT_BALANCED, EFFORT_THOROUGH = 0, 1, 2, 3
MB_LF_INFO_DTYPE = np.dtype(
    [
        ("y_mode_is_bpred", "u1"),
        ("has_coeffs", "u1"),
        ("ref_frame", "u1"),
        ("inter_mode", "u1"),
        ("segment_id", "i1"),
        ("reserved", "u1", (3,)),
    ]
)

# Sizes the C compiler gives these records (x86-64 and the CUDA host ABI).
C_SIZES = {
    "vp8a_mv": 4,
    "vp8a_search_result": 8,
    "vp8a_luma_ref": 24,
    "vp8a_i420": 48,
    "vp8a_planes": 48,
    "vp8a_mv_contexts": 38,
    "vp8a_mb_decision": 104,
    "vp8a_ref_search": 64,
    "vp8a_mb_lf_info": 8,
    "vp8a_filter_config": 32,
    "vp8a_source": 48,
    "vp8a_mb_info": 72,
    "vp8a_rd_inter": 56,
    "vp8a_quant_indices": 8,
    "vp8a_analysis_job": 104,
    "vp8a_arnr_job": 48,
    "vp8a_recon_job": 184,
    "vp8a_sweep_job": 152,
    "vp8a_frame_header": 52,
    "vp8a_arnr_planes_job": 72,
}


def check_layouts():
    """Assert that the Python mirrors match the C record sizes."""
    got = {
        "vp8a_mv": C.sizeof(Mv),
        "vp8a_search_result": C.sizeof(SearchResult),
        "vp8a_luma_ref": C.sizeof(LumaRef),
        "vp8a_i420": C.sizeof(I420),
        "vp8a_planes": C.sizeof(Planes),
        "vp8a_mv_contexts": C.sizeof(MvContexts),
        "vp8a_mb_decision": MB_DECISION_DTYPE.itemsize,
        "vp8a_ref_search": REF_SEARCH_DTYPE.itemsize,
        "vp8a_mb_lf_info": MB_LF_INFO_DTYPE.itemsize,
        "vp8a_filter_config": C.sizeof(FilterConfig),
        "vp8a_source": C.sizeof(Source),
        "vp8a_mb_info": MB_INFO_DTYPE.itemsize,
        "vp8a_rd_inter": RD_INTER_DTYPE.itemsize,
        "vp8a_quant_indices": C.sizeof(QuantIndices),
        "vp8a_analysis_job": C.sizeof(AnalysisJob),
        "vp8a_arnr_job": C.sizeof(ArnrJob),
        "vp8a_recon_job": C.sizeof(ReconJob),
        "vp8a_sweep_job": C.sizeof(SweepJob),
        "vp8a_frame_header": C.sizeof(FrameHeader),
        "vp8a_arnr_planes_job": C.sizeof(ArnrPlanesJob),
    }
    assert got == C_SIZES, (got, C_SIZES)
    return got


def default_mv_contexts():
    """DEFAULT_MV_CONTEXT (RFC 6386 §17.2 default MV probabilities)."""
    ctx = MvContexts()
    row = [162, 128, 225, 146, 172, 147, 214, 39, 156, 128, 129, 132, 75, 145, 178, 206, 239, 254, 254]
    col = [164, 128, 204, 170, 119, 235, 140, 230, 228, 128, 130, 130, 74, 148, 180, 203, 236, 254, 254]
    for i in range(19):
        ctx.p[0][i] = row[i]
        ctx.p[1][i] = col[i]
    return ctx


def filter_config(level=0, sharpness=0, simple=False, key_frame=False, **kw):
    """A FrameFilterConfig (src/loop_filter.rs:891) with keyword overrides."""
    c = FilterConfig()
    c.loop_filter_level = level
    c.sharpness_level = sharpness
    c.simple = int(bool(simple))
    c.key_frame = int(bool(key_frame))
    for k, v in kw.items():
        if k == "segment_lf_level":
            for i, x in enumerate(v):
                c.segment_lf_level[i] = x
        else:
            setattr(c, k, v)
    return c
