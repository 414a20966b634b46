"""The C-ABI library loads and exports exactly what include/vp8a.h declares,
and the Python record mirrors match the C layouts (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

import vp8a
from vp8a import abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "vp8a.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vp8a_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_prototyped_functions():
    assert declared_functions() == sorted(vp8a.PROTOTYPES)


def test_library_exports_every_declared_symbol():
    lib = vp8a.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.vp8a_abi_version() >> 16 == 1


def test_wait_limit_needs_a_context():
    # Host-side argument check only: no device work without a context.
    assert vp8a.load().vp8a_ctx_set_wait_limit(None, 5) == abi.E_INVALID_ARGUMENT


def test_record_layouts_match_c(oracle):
    assert abi.check_layouts() == oracle.type_sizes()


def test_no_cpu_fallback_without_gpu():
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is visible")
    lib = vp8a.load()
    h = C.c_void_p()
    assert lib.vp8a_ctx_create(0, C.byref(h)) == abi.E_NO_DEVICE
    assert b"no CPU fallback" in lib.vp8a_last_error()
    with pytest.raises(vp8a.Vp8aError):
        vp8a.Context(0)


def test_rd_lambda_host_helper(oracle):
    for qi in (0, 44, 100, 127):
        assert vp8a.rd_lambda(qi) == oracle.rd_lambda(qi)


def test_key_frame_sampling_helper(oracle):
    # FilterSampling::for_key_frame, host-side in the library.
    for mb_rows in list(range(1, 300)) + [4096]:
        assert vp8a.key_frame_sampling(mb_rows) == oracle.key_frame_sampling(mb_rows), mb_rows


def test_dequant_factors_helper(oracle):
    # MbDequantFactors::from_quant_indices / for_segment, host-side in the library.
    for qi in (abi.quant_indices(44, y_dc=-3, y2_dc=5, y2_ac=-7, uv_dc=9, uv_ac=-2), abi.quant_indices(0),
               abi.quant_indices(127, y_dc=15, uv_dc=-15)):
        assert vp8a.dequant_factors(qi) == oracle.segment_factors(qi)
        for sq, absolute in ((15, False), (-60, False), (100, True), (2**31 - 1, False), (-2**31, True)):
            assert vp8a.dequant_factors(qi, sq, absolute) == oracle.segment_factors(qi, sq, absolute)
