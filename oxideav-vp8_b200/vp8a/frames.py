"""Building the ABI picture records from numpy arrays or torch tensors.

A picture is a tuple (y, u, v) of 2-D uint8 arrays (rows x columns; a row
stride larger than the width is allowed through slicing). numpy arrays are
host memory; torch CUDA tensors are device memory; the library accepts both.
"""
import ctypes as C

import numpy as np

from . import abi


def ptr(x):
    """Address of a numpy array / torch tensor (or an int) for the ABI."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    raise TypeError(f"cannot take the address of {type(x)}")


def row_stride(a):
    """Row pitch in bytes of a 2-D uint8 array/tensor (unit column stride)."""
    if isinstance(a, np.ndarray):
        assert a.dtype == np.uint8 and a.ndim == 2 and a.strides[1] == 1, "need a 2-D uint8 row-major plane"
        return a.strides[0]
    assert a.dim() == 2 and a.stride(1) == 1, "need a 2-D uint8 row-major plane"
    return a.stride(0)


def i420(y, u, v, width=None, height=None):
    """vp8a_i420 (I420Frame, src/encoder.rs:5419) over three planes."""
    f = abi.I420()
    f.height = height if height is not None else y.shape[0]
    f.width = width if width is not None else y.shape[1]
    f.y, f.u, f.v = ptr(y), ptr(u), ptr(v)
    f.y_stride = row_stride(y)
    f.uv_stride = row_stride(u)
    return f


def planes(y, u, v):
    """vp8a_planes (KeyframePlanes, src/frame.rs:123) over MB-padded planes."""
    p = abi.Planes()
    p.y, p.u, p.v = ptr(y), ptr(u), ptr(v)
    p.y_stride = row_stride(y)
    p.uv_stride = row_stride(u)
    p.mb_rows = y.shape[0] // 16
    p.mb_cols = y.shape[1] // 16
    return p


def source(y, u, v, width=None, height=None):
    """vp8a_source (SourcePlanes, src/loop_filter.rs:1916)."""
    s = abi.Source()
    s.height = height if height is not None else y.shape[0]
    s.width = width if width is not None else y.shape[1]
    s.y, s.u, s.v = ptr(y), ptr(u), ptr(v)
    s.y_stride = row_stride(y)
    s.uv_stride = row_stride(u)
    return s


def luma_ref(plane, width=None, height=None):
    """vp8a_luma_ref (LumaRef, src/motion_search.rs:230)."""
    r = abi.LumaRef()
    r.plane = ptr(plane)
    r.stride = row_stride(plane)
    r.height = height if height is not None else plane.shape[0]
    r.width = width if width is not None else plane.shape[1]
    return r


def pad_to_mb(y, u, v):
    """Edge-replicate a visible I420 picture into MB-padded planes (the
    layout KeyframePlanes uses: mb_cols*16 x mb_rows*16 luma)."""
    h, w = y.shape
    mbr, mbc = (h + 15) // 16, (w + 15) // 16
    Y = np.pad(y, ((0, mbr * 16 - h), (0, mbc * 16 - w)), mode="edge")
    U = np.pad(u, ((0, mbr * 8 - u.shape[0]), (0, mbc * 8 - u.shape[1])), mode="edge")
    V = np.pad(v, ((0, mbr * 8 - v.shape[0]), (0, mbc * 8 - v.shape[1])), mode="edge")
    return np.ascontiguousarray(Y), np.ascontiguousarray(U), np.ascontiguousarray(V)


def struct_array(records, ctype):
    arr = (ctype * len(records))(*records)
    return arr, C.cast(arr, C.c_void_p).value
