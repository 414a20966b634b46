"""vp8a_filter_sweep_noalloc: the loop-filter candidate sweep for callers
that cannot allocate device memory while they run (a host that gives the
library a fixed memory budget, or a real-time loop where an allocation may
stall). It must give exactly the SSD table of vp8a_filter_sweep, call after
call, while using only its fixed built-in scratch, and must refuse what
that scratch cannot hold or buffers it would have to stage.

This file is collected last on purpose; it passes on its own in a fresh
process as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import vp8a
from vp8a import abi, synth
from vp8a.frames import planes, ptr, source

pytestmark = pytest.mark.gpu


def sweep_case(width, height, seed):
    frames, _ = synth.make_sequence(width, height, 1, seed=seed)
    src = frames[0]
    recon, has = synth.quantised_recon(vp8a.pad_to_mb(*src))
    rng = np.random.default_rng(seed)
    n = has.size
    m = np.zeros(n, abi.MB_LF_INFO_DTYPE)
    m["has_coeffs"] = (rng.random(n) < 0.6) & has.reshape(-1)
    m["ref_frame"] = rng.integers(0, 4, n)
    m["inter_mode"] = np.where(m["ref_frame"] == 0, abi.MODE_NONE, rng.integers(0, 5, n))
    m["y_mode_is_bpred"] = (rng.random(n) < 0.2) | (m["inter_mode"] == abi.MODE_SPLIT)
    m["segment_id"] = rng.integers(-1, 4, n)
    return src, recon, m


def on_device(arrays):
    import torch

    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]


def noalloc_sweep(ctx, drecon, dmbs, base, dsrc, every_rows, dout):
    p, s = planes(*drecon), source(*dsrc)
    return ctx._lib.vp8a_filter_sweep_noalloc(ctx.handle, C.byref(p), ptr(dmbs), C.byref(base), C.byref(s),
                                             every_rows, ptr(dout))


def pool_high_water_reset():
    """Resets the high-water mark of the device's default memory pool (the
    pool the library's stream-ordered staging draws from) and returns a
    function that reads it back."""
    from cuda.bindings import driver as drv

    import torch

    dev = torch.cuda.current_device()
    err, pool = drv.cuDeviceGetDefaultMemPool(dev)
    assert err == drv.CUresult.CUDA_SUCCESS, err
    attr = drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH
    (err,) = drv.cuMemPoolSetAttribute(pool, attr, drv.cuuint64_t(0))
    assert err == drv.CUresult.CUDA_SUCCESS, err

    def read():
        e, v = drv.cuMemPoolGetAttribute(pool, attr)
        assert e == drv.CUresult.CUDA_SUCCESS, e
        return int(v)

    return read


@pytest.mark.parametrize("size", [(640, 368), (320, 240), (4096, 2176)])
def test_noalloc_sweep_matches_filter_sweep_twice(ctx, size):
    import torch

    src, recon, m = sweep_case(*size, seed=size[0] + size[1])
    base = abi.filter_config(20, 0)
    dsrc, drecon = on_device(src), on_device(recon)
    dmbs = torch.from_numpy(m.view(np.uint8).copy()).cuda()
    dout = torch.zeros(512, dtype=torch.int64, device="cuda")
    wants = {er: vp8a.filter_sweep(ctx, recon, m, base, src, every_rows=er) for er in (0, 3)}
    # A first call loads the kernels and looks the scratch address up; the
    # calls after it must take no device memory at all: the default pool's
    # high-water mark stays at zero and the GPU's free memory is unchanged.
    assert noalloc_sweep(ctx, drecon, dmbs, base, dsrc, 0, dout) == abi.OK
    assert ctx._lib.vp8a_ctx_synchronize(ctx.handle) == abi.OK
    torch.cuda.synchronize()
    high = pool_high_water_reset()
    free0 = torch.cuda.mem_get_info()[0]
    for every_rows in (0, 0, 3):  # two whole-frame calls in a row, then a sampled one
        dout.fill_(-1)
        torch.cuda.synchronize()
        assert noalloc_sweep(ctx, drecon, dmbs, base, dsrc, every_rows, dout) == abi.OK
        assert ctx._lib.vp8a_ctx_synchronize(ctx.handle) == abi.OK
        got = dout.cpu().numpy().view(np.uint64).reshape(64, 8)
        assert np.array_equal(got, wants[every_rows]), every_rows
    assert high() == 0
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_sweep_refuses_host_buffers_and_oversized_grids(ctx):
    import torch

    src, recon, m = sweep_case(64, 48, seed=5)
    base = abi.filter_config(20, 0)
    host_out = np.zeros(512, np.uint64)
    # Host buffers would need staging, which allocates.
    st = ctx._lib.vp8a_filter_sweep_noalloc(ctx.handle, C.byref(planes(*recon)), ptr(m), C.byref(base),
                                            C.byref(source(*src)), 0, ptr(host_out))
    assert st == abi.E_INVALID_ARGUMENT
    assert b"device memory" in ctx._lib.vp8a_last_error()
    # 4112 pixels wide is one MB column more than the scratch holds.
    wide = [torch.zeros((16, 4112), dtype=torch.uint8, device="cuda"),
            torch.zeros((8, 2056), dtype=torch.uint8, device="cuda"),
            torch.zeros((8, 2056), dtype=torch.uint8, device="cuda")]
    dmbs = torch.zeros(257 * abi.MB_LF_INFO_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    dout = torch.zeros(512, dtype=torch.int64, device="cuda")
    st = noalloc_sweep(ctx, wide, dmbs, base, wide, 0, dout)
    assert st == abi.E_INVALID_DIMENSIONS
    assert b"4096x2176" in ctx._lib.vp8a_last_error()
    # 2192 pixels tall is one MB row more than the scratch holds.
    tall = [torch.zeros((2192, 16), dtype=torch.uint8, device="cuda"),
            torch.zeros((1096, 8), dtype=torch.uint8, device="cuda"),
            torch.zeros((1096, 8), dtype=torch.uint8, device="cuda")]
    dmbs = torch.zeros(137 * abi.MB_LF_INFO_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    st = noalloc_sweep(ctx, tall, dmbs, base, tall, 0, dout)
    assert st == abi.E_INVALID_DIMENSIONS
    assert b"4096x2176" in ctx._lib.vp8a_last_error()
