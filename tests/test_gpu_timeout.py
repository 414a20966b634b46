"""The analysis wavefront's bounded wait, made to run out on purpose.

An MB row of vp8a_analyse_inter_frame waits (polling a progress counter in
global memory) for the row above it. The wait has a poll budget; when it is
spent the kernel records a timeout in the context's status word, every CTA
of every cluster leaves at its next MB boundary, and the call returns
VP8A_E_DEVICE_TIMEOUT — the device-side form of the reference's abort
contract for its row workers (src/encoder/inter.rs:289-326). With the budget
at 0 the first poll that finds the row above behind gives up, which any
frame of several MB rows meets (the rows start together and row r needs row
r - 1's first MB). Nothing here faults or hangs: the wait is a plain
load-and-compare loop with nothing in flight, and the context must analyse
the next frame exactly once the budget is back."""
import numpy as np
import pytest

import vp8a
from vp8a import abi, synth

pytestmark = pytest.mark.gpu


def case():
    frames, _ = synth.make_sequence(320, 240, 4, seed=41, pieces=3, occluders=2)
    refs = [vp8a.pad_to_mb(*frames[2]), vp8a.pad_to_mb(*frames[0])]
    return frames[3], refs, [abi.REF_LAST, abi.REF_GOLDEN], vp8a.rd_lambda(44)


def same(got, want):
    return all(np.array_equal(got[f], want[f]) for f in got.dtype.names if f != "reserved")


def test_analysis_wait_runs_out_and_the_context_recovers(oracle):
    frame, refs, ids, lam = case()
    want = oracle.analyse_inter_frame(frame, refs, ids, lam, threads=4)
    with vp8a.Context(0) as c:
        c.set_wait_limit(0)
        for _ in range(2):
            with pytest.raises(vp8a.Vp8aError, match="DeviceTimeout") as ei:
                vp8a.analyse_inter_frame(c, frame, refs, ids, lam)
            assert ei.value.status == abi.E_DEVICE_TIMEOUT
        # The status word was read and cleared: the next synchronize is clean.
        c.synchronize()
        c.set_wait_limit(1 << 24)
        got = vp8a.analyse_inter_frame(c, frame, refs, ids, lam)
        assert same(got, want)


def test_device_resident_analysis_reports_the_timeout_at_synchronize(oracle):
    # With every buffer on the device the call is asynchronous: it returns
    # OK and the next synchronize reports the wait that ran out.
    import ctypes as C

    import torch

    frame, refs, ids, lam = case()
    want = oracle.analyse_inter_frame(frame, refs, ids, lam, threads=4)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    cur = [d(p) for p in frame]
    drefs = [[d(p) for p in r] for r in refs]
    n = want.size
    out = torch.zeros(n * abi.MB_DECISION_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    host_ids = np.array(ids, np.uint8)
    torch.cuda.synchronize()
    with vp8a.Context(0) as c:
        lib = c._lib
        f = vp8a.i420(*cur)
        pl = (abi.Planes * 2)(*[vp8a.planes(*r) for r in drefs])
        ctxs = abi.default_mv_contexts()
        call = lambda: lib.vp8a_analyse_inter_frame(c.handle, C.byref(f), C.cast(pl, C.c_void_p),  # noqa: E731
                                                    host_ids.ctypes.data, 2, C.byref(ctxs), lam, out.data_ptr(),
                                                    None)
        c.set_wait_limit(0)
        assert call() == abi.OK
        assert lib.vp8a_ctx_synchronize(c.handle) == abi.E_DEVICE_TIMEOUT
        c.set_wait_limit(1 << 24)
        assert call() == abi.OK
        assert lib.vp8a_ctx_synchronize(c.handle) == abi.OK
        got = np.frombuffer(out.cpu().numpy().tobytes(), abi.MB_DECISION_DTYPE).reshape(want.shape)
        assert same(got, want)


def test_batched_analysis_wait_runs_out_and_the_context_recovers(oracle):
    frame, refs, ids, lam = case()
    want = oracle.analyse_inter_frame(frame, refs, ids, lam, threads=4)
    jobs = [dict(frame=frame, refs=refs, ref_ids=ids, lam=lam)] * 2
    with vp8a.Context(0) as c:
        c.set_wait_limit(0)
        with pytest.raises(vp8a.Vp8aError, match="DeviceTimeout"):
            vp8a.analyse_inter_frames(c, jobs)
        c.set_wait_limit(1 << 24)
        for got in vp8a.analyse_inter_frames(c, jobs):
            assert same(got, want)

