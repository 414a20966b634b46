"""Benchmark of the B200 encoder-analysis path on the 1080p P-frame workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload (one step = one 1920x1080 P frame, synthetic seeded I420 input):
  1. ARNR anchor over a 7-frame lookahead window, centre anchor
     (vp8a_build_arnr_altref);
  2. exhaustive inter analysis of the frame against LAST (k-1), GOLDEN
     (k-8) and ALTREF (the fresh anchor, edge-padded) with full sub-pel
     search and SPLITMV per MB per reference (vp8a_analyse_inter_frame);
  3. the prediction, transform, quantisation (qi 44, trellis off) and
     reconstruction of every MB's chosen mode, with its loop-filter side
     information (vp8a_reconstruct_inter_frame);
  4. the loop-filter sweep over all 64 levels x 8 sharpness values of that
     reconstruction, SSD vs source per candidate (vp8a_filter_sweep), and
     the reference's (level, sharpness) walk.
Metric: 1080p macroblocks per second through those stages.

`value` times the step with every input resident in HBM (device pointers);
`e2e` times the step as a frame pipeline through the C ABI: the step's
input frames are copied from pinned host memory to the device, the step
runs on the device, and its results (MB decisions, loop-filter table) are
read back, all inside the timed region; `e2e_per_call` times the drop-in
form, every C-ABI call with pinned host buffers (each call stages its own
inputs and outputs, so references and the reconstruction cross the bus
more than once). L2 is flushed (256 MiB write) between timed steps. With N>1
ranks each GPU analyses its own frames (replicas, no collective on the data
path); `value` is all ranks' MBs over the slowest rank's time.

`--impl reference` times the reference path's CPU restatement (the oracle,
C, all host threads) on the same workload and metric.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "oxideav-vp8_b200"))

W, H = 1920, 1080
MB_COLS, MB_ROWS = 120, 68
N_MB = MB_COLS * MB_ROWS
LOOKAHEAD = 7
QI = 44
SEED = 20261203
METRIC = "1080p MBs/s (ME+ARNR+LF search)"
WORKLOAD = ("1080p P frame: ARNR(7, centre) + exhaustive ME/SPLITMV vs LAST/GOLDEN/ALTREF + qi-44 reconstruction "
            "+ LF 64x8 sweep")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_inputs(seed):
    """Frames 0..15 of the seeded sequence; the P frame is frame 8
    (LAST = 7, GOLDEN = 0); the ARNR window is frames 9..15 (centre 12)."""
    from vp8a import synth

    frames, _ = synth.make_sequence(W, H, 16, seed)
    return frames, synth.digest(frames)


def pad_planes(f):
    import vp8a

    return vp8a.pad_to_mb(*f)


class Clocks:
    """SM clock and throttle-reason sampler over the timed region: NVML in a
    background thread every 10 ms (the first sample is taken before the
    region starts), else nvidia-smi at its 200 ms floor."""

    REASONS = {  # NVML clocks-event reason bits
        "sw_power_cap": 0x4,
        "hw_slowdown": 0x8,
        "sw_thermal_slowdown": 0x20,
        "hw_thermal_slowdown": 0x40,
    }

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.samples = []
        self.nvml = None

    def _nvml_loop(self):
        nv, h = self.nvml, self.handle
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx), int(rs)))
            except Exception:
                pass
            self.first.set()
            self.stop.wait(0.01)

    def __enter__(self):
        import threading

        try:
            import pynvml as nv

            nv.nvmlInit()
            self.handle = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.nvml = nv
            self.stop, self.first = threading.Event(), threading.Event()
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self.thread.start()
            self.first.wait(2.0)
            return self
        except Exception:
            self.nvml = None
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.nvml is not None:
            self.stop.set()
            self.thread.join(2.0)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
            return
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for l in out.splitlines():
                p = [x.strip() for x in l.split(",")]
                if len(p) < 7:
                    continue
                try:
                    sm, mx = float(p[0]), float(p[1])
                except ValueError:
                    continue
                bits = sum(self.REASONS[n] for n, v in zip(names, p[3:7]) if v.lower() == "active")
                self.samples.append((sm, mx, bits))

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [x[0] for x in self.samples]
        reasons = sorted({n for _, _, b in self.samples for n, bit in self.REASONS.items() if b & bit})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(x[1] for x in self.samples), "reasons": reasons,
                "samples": len(sm), "source": "nvml" if self.nvml is not None else "nvidia-smi"}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# --------------------------------------------------------------- GPU arm


class GpuStep:
    """Device-resident buffers and the C-ABI calls of one step."""

    def __init__(self, ctx, frames, lib, torch, device):
        import vp8a
        from vp8a import abi

        self.vp8a, self.abi, self.lib, self.torch, self.ctx = vp8a, abi, lib, torch, ctx
        dev = torch.device("cuda", device)
        # Torch work of the step runs on the library's stream, in order.
        self.stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        cur = frames[8]
        self.cur = [t(p) for p in cur]
        self.last = [t(p) for p in pad_planes(frames[7])]
        self.golden = [t(p) for p in pad_planes(frames[0])]
        self.window = [[t(p) for p in frames[9 + i]] for i in range(LOOKAHEAD)]
        self.alt = [torch.zeros((MB_ROWS * 16, MB_COLS * 16), dtype=torch.uint8, device=dev),
                    torch.zeros((MB_ROWS * 8, MB_COLS * 8), dtype=torch.uint8, device=dev),
                    torch.zeros((MB_ROWS * 8, MB_COLS * 8), dtype=torch.uint8, device=dev)]
        # The chosen modes' reconstruction (and the MBs' loop-filter side
        # information) are rebuilt every step by run_recon.
        self.recon = [torch.zeros_like(p) for p in self.last]
        self.mbs = torch.zeros(N_MB * abi.MB_LF_INFO_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.quant = abi.quant_indices(QI)
        self.dec = torch.zeros(N_MB * abi.MB_DECISION_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.table = torch.zeros(512, dtype=torch.int64, device=dev)
        self.lam = vp8a.rd_lambda(QI)
        self.ids = torch.tensor([1, 2, 3], dtype=torch.uint8, device=dev)
        self.ctxs = abi.default_mv_contexts()
        self.base = abi.filter_config(0, 0)
        self.i420_window = (abi.I420 * LOOKAHEAD)(*[vp8a.i420(*f) for f in self.window])
        self.alt_planes = vp8a.planes(*self.alt)
        self.host_ids = np.array([1, 2, 3], np.uint8)
        torch.cuda.synchronize(dev)  # uploads (torch stream) before library calls
        # Per-MB loop-filter side information from the frame's decisions.
        self.run_arnr()
        self.run_analysis()
        ctx.synchronize()
        torch.cuda.synchronize(dev)
        dec = np.frombuffer(self.dec.cpu().numpy().tobytes(), abi.MB_DECISION_DTYPE)
        self.decisions = dec
        torch.cuda.synchronize(dev)
        self.i420_cur = vp8a.i420(*self.cur)
        self.planes = (abi.Planes * 3)(vp8a.planes(*self.last), vp8a.planes(*self.golden), vp8a.planes(*self.alt))
        self.recon_planes = vp8a.planes(*self.recon)
        self.src = vp8a.source(*self.cur)
        # §18 prediction of every MB's decision (the encoder's next step after
        # the analysis; timed as its own stage, outside the metric's step).
        self.pred = [torch.zeros_like(p) for p in self.last]
        self.pred_planes = vp8a.planes(*self.pred)
        self.run_recon()
        ctx.synchronize()

    def run_arnr(self):
        # The anchor goes straight into the MB-padded ALTREF planes (the
        # blend kernel writes the edge-replicated padding).
        st = self.lib.vp8a_build_arnr_altref_planes(self.ctx.handle, C.cast(self.i420_window, C.c_void_p), LOOKAHEAD,
                                                    3, 3, C.byref(self.alt_planes))
        assert st == 0, self.vp8a.load().vp8a_last_error()

    def run_analysis(self):
        v = self.vp8a
        f = v.i420(*self.cur)
        pl = (self.abi.Planes * 3)(v.planes(*self.last), v.planes(*self.golden), v.planes(*self.alt))
        st = self.lib.vp8a_analyse_inter_frame(self.ctx.handle, C.byref(f), C.cast(pl, C.c_void_p),
                                               self.host_ids.ctypes.data, 3, C.byref(self.ctxs), self.lam,
                                               self.dec.data_ptr(), None)
        assert st == 0, v.load().vp8a_last_error()

    def run_lf(self):
        st = self.lib.vp8a_filter_sweep(self.ctx.handle, C.byref(self.recon_planes), self.mbs.data_ptr(),
                                        C.byref(self.base), C.byref(self.src), 0, self.table.data_ptr())
        assert st == 0, self.vp8a.load().vp8a_last_error()
        # The reference's coarse-grid / refine / sharpness walk over the table.
        self.ctx.synchronize()
        t = self.table.cpu().numpy().view(np.uint64)
        return select_full(t, 0)

    def run_predict(self):
        st = self.lib.vp8a_predict_inter_frame(self.ctx.handle, C.cast(self.planes, C.c_void_p),
                                               self.host_ids.ctypes.data, 3, self.dec.data_ptr(), 0,
                                               self.abi.FILTER_SIXTAP, C.byref(self.pred_planes))
        assert st == 0, self.vp8a.load().vp8a_last_error()

    def run_recon(self):
        st = self.lib.vp8a_reconstruct_inter_frame(self.ctx.handle, C.byref(self.i420_cur), C.cast(self.planes, C.c_void_p),
                                                   self.host_ids.ctypes.data, 3, self.dec.data_ptr(),
                                                   C.byref(self.quant), None, None, 0, 0, self.abi.FILTER_SIXTAP,
                                                   C.byref(self.recon_planes), None, None, self.mbs.data_ptr())
        assert st == 0, self.vp8a.load().vp8a_last_error()

    def step(self):
        self.run_arnr()
        self.run_analysis()
        self.run_recon()
        return self.run_lf()


def select_full(t, bs):
    """select_filter_params_threaded's walk (src/loop_filter.rs:2133-2199)
    over a 64 x 8 candidate table."""
    best_level, best = 0, int(t[bs])
    for lv in list(range(4, 61, 4)) + [63]:
        if int(t[lv * 8 + bs]) < best:
            best, best_level = int(t[lv * 8 + bs]), lv
    g = best_level
    for lv in range(max(0, g - 3), min(63, g + 3) + 1):
        if lv != g and int(t[lv * 8 + bs]) < best:
            best, best_level = int(t[lv * 8 + bs]), lv
    if best_level == 0:
        return 0, bs
    best_sharp = bs
    for sh in range(8):
        if sh != bs and int(t[best_level * 8 + sh]) < best:
            best, best_sharp = int(t[best_level * 8 + sh]), sh
    return best_level, best_sharp


class HostStep:
    """The same step through the C ABI with pinned host buffers (e2e)."""

    def __init__(self, gs, torch):
        self.gs, self.torch = gs, torch
        pin = lambda x: x.cpu().pin_memory()  # noqa: E731
        self.cur = [pin(p) for p in gs.cur]
        self.last = [pin(p) for p in gs.last]
        self.golden = [pin(p) for p in gs.golden]
        self.window = [[pin(p) for p in f] for f in gs.window]
        self.alt = [pin(p) for p in gs.alt]
        self.recon = [pin(p) for p in gs.recon]
        self.mbs = pin(gs.mbs)
        self.dec = torch.zeros(N_MB * gs.abi.MB_DECISION_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
        self.table = torch.zeros(512, dtype=torch.int64).pin_memory()
        self.ids = np.array([1, 2, 3], np.uint8)
        nb = lambda ts: sum(x.numel() * x.element_size() for x in ts)  # noqa: E731
        # Bytes the library copies in and out per step (what each call stages):
        # ARNR window in, anchor out; analysis luma in, decisions out;
        # reconstruction source + references + decisions + recon/LF-info
        # (in/out) in, recon + LF info out; LF sweep recon + info + source in,
        # table out.
        refs = nb(self.last) + nb(self.golden) + nb(self.alt)
        self.h2d = (sum(nb(f) for f in self.window) + self.cur[0].numel() + self.last[0].numel() +
                    self.golden[0].numel() + self.alt[0].numel() +
                    nb(self.cur) + refs + nb([self.dec]) + nb(self.recon) + nb([self.mbs]) +
                    nb(self.recon) + nb([self.mbs]) + nb(self.cur))
        self.d2h = nb(self.alt) + nb([self.dec]) + nb(self.recon) + nb([self.mbs]) + nb([self.table])

    def step(self):
        gs, v, abi, lib = self.gs, self.gs.vp8a, self.gs.abi, self.gs.lib
        win = (abi.I420 * LOOKAHEAD)(*[v.i420(*f) for f in self.window])
        ap = v.planes(*self.alt)
        st = lib.vp8a_build_arnr_altref_planes(gs.ctx.handle, C.cast(win, C.c_void_p), LOOKAHEAD, 3, 3, C.byref(ap))
        assert st == 0
        f = v.i420(*self.cur)
        pl = (abi.Planes * 3)(v.planes(*self.last), v.planes(*self.golden), v.planes(*self.alt))
        st = lib.vp8a_analyse_inter_frame(gs.ctx.handle, C.byref(f), C.cast(pl, C.c_void_p),
                                          self.ids.ctypes.data, 3, C.byref(gs.ctxs), gs.lam, self.dec.data_ptr(),
                                          None)
        assert st == 0
        rp, src = v.planes(*self.recon), v.source(*self.cur)
        st = lib.vp8a_reconstruct_inter_frame(gs.ctx.handle, C.byref(f), C.cast(pl, C.c_void_p), self.ids.ctypes.data,
                                              3, self.dec.data_ptr(), C.byref(gs.quant), None, None, 0, 0,
                                              abi.FILTER_SIXTAP, C.byref(rp), None, None, self.mbs.data_ptr())
        assert st == 0
        st = lib.vp8a_filter_sweep(gs.ctx.handle, C.byref(rp), self.mbs.data_ptr(), C.byref(gs.base), C.byref(src),
                                   0, self.table.data_ptr())
        assert st == 0
        return select_full(self.table.numpy().view(np.uint64), 0)


def max_over_ranks(values, dist, device):
    """Every rank's timing scalars replaced by their maximum over the ranks
    (the slowest rank sets the job's time)."""
    import torch

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def whole_job_rate(units_per_rank_step, steps, world, ms):
    """Units per second of the whole job: every rank's units over the
    slowest rank's time (replicas: each rank processes its own frames)."""
    return units_per_rank_step * steps * world / (ms / 1000.0)


class PipelineStep:
    """The step as a user of the library runs it on a frame stream: the
    step's inputs — the 7 lookahead frames, the P frame and the MB-padded
    LAST and GOLDEN planes — are copied from pinned host memory into device
    buffers, the device-resident step runs through the C ABI, and its
    results (the MB decisions and the loop-filter candidate table) are read
    back; intermediates (the anchor, the reconstruction) stay on the device.
    Two sets of input buffers (two GpuSteps on one context) let the next
    step's upload run on a copy stream while the current step computes, as
    a frame pipeline would: `run(k, between)` uploads and runs k steps,
    every upload inside the call (the first before the first step, each
    later one overlapping the step before it), and calls `between()` on the
    compute stream after each step (the L2 flush)."""

    def __init__(self, gss, torch):
        self.gss, self.torch = gss, torch
        pin = lambda x: x.cpu().pin_memory()  # noqa: E731
        self.pairs = []
        for gs in gss:
            self.pairs.append([(pin(d), d) for dev_planes in [gs.cur, gs.last, gs.golden] + list(gs.window)
                               for d in dev_planes])
        self.dec = torch.zeros(gss[0].dec.numel(), dtype=torch.uint8).pin_memory()
        self.h2d = sum(h.numel() * h.element_size() for h, _ in self.pairs[0])
        self.d2h = self.dec.numel() + gss[0].table.numel() * gss[0].table.element_size()
        self.copy = torch.cuda.Stream(device=gss[0].stream.device)
        self.ready = [torch.cuda.Event() for _ in gss]
        self.free = [torch.cuda.Event() for _ in gss]
        for e in self.free:
            e.record(gss[0].stream)

    def upload(self, i):
        """Step inputs into buffer set i on the copy stream, once the step
        that last read them is done."""
        with self.torch.cuda.stream(self.copy):
            self.copy.wait_event(self.free[i])
            for h, d in self.pairs[i]:
                d.copy_(h, non_blocking=True)
            self.ready[i].record(self.copy)

    def run(self, k, between=None):
        choice = None
        # The first upload follows everything already on the compute stream
        # (a timing event recorded there included).
        self.copy.wait_stream(self.gss[0].stream)
        self.upload(0)
        for n in range(k):
            i = n % 2
            gs = self.gss[i]
            gs.stream.wait_event(self.ready[i])
            if n + 1 < k:
                self.upload(1 - i)
            choice = gs.step()  # ends with the table's read-back and the walk
            with self.torch.cuda.stream(gs.stream):
                self.dec.copy_(gs.dec, non_blocking=True)
            self.free[i].record(gs.stream)
            if between is not None:
                between()
            gs.ctx.synchronize()
        return choice


def gpu_arm(args):
    import torch
    import torch.distributed as dist

    import vp8a

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = vp8a.load()
    ctx = vp8a.Context(local)
    # Each rank analyses its own frames (replicas): seed by rank.
    frames, digest = make_inputs(SEED + rank)
    gs = GpuStep(ctx, frames, lib, torch, local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    # Warm-up.
    for _ in range(args.warmup):
        gs.step()
    torch.cuda.synchronize(dev)
    # Timed region (device-resident inputs).
    times = []
    launches0 = ctx.launches
    barrier()
    torch.cuda.synchronize(dev)
    with Clocks(local) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            choice = gs.step()
            e.record(stream)
            e.synchronize()
            times.append(s.elapsed_time(e))
        torch.cuda.synchronize(dev)
    barrier()
    launches = ctx.launches - launches0
    lf_layout = ctx.last_sweep_layout()
    ms = float(np.sum(times))
    step_ms = [round(x, 3) for x in times]
    # Per-kernel-stage timing for the roofline (separate, after the timed run).
    stage = stage_times(gs, stream, torch, flush)
    # End-to-end through host buffers.
    hs = HostStep(gs, torch)
    for _ in range(max(1, args.warmup)):
        hs.step()
    e_times = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        hs.step()
        e.record(stream)
        e.synchronize()
        e_times.append(s.elapsed_time(e))
    e_ms_call = float(np.sum(e_times))
    e_times_call = e_times
    # End-to-end as a frame pipeline: inputs up (the next step's upload
    # overlapping the current step), device step, results down; the L2
    # flush between steps is inside the timed region.
    gs2 = GpuStep(ctx, frames, lib, torch, local)
    ps = PipelineStep([gs, gs2], torch)

    def flush_l2():
        with torch.cuda.stream(stream):
            flush.fill_(1)

    ps.run(max(1, args.warmup), flush_l2)
    torch.cuda.synchronize(dev)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    choice = ps.run(args.steps, flush_l2)
    e.record(stream)
    e.synchronize()
    e_times = [s.elapsed_time(e) / args.steps] * args.steps
    got_gs = gs if args.steps % 2 == 1 else gs2
    e_ms = float(np.sum(e_times))
    # The device step's outputs of its last run, for the parity check.
    got = gpu_step_outputs(got_gs, choice)
    if world > 1:
        ms, e_ms, e_ms_call = max_over_ranks([ms, e_ms, e_ms_call], dist, dev)
    result = None
    if rank == 0:
        value = whole_job_rate(N_MB, args.steps, world, ms)
        e2e = whole_job_rate(N_MB, args.steps, world, e_ms)
        e2e_call = whole_job_rate(N_MB, args.steps, world, e_ms_call)
        peak, peak_kind = peaks()
        dom = max((k for k in stage if k not in EXTRA_STAGES), key=lambda k: stage[k]["ms"])
        d = stage[dom]
        achieved = d["bytes"] / (d["ms"] / 1000.0) / 1e9
        ipeak = int32_peak_tops()
        stages = {}
        for k, v in stage.items():
            gbs = v["bytes"] / (v["ms"] / 1000.0) / 1e9
            tops = v["ops"] / (v["ms"] / 1000.0) / 1e12
            stages[k] = {"ms": round(v["ms"], 4), "reps_ms": v["reps"], "alg_bytes": int(v["bytes"]),
                         "dram_traffic": dram_traffic(k), "gbs": round(gbs, 2), "hbm_frac": round(gbs / peak, 5),
                         "alg_ops": int(v["ops"]), "tops": round(tops, 3), "alu_frac": round(tops / ipeak, 4),
                         "in_step": k not in EXTRA_STAGES}
        result = {
            "metric": METRIC,
            "value": round(value, 1),
            "unit": "MB/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u8",
            "data": "synthetic (seeded gratings + quarter-pel six-tap translation + noise)",
            "config": {
                "workload": WORKLOAD,
                "width": W,
                "height": H,
                "refs": 3,
                "lookahead": LOOKAHEAD,
                "lf_candidates": 512,
                "qi": QI,
                "seed": SEED,
                "input_sha256": digest[:16],
                "l2": "flushed between timed steps (256 MiB write)",
                "parallelism": f"replicas x{world}",
                "lf_choice": list(choice),
                "lf_layout": {"passes_per_cta": lf_layout[0], "threads_per_cta": lf_layout[1],
                              "prefetch": bool(lf_layout[2]), "ctas_per_sm": lf_layout[3],
                              "chosen_by": "autotune (timed on the first sweep of this picture shape)"},
            },
            "e2e": {"value": round(e2e, 1), "unit": "MB/s", "h2d_bytes_per_step": int(ps.h2d),
                    "d2h_bytes_per_step": int(ps.d2h),
                    "form": "frame pipeline: each step's inputs up from pinned host memory on a copy stream (two input buffer sets, the next upload overlapping the current step), device-resident step, decisions + LF table down; the L2 flush between steps counted inside"},
            "e2e_per_call": {"value": round(e2e_call, 1), "unit": "MB/s", "h2d_bytes_per_step": int(hs.h2d),
                             "d2h_bytes_per_step": int(hs.d2h),
                             "form": "every C-ABI call with pinned host buffers (the drop-in form: each call "
                                     "stages its own inputs and outputs)"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 5), "traffic": dram_traffic(dom),
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6.65 TB/s",
                         "alu": {"kernel": dom, "achieved": stages[dom]["tops"], "peak": round(ipeak, 2),
                                 "unit": "Tops/s (int32, algorithmic op model)", "frac": stages[dom]["alu_frac"],
                                 "peak_source": "nominal: 148 SMs x 128 INT32 lanes x max SM clock"},
                         "stages": stages},
            "gpu_launches": int(launches),
            "step_ms": step_ms,
            "e2e_step_ms": [round(x, 3) for x in e_times],
            "e2e_per_call_step_ms": [round(x, 3) for x in e_times_call],
            "clocks": clk.summary(),
        }
        want = None
        if args.gpus == 1 and world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"], want = cpu_baseline(frames, budget_s=args.cpu_budget)
        if not args.no_parity:
            if want is None:
                sys.path.insert(0, os.path.join(ROOT, "oracle"))
                import oracle

                oracle.build()
                want = cpu_step(oracle, frames, os.cpu_count() or 1)
            ok, detail = step_parity(got, want)
            result["parity"] = ok
            result["parity_detail"] = {**detail, "against": "the oracle (C restatement of the reference) on the "
                                                            "same inputs; rank 0's frames"}
    # Pinned buffers copied on the library's stream are released while that
    # stream still exists (their release records an event on it).
    ctx.synchronize()
    torch.cuda.synchronize(dev)
    del ps, hs, stream
    __import__("gc").collect()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result


# Algorithmic integer operations per stage at 1080p (the op model of the
# scope table's measurement row): ME 3 refs x ~92 k ops per (MB, ref);
# ARNR (L-1) x MBs x 33 x 256 search abs-diffs + (L-1) x picture pixels x 4
# blend ops; LF ~9 k ops per candidate-MB (192 edge segments x ~40 ops plus
# a 384-pixel SSD) over 512 candidates.
STAGE_OPS = {
    "analysis": N_MB * 3 * 92_000,
    "arnr": (LOOKAHEAD - 1) * N_MB * 33 * 256 + (LOOKAHEAD - 1) * (W * H * 3 // 2) * 4,
    "lf_sweep": 512 * N_MB * 9_000,
    # Prediction MACs (below) plus 25 forward and inverse 4x4 transforms
    # (~64 ops each), quantisation and dequantisation (16 each) per MB.
    "recon": N_MB * (6 * (21 * 16 + 16 * 16 + 2 * (13 * 8 + 8 * 8)) + 25 * (64 + 16 + 16 + 64)),
    # Two-pass six-tap MACs of a sub-pel MB: luma 21x16 + 16x16, chroma
    # 2 x (13x8 + 8x8) outputs, 6 taps each.
    "predict": N_MB * 6 * (21 * 16 + 16 * 16 + 2 * (13 * 8 + 8 * 8)),
}
# Stages outside the metric's step (reported, not in `value`).
EXTRA_STAGES = ("predict",)
def int32_peak_tops():
    """Nominal INT32 issue peak: 148 SMs x 128 lanes x max SM clock (no
    measured integer peak is available)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            mhz = float(json.load(f).get("sm_max_mhz", 1965.0))
    except (OSError, ValueError):
        mhz = 1965.0
    return 148 * 128 * mhz * 1e6 / 1e12


def dram_traffic(stage):
    """DRAM bytes per launch of the stage's kernels from the committed ncu
    capture (profiles/dram_traffic_1080p.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic_1080p.json")) as f:
            d = json.load(f)["bytes_per_launch"][stage]
        return int(sum(v["read"] + v["write"] for v in d.values()))
    except (OSError, KeyError, ValueError):
        return None


def stage_times(gs, stream, torch, flush, reps=3):
    """Mean device time per stage (CUDA events on the context stream) and
    each stage's algorithmic bytes (inputs read once + outputs written)."""
    out = {}
    luma = W * H
    pic = luma + 2 * ((W + 1) // 2) * ((H + 1) // 2)
    padded = MB_COLS * 16 * MB_ROWS * 16
    padded_pic = padded + 2 * MB_COLS * 8 * MB_ROWS * 8
    fns = {
        "arnr": (gs.run_arnr, LOOKAHEAD * pic + pic),
        "analysis": (gs.run_analysis, luma + 3 * padded + N_MB * gs.abi.MB_DECISION_DTYPE.itemsize),
        # Source MB, decision and reference MB read, reconstruction and LF
        # info written per MB.
        "recon": (gs.run_recon, N_MB * (384 + gs.abi.MB_DECISION_DTYPE.itemsize + 384 + 384 + 8)),
        "lf_sweep": (lambda: gs.run_lf(), padded_pic + pic + N_MB * 8 + 512 * 8),
        # Decisions read, one MB of reference pixels read and one written per
        # MB; a short kernel, so timed over 10 back-to-back calls.
        "predict": (gs.run_predict, N_MB * (gs.abi.MB_DECISION_DTYPE.itemsize + 2 * 384), 10),
    }
    for name, spec in fns.items():
        fn, nbytes = spec[0], spec[1]
        calls = spec[2] if len(spec) > 2 else 1
        ts = []
        for _ in range(reps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            for _ in range(calls):
                fn()
            e.record(stream)
            e.synchronize()
            ts.append(s.elapsed_time(e) / calls)
        out[name] = {"ms": float(np.median(ts)), "bytes": nbytes, "ops": STAGE_OPS[name],
                     "reps": [round(x, 3) for x in ts]}
    return out


# ----------------------------------------------------------- CPU baseline


def cpu_step(oracle, frames, threads):
    """The step on the CPU by the oracle. Returns every output the device
    step produces: the MB-padded ALTREF anchor, the MB decisions, the qi-44
    reconstruction, the MBs' loop-filter records, the 64 x 8 candidate table
    and the walk's (level, sharpness)."""
    import vp8a

    anchor = oracle.build_arnr_altref([frames[9 + i] for i in range(LOOKAHEAD)], 3, 3, threads=threads)
    refs = [pad_planes(frames[7]), pad_planes(frames[0]), pad_planes(anchor)]
    lam = oracle.rd_lambda(QI)
    dec = oracle.analyse_inter_frame(frames[8], refs, [1, 2, 3], lam, threads=threads)
    recon = tuple(np.zeros_like(p) for p in refs[0])
    mbs = np.zeros(N_MB, vp8a.abi.MB_LF_INFO_DTYPE)
    oracle.reconstruct_inter_frame(frames[8], refs, [1, 2, 3], dec, vp8a.abi.quant_indices(QI), recon, lf_info=mbs,
                                   threads=threads)
    table = oracle.filter_sweep(recon, mbs, vp8a.abi.filter_config(0, 0), frames[8], 0, threads=threads)
    return {"altref": refs[2], "decisions": dec.reshape(-1), "recon": recon, "lf_info": mbs,
            "lf_table": table.reshape(-1), "lf_choice": select_full(table.reshape(-1), 0)}


def gpu_step_outputs(gs, choice):
    """The device step's outputs read back after its last run (same keys as
    cpu_step's)."""
    gs.ctx.synchronize()
    gs.torch.cuda.synchronize()
    abi = gs.abi
    return {"altref": tuple(p.cpu().numpy() for p in gs.alt),
            "decisions": np.frombuffer(gs.dec.cpu().numpy().tobytes(), abi.MB_DECISION_DTYPE),
            "recon": tuple(p.cpu().numpy() for p in gs.recon),
            "lf_info": np.frombuffer(gs.mbs.cpu().numpy().tobytes(), abi.MB_LF_INFO_DTYPE),
            "lf_table": gs.table.cpu().numpy().view(np.uint64).copy(), "lf_choice": tuple(choice)}


def step_parity(got, want):
    """Exact equality of the device step's outputs with the oracle's, per
    output: ALTREF planes, every decision field, the reconstruction planes,
    the loop-filter records, all 512 table entries (505 distinct candidates)
    and the selected (level, sharpness)."""
    dec_fields = [f for f in got["decisions"].dtype.names if f != "reserved"]
    lf_fields = [f for f in got["lf_info"].dtype.names if f != "reserved"]
    out = {
        "altref": all(np.array_equal(a, b) for a, b in zip(got["altref"], want["altref"])),
        "decisions": all(np.array_equal(got["decisions"][f], want["decisions"][f]) for f in dec_fields),
        "recon": all(np.array_equal(a, b) for a, b in zip(got["recon"], want["recon"])),
        "lf_info": all(np.array_equal(got["lf_info"][f], want["lf_info"][f]) for f in lf_fields),
        "lf_table": bool(np.array_equal(got["lf_table"], want["lf_table"])),
        "lf_choice": tuple(got["lf_choice"]) == tuple(want["lf_choice"]),
    }
    return all(out.values()), out


def cpu_baseline(frames, budget_s=30.0):
    """Times the oracle's step on all host threads (a bounded sample) and
    returns (baseline record, the first step's outputs)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.build()
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    n = 0
    first = None
    while True:
        out = cpu_step(oracle, frames, threads)
        first = first or out
        n += 1
        if time.perf_counter() - t0 > min(budget_s, 30.0) or n >= 3:
            break
    dt = time.perf_counter() - t0
    return {"value": round(N_MB * n / dt, 1), "unit": "MB/s", "cores": threads, "kind": "port",
            "sample": f"{n} full 1080p step(s) (ARNR + 3-ref analysis + qi-44 reconstruction + 505-candidate "
                      f"LF sweep) by the C oracle on {threads} threads in {dt:.2f} s",
            "note": "a scalar C restatement of the reference's algorithm on the 64x8 grid (505 candidates); the "
                    "reference's own walk scores ~24 candidates and its nightly SIMD kernels are not in the port",
            "cpu_model": cpu_model()}, first


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.build()
    frames, digest = make_inputs(SEED)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_step(oracle, frames, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_step(oracle, frames, threads)
    dt = time.perf_counter() - t0
    value = N_MB * args.steps / dt
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 1),
        "unit": "MB/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(dt * 1000.0 / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic (seeded gratings + quarter-pel six-tap translation + noise)",
        "config": {"workload": WORKLOAD, "width": W, "height": H, "refs": 3, "lookahead": LOOKAHEAD,
                   "lf_candidates": 512, "qi": QI, "seed": SEED, "input_sha256": digest[:16]},
        "cpu_baseline": {"value": round(value, 1), "unit": "MB/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full 1080p steps after {args.warmup} warm-up, C oracle "
                                   f"(restatement of the Rust reference, which has no toolchain here) "
                                   f"on {threads} threads", "cpu_model": cpu_model()},
        "e2e": {"value": round(value, 1), "unit": "MB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def extra_case(ctx, gs, torch, case):
    """Single-kernel cases over the frame of a GpuStep: `me` (the batched
    motion descent, vp8a_motion_descent, every MB against LAST from the zero
    vector: diamond + half + quarter), `lp_windows` (the proposal's cost
    volumes of every MB against LAST) and `lp_bwd` (one 32 -> 32 conv layer's
    data and weight gradients over every MB's 32 x 32 map)."""
    import vp8a
    from vp8a import abi, learned
    from vp8a.frames import luma_ref

    lib = ctx._lib
    with torch.cuda.stream(gs.stream):
        xy = learned.all_mbs(MB_COLS, MB_ROWS)
        n = xy.shape[0]
        if case == "me":
            src = learned._source_mbs(gs.cur[0], xy, H, W)
            zero = torch.zeros((n, 2), dtype=torch.int16, device="cuda")
            outs = [torch.empty((n, 2), dtype=torch.int32, device="cuda") for _ in range(3)]
            ref = luma_ref(gs.last[0])

            def fn():
                st = lib.vp8a_motion_descent(ctx.handle, C.byref(ref), src.data_ptr(), xy.data_ptr(), zero.data_ptr(),
                                             8, n, outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr())
                assert st == 0, vp8a.load().vp8a_last_error()
            fn.keep = (src, zero, outs, ref)
        elif case == "lp_windows":
            out = torch.empty((n, 32, 32, 2), dtype=torch.bfloat16, device="cuda")
            s, r = luma_ref(gs.cur[0]), luma_ref(gs.last[0][:H, :W])

            def fn():
                st = lib.vp8a_lp_windows(ctx.handle, C.byref(s), C.byref(r), xy.data_ptr(), n, out.data_ptr())
                assert st == 0, vp8a.load().vp8a_last_error()
            fn.keep = (out, s, r)
        elif case == "lp_bwd":
            g = torch.Generator(device="cuda").manual_seed(5)
            x = torch.relu(torch.randn(n, 32, 32, 32, device="cuda", generator=g)).to(torch.bfloat16)
            wt = (torch.randn(32 * 9 * 32, device="cuda", generator=g) * 0.2).to(torch.bfloat16)
            dy = (torch.randn(n, 32, 32, 32, device="cuda", generator=g) * 0.01).to(torch.bfloat16)
            dx = torch.empty_like(x)
            gw = torch.zeros(32 * 9 * 32, device="cuda")
            gb = torch.zeros(32, device="cuda")

            def fn():
                st = lib.vp8a_lp_conv_backward(ctx.handle, x.data_ptr(), 32, wt.data_ptr(), 32, n, dy.data_ptr(), 1,
                                               dx.data_ptr(), gw.data_ptr(), gb.data_ptr())
                assert st == 0, vp8a.load().vp8a_last_error()
            fn.keep = (x, wt, dy, dx, gw, gb)
        else:
            raise ValueError(case)
    ctx.synchronize()
    return fn


def case_arm(args):
    """One stage alone on a WxH frame, for profiling captures: runs
    `--warmup` + `--steps` calls of the stage and prints its mean device ms."""
    import torch

    import vp8a
    from vp8a import synth

    w, h = (int(v) for v in args.size.split("x"))
    global W, H, MB_COLS, MB_ROWS, N_MB
    W, H = w, h
    MB_COLS, MB_ROWS = (w + 15) // 16, (h + 15) // 16
    N_MB = MB_COLS * MB_ROWS
    ctx = vp8a.Context(0)
    ctx.set_subpel_planes(args.subpel_planes)
    if args.lf_layout:
        ctx.force_sweep_layout(*(int(v) for v in args.lf_layout.split(",")))
    if args.case in ("predict_mb", "predict_split"):
        fn = batched_predict(ctx, vp8a, torch, args.case == "predict_split")
    else:
        frames, _ = synth.make_sequence(w, h, 16, SEED, pieces=4, occluders=4)
        gs = GpuStep(ctx, frames, vp8a.load(), torch, 0)
        if args.case == "trellis":
            ctx.set_trellis_strength(1.0)
        fn = {"arnr": gs.run_arnr, "analysis": gs.run_analysis, "lf": gs.run_lf, "predict": gs.run_predict,
              "recon": gs.run_recon, "trellis": gs.run_recon}.get(args.case) or extra_case(ctx, gs, torch, args.case)
    stream = torch.cuda.ExternalStream(ctx.stream)
    for _ in range(args.warmup):
        fn()
    ctx.synchronize()
    ts = []
    for _ in range(args.steps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        fn()
        e.record(stream)
        e.synchronize()
        ts.append(s.elapsed_time(e))
    ctx.close()
    return {"case": args.case, "size": args.size, "ms": [round(x, 4) for x in ts]}


# ------------------------------------------------- batched streams case

BATCH_RESOLUTIONS = [(176, 144), (640, 360), (1280, 720), (1920, 1080), (3840, 2160)]
BATCH_LOOKAHEAD = 5


class BatchStep:
    """The batched plain path over many independent streams of uneven size:
    per stream one P frame analysed against LAST (the previous frame) and
    ALTREF (the ARNR anchor of a 5-frame lookahead, centre anchor), its
    qi-44 reconstruction and the 64 x 8 loop-filter sweep over it. Each
    stage of all streams is one call of the batched entry points
    (vp8a_build_arnr_altrefs_planes, vp8a_analyse_inter_frames,
    vp8a_reconstruct_inter_frames, vp8a_filter_sweeps) on device-resident
    buffers."""

    def __init__(self, ctx, streams, torch):
        import vp8a
        from vp8a import abi

        self.vp8a, self.abi, self.ctx, self.torch = vp8a, abi, ctx, torch
        self.stream = torch.cuda.ExternalStream(ctx.stream)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
        self.keep = []
        self.s = []
        for frames in streams:
            h, w = frames[0][0].shape
            mbc, mbr = (w + 15) // 16, (h + 15) // 16
            st = {"w": w, "h": h, "mbs": mbc * mbr}
            st["cur"] = [t(p) for p in frames[1]]
            st["last"] = [t(p) for p in pad_planes(frames[0])]
            st["win"] = [[t(p) for p in f] for f in frames[2:2 + BATCH_LOOKAHEAD]]
            st["alt"] = [torch.zeros_like(p) for p in st["last"]]
            st["recon"] = [torch.zeros_like(p) for p in st["last"]]
            st["lf"] = torch.zeros(st["mbs"] * abi.MB_LF_INFO_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
            st["dec"] = torch.zeros(st["mbs"] * abi.MB_DECISION_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
            self.s.append(st)
        self.tables = torch.zeros((len(streams), 512), dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        ids = np.array([abi.REF_LAST, abi.REF_ALTREF], np.uint8)
        self.ctxs = abi.default_mv_contexts()
        lam = vp8a.rd_lambda(QI)
        aj, anj, rj, sj = [], [], [], []
        for i, st in enumerate(self.s):
            win = (abi.I420 * BATCH_LOOKAHEAD)(*[vp8a.i420(*f) for f in st["win"]])
            refs = (abi.Planes * 2)(vp8a.planes(*st["last"]), vp8a.planes(*st["alt"]))
            self.keep += [win, refs]
            aj.append(abi.ArnrPlanesJob(C.cast(win, C.c_void_p), BATCH_LOOKAHEAD, BATCH_LOOKAHEAD // 2, 3,
                                        vp8a.planes(*st["alt"])))
            cur = vp8a.i420(*st["cur"])
            anj.append(abi.AnalysisJob(cur, C.cast(refs, C.c_void_p), ids.ctypes.data, 2,
                                       C.cast(C.pointer(self.ctxs), C.c_void_p), lam, st["dec"].data_ptr(), None))
            rj.append(abi.ReconJob(cur, C.cast(refs, C.c_void_p), ids.ctypes.data, 2, 0, st["dec"].data_ptr(),
                                   abi.quant_indices(QI), None, None, 0, abi.FILTER_SIXTAP, vp8a.planes(*st["recon"]),
                                   None, None, st["lf"].data_ptr()))
            sj.append(abi.SweepJob(vp8a.planes(*st["recon"]), st["lf"].data_ptr(), abi.filter_config(0, 0),
                                   vp8a.source(*st["cur"]), 0, self.tables[i].data_ptr()))
        self.ids = ids
        self.jobs = {k: (type(v[0]) * len(v))(*v) for k, v in
                     (("arnr", aj), ("analysis", anj), ("recon", rj), ("lf", sj))}
        self.n_mb = sum(st["mbs"] for st in self.s)

    def _call(self, fn, key):
        arr = self.jobs[key]
        st = getattr(self.ctx._lib, fn)(self.ctx.handle, C.cast(arr, C.c_void_p), len(arr))
        assert st == 0, self.vp8a.load().vp8a_last_error()

    def run_arnr(self):
        # Every stream's anchor straight into its MB-padded ALTREF planes.
        self._call("vp8a_build_arnr_altrefs_planes", "arnr")

    def run_analysis(self):
        self._call("vp8a_analyse_inter_frames", "analysis")

    def run_recon(self):
        self._call("vp8a_reconstruct_inter_frames", "recon")

    def run_lf(self):
        self._call("vp8a_filter_sweeps", "lf")
        self.ctx.synchronize()
        t = self.tables.cpu().numpy().view(np.uint64)
        return [select_full(row, 0) for row in t]

    def step(self):
        self.run_arnr()
        self.run_analysis()
        self.run_recon()
        return self.run_lf()


def batch_streams(n_streams, seed):
    """`n_streams` streams with resolutions drawn from BATCH_RESOLUTIONS by
    `seed`; each stream is 2 + BATCH_LOOKAHEAD consecutive frames of one
    seeded sequence per resolution (streams of one resolution start at
    different frames)."""
    from vp8a import synth

    rng = np.random.default_rng(seed)
    pick = rng.integers(0, len(BATCH_RESOLUTIONS), n_streams)
    need = 2 + BATCH_LOOKAHEAD
    seqs = {}
    for r in sorted(set(int(x) for x in pick)):
        w, h = BATCH_RESOLUTIONS[r]
        seqs[r], _ = synth.make_sequence(w, h, need - 1 + int((pick == r).sum()), seed + 17 * r, pieces=4,
                                         occluders=4)
    used = {r: 0 for r in seqs}
    streams = []
    for r in pick:
        r = int(r)
        streams.append(seqs[r][used[r]:used[r] + need])
        used[r] += 1
    return streams, pick


def batch_arm(args):
    """The batched plain path (48 streams of uneven size by default): MBs
    per second through ARNR + analysis + reconstruction + LF sweep, every
    stage one batched launch, inputs resident on the device, L2 flushed
    between timed steps."""
    import torch

    import vp8a

    streams, pick = batch_streams(args.streams, SEED)
    ctx = vp8a.Context(0)
    bs = BatchStep(ctx, streams, torch)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = bs.stream
    for _ in range(args.warmup):
        bs.step()
    ctx.synchronize()
    ts = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        bs.step()
        e.record(stream)
        e.synchronize()
        ts.append(s.elapsed_time(e))
    stages = {}
    for name in ("arnr", "analysis", "recon", "lf"):
        fn = getattr(bs, "run_" + name)
        xs = []
        for _ in range(3):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            e.synchronize()
            xs.append(s.elapsed_time(e))
        stages[name] = round(float(np.median(xs)), 3)
    mixed_layout = ctx.last_sweep_layout()
    ms = float(np.median(ts))
    n_mb = bs.n_mb
    # Each resolution's streams as a batch of their own: MB/s and each
    # stage's algorithmic GB/s (per MB: ARNR 6 frames x 384 B in + 384 out;
    # analysis source 256 + 2 refs x 256 + decision 104; reconstruction
    # 1264; LF sweep 774 read once), with the launch shape the sweep's
    # autotuner picked for that batch.
    per_alg = {"arnr": (BATCH_LOOKAHEAD + 1) * 384, "analysis": 256 + 2 * 256 + 104, "recon": 1264, "lf": 774}
    per_res = {}
    del bs
    for r in sorted(set(int(x) for x in pick)):
        sub = [s_ for s_, p_ in zip(streams, pick) if int(p_) == r]
        rb = BatchStep(ctx, sub, torch)
        for _ in range(args.warmup):
            rb.step()
        ctx.synchronize()
        rts = []
        for _ in range(max(3, args.steps // 2)):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            torch.cuda.synchronize()
            s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_.record(stream)
            rb.step()
            e_.record(stream)
            e_.synchronize()
            rts.append(s_.elapsed_time(e_))
        st_ms = {}
        for name in ("arnr", "analysis", "recon", "lf"):
            fn = getattr(rb, "run_" + name)
            xs = []
            for _ in range(3):
                with torch.cuda.stream(stream):
                    flush.fill_(1)
                torch.cuda.synchronize()
                s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s_.record(stream)
                fn()
                e_.record(stream)
                e_.synchronize()
                xs.append(s_.elapsed_time(e_))
            st_ms[name] = float(np.median(xs))
        rms = float(np.median(rts))
        lay = ctx.last_sweep_layout()
        per_res["%dx%d" % BATCH_RESOLUTIONS[r]] = {
            "streams": len(sub), "mbs": rb.n_mb, "ms_per_step": round(rms, 3),
            "mbs_per_s": round(rb.n_mb / (rms / 1e3), 1),
            "stage_ms": {k: round(v, 3) for k, v in st_ms.items()},
            "stage_gbs": {k: round(rb.n_mb * per_alg[k] / (v / 1e3) / 1e9, 2) for k, v in st_ms.items()},
            "lf_layout": {"passes_per_cta": lay[0], "threads_per_cta": lay[1], "prefetch": bool(lay[2]),
                          "ctas_per_sm": lay[3]}}
        del rb
    ctx.close()
    return {"case": "batch", "metric": "MBs/s (ARNR+ME+recon+LF search), batched streams", "unit": "MB/s",
            "value": round(n_mb / (ms / 1e3), 1), "ms_per_step": round(ms, 3), "steps": args.steps,
            "warmup": args.warmup, "streams": args.streams, "mbs_per_step": n_mb, "per_resolution": per_res,
            "lf_layout_mixed": {"passes_per_cta": mixed_layout[0], "threads_per_cta": mixed_layout[1],
                                "prefetch": bool(mixed_layout[2]), "ctas_per_sm": mixed_layout[3],
                                "chosen_by": "autotune (timed on the first batch of these picture shapes)"},
            "stage_ms": stages, "step_ms": [round(x, 3) for x in ts],
            "config": {"workload": "%d streams from {176x144, 640x360, 1280x720, 1920x1080, 3840x2160}: "
                                   "P frame vs LAST/ALTREF, ARNR(5, centre), qi-44 reconstruction, LF 64x8 sweep"
                                   % args.streams, "seed": SEED, "l2": "flushed between timed steps (256 MiB write)"}}


# --------------------------------------------------- learned proposal case

def train_proposal_net(ctx, train_steps):
    """The learned proposal's net, trained (untimed) on ~200k labels: the
    plain search's LAST-reference vectors over 24 seeded 1080p frame pairs
    (gratings, noise, piecewise motion, moving occluders), Adam, lr 1e-3,
    batches of 4096 MBs. Returns (net, stats)."""
    import torch

    from vp8a import learned, synth

    lam = __import__("vp8a").rd_lambda(QI)
    t0 = time.time()
    xs, ys = [], []
    with learned.on_ctx_stream(ctx):
        for sidx in range(4):
            frames, _ = synth.make_sequence(W, H, 7, SEED + 1000 + sidx, pieces=4, occluders=4)
            for k in range(1, 7):
                ref = pad_planes(frames[k - 1])
                lab, _ = learned.labels_from_search(ctx, frames[k], ref, lam)
                xy = learned.all_mbs(MB_COLS, MB_ROWS)
                src = torch.from_numpy(frames[k][0]).cuda()
                refy = torch.from_numpy(ref[0]).cuda()
                xs.append(learned.windows(ctx, src, refy[:H, :W], xy))
                ys.append(torch.from_numpy(lab).cuda())
        x = torch.cat(xs)
        y = torch.cat(ys)
    ctx.synchronize()
    t_labels = time.time() - t0
    net = learned.ProposalNet(ctx, seed=7)
    g = torch.Generator().manual_seed(5)
    n = x.shape[0]
    losses = []
    t1 = time.time()
    for it in range(train_steps):
        with learned.on_ctx_stream(ctx):
            idx = torch.randint(0, n, (4096,), generator=g).cuda()
            xb, yb = x[idx].contiguous(), y[idx].contiguous()
        losses.append(net.train_step(xb, yb, lr=1e-3))
    ctx.synchronize()
    t_train = time.time() - t1
    with learned.on_ctx_stream(ctx):
        cells = net.propose(x[:65536], 4)
        top4 = float(((cells == y[:65536, None].long()).any(1) & (y[:65536] >= 0)).float().sum() /
                     (y[:65536] >= 0).sum())
    del x, y, xs, ys
    return net, {"labels": int(n), "losses": losses, "top4": top4, "label_s": t_labels, "train_s": t_train}


def learned_arm(args):
    """The learned motion proposal at 1080p (the survey's config 4): the net
    is trained (untimed) on ~200k labels — the plain search's LAST-reference
    vectors over 24 seeded 1080p frame pairs (gratings, noise, piecewise
    motion, moving occluders) — with Adam, lr 1e-3, batches of 4096 MBs;
    then, on the bench's P frame, the learned search (proposal + exact
    +-2 px search around 4 seeds + sub-pel + descent fallback) for LAST,
    GOLDEN and ALTREF is timed against the plain exhaustive analysis of the
    same frame and references. Quality: mean SAD per reference against the
    plain search's own per-reference result."""
    import torch

    import vp8a
    from vp8a import abi, learned, synth

    ctx = vp8a.Context(0)
    lam = vp8a.rd_lambda(QI)
    net, tstats = train_proposal_net(ctx, args.train_steps)
    n, losses, top4 = tstats["labels"], tstats["losses"], tstats["top4"]
    t_labels, t_train = tstats["label_s"], tstats["train_s"]
    # Loop-filter window head: the plain path's level choice on training
    # frames at several quantisers (reconstruction + full sweep + walk).
    head = learned.LfWindowHead(ctx, seed=3)
    sample = learned.sample_mbs(MB_COLS, MB_ROWS, 256, seed=1)
    lf_frames, lf_levels = [], []
    qis = [24, 44, 64, 100]
    for sidx in range(4):
        frames_t, _ = synth.make_sequence(W, H, 7, SEED + 1000 + sidx, pieces=4, occluders=4)
        for k in range(1, 7):
            qi = qis[(sidx * 6 + k) % len(qis)]
            ref = pad_planes(frames_t[k - 1])
            dec = vp8a.analyse_inter_frame(ctx, frames_t[k], [ref], [abi.REF_LAST], vp8a.rd_lambda(qi))
            rec = tuple(np.array(p_) for p_ in ref)
            lfi = np.zeros(N_MB, abi.MB_LF_INFO_DTYPE)
            vp8a.reconstruct_inter_frame(ctx, frames_t[k], [ref], [abi.REF_LAST], dec, abi.quant_indices(qi), rec,
                                         lf_info=lfi)
            tab = vp8a.filter_sweep(ctx, rec, lfi, abi.filter_config(0, 0), frames_t[k])
            level, _ = select_full(tab.reshape(-1), 0)
            with learned.on_ctx_stream(ctx):
                src_t = torch.from_numpy(frames_t[k][0]).cuda()
                ref_t = torch.from_numpy(ref[0]).cuda()
            sums, count = head.features(net, src_t, ref_t, sample, qi)
            lf_frames.append((sums, count, level))
            lf_levels.append(int(level))
    head_losses = [head.train_step(lf_frames, lr=1e-2) for _ in range(200)]
    head_hits = sum(1 for (sm_, ct_, lv_) in lf_frames if head.window(sm_, ct_)[0] <= lv_ <= head.window(sm_, ct_)[1])
    # The bench's P frame and references.
    frames, _ = make_inputs(SEED)
    gs = GpuStep(ctx, frames, vp8a.load(), torch, 0)
    with learned.on_ctx_stream(ctx):
        src = gs.cur[0]
        refs = [gs.last[0], gs.golden[0], gs.alt[0]]
        xy = learned.all_mbs(MB_COLS, MB_ROWS)
    ctx.synchronize()
    stream = gs.stream

    def learned_step():
        return [learned.learned_search(ctx, net, src, r, xy) for r in refs]

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        ctx.synchronize()
        ts = []
        for _ in range(steps):
            torch.cuda.synchronize()
            s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_.record(stream)
            fn()
            e_.record(stream)
            e_.synchronize()
            ts.append(s_.elapsed_time(e_))
        return float(np.median(ts)), ts

    ms_learned, ts_l = timed(learned_step, args.steps, args.warmup)
    ms_plain, ts_p = timed(gs.run_analysis, args.steps, args.warmup)
    # Per-stage device time of one learned frame (3 references), CUDA events
    # on the library stream: the gaps between stages (host orchestration)
    # fall into the stage that follows them.
    stage_ms = {}
    for r in refs:
        learned.learned_search(ctx, net, src, r, xy, timings=stage_ms)
    stage_ms = {k_: round(v_, 4) for k_, v_ in stage_ms.items()}
    # The full step with the learned loop-filter window: ARNR, the plain
    # analysis and reconstruction, the head's window from 256 sampled MBs
    # (net layers 1-3 against LAST), the sweep over level 0 and the window's
    # 9 levels, the reference's walk over that table.
    win_tab = torch.zeros(512, dtype=torch.int64, device="cuda")
    choice = {}

    def window_step():
        gs.run_arnr()
        gs.run_analysis()
        gs.run_recon()
        sums, count = head.features(net, src, refs[0], sample, QI)
        lo, hi = head.window(sums, count)
        st_ = gs.lib.vp8a_filter_sweep_window(ctx.handle, C.byref(gs.recon_planes), gs.mbs.data_ptr(),
                                              C.byref(gs.base), C.byref(gs.src), lo, hi, win_tab.data_ptr())
        assert st_ == 0, vp8a.load().vp8a_last_error()
        ctx.synchronize()
        choice["window"] = (lo, hi)
        choice["learned"] = select_full(win_tab.cpu().numpy().view(np.uint64), 0)

    def plain_step():
        choice["plain"] = gs.step()

    ms_wstep, ts_w = timed(window_step, args.steps, args.warmup)
    ms_pstep, ts_ps = timed(plain_step, args.steps, args.warmup)
    # Quality against the plain search's per-reference results (trace).
    res = learned_step()
    plain_sad = []
    for rp in (gs.last, gs.golden, gs.alt):
        planes_np = tuple(p.cpu().numpy() for p in rp)
        _, tr = vp8a.analyse_inter_frame(ctx, frames[8], [planes_np], [abi.REF_LAST], lam, trace=True)
        plain_sad.append(tr[..., 0]["quarter"]["sad"].reshape(-1).astype(np.float64))
    ratio = [float(np.asarray(o[1], np.float64).mean() / ps.mean()) for o, ps in zip(res, plain_sad)]
    fb = [float(np.mean(o[2])) for o in res]
    rd = learned_rd(ctx, net, head, sample)
    ctx.close()
    return {"case": "learned", "size": "%dx%d" % (W, H), "unit": "MB/s",
            "learned_me_mbs_per_s": round(N_MB / (ms_learned / 1e3), 1), "learned_me_ms": round(ms_learned, 3), "learned_stage_ms": stage_ms,
            "plain_analysis_mbs_per_s": round(N_MB / (ms_plain / 1e3), 1), "plain_analysis_ms": round(ms_plain, 3),
            "speedup_vs_plain_analysis": round(ms_plain / ms_learned, 2),
            "mean_sad_ratio_vs_plain_per_ref": [round(v, 4) for v in ratio],
            "fallback_rate_per_ref": [round(v, 4) for v in fb],
            "training": {"labels": int(n), "steps": args.train_steps, "batch": 4096, "lr": 1e-3,
                         "first_loss": round(float(np.mean(losses[:5])), 4),
                         "last_loss": round(float(np.mean(losses[-5:])), 4), "top4_label_hit": round(top4, 4),
                         "label_s": round(t_labels, 1), "train_s": round(t_train, 1)},
            "learned_ms": [round(v, 3) for v in ts_l], "plain_ms": [round(v, 3) for v in ts_p],
            "lf_window": {"step_ms_learned_window": round(ms_wstep, 3), "step_ms_plain": round(ms_pstep, 3),
                          "step_mbs_per_s_learned_window": round(N_MB / (ms_wstep / 1e3), 1),
                          "step_mbs_per_s_plain": round(N_MB / (ms_pstep / 1e3), 1),
                          "speedup": round(ms_pstep / ms_wstep, 2), "window": list(choice["window"]),
                          "choice_learned": list(choice["learned"]), "choice_plain": list(choice["plain"]),
                          "train_frames": len(lf_frames), "train_levels": sorted(set(lf_levels)),
                          "train_window_hits": head_hits, "head_loss_first_last": [round(head_losses[0], 4),
                                                                                    round(head_losses[-1], 4)]},
            "rd": rd,
            "note": "learned = proposal net + exact +-2 px search at 4 seeds + sub-pel + descent fallback, 3 refs, "
                    "per-reference vectors; plain = the exhaustive analysis (census, SPLITMV, RD decision) of the "
                    "same frame and references"}


STREAM_SIZES = [(3840, 2160)] * 8 + [(1280, 720)] * 8
STREAM_GROUP = 15


def stream_learned(ctx, torch, sizes, frames, g, train_steps):
    """The learned proposal on the altref stream path (the survey's config
    5): every coded frame of every stream gets, per reference, the learned
    search's vector (net proposal, exact +-2 px search around 4 seeds,
    sub-pel, descent fallback) as a second NEWMV candidate of the batched
    exhaustive analysis; the plain path is the same pipeline without it.
    One group after the opening one, on the same inputs for both: wall time
    per group with the bitstream writer off (the learned searches run one
    frame and reference at a time), then bytes and luma PSNR per resolution
    with the writer on, and the fallback rate of the learned searches."""
    from vp8a import abi, learned
    from vp8a.stream import AltrefStreams

    net, tstats = train_proposal_net(ctx, train_steps)
    xy_cache, fbs = {}, []

    def proposer(streams, srcs):
        out = []
        for st, src in zip(streams.s, srcs):
            key = (st.mb_cols, st.mb_rows)
            if key not in xy_cache:
                xy_cache[key] = learned.all_mbs(st.mb_cols, st.mb_rows)
            p = np.zeros((st.n_mb, 3), abi.MV_DTYPE)
            for k, ref in enumerate((st.last, st.golden, st.altref)):
                mv, _, fb = learned.learned_search(ctx, net, src[0], ref[0], xy_cache[key])
                p["row"][:, k] = mv[:, 0]
                p["col"][:, k] = mv[:, 1]
                fbs.append(float(fb.mean()))
            out.append(p)
        return out

    mbs_group = sum(((w + 15) // 16) * ((h + 15) // 16) for w, h in sizes) * g
    res = {}
    for mode in ("plain", "learned"):
        prop = proposer if mode == "learned" else None
        for write in (False, True):
            streams = AltrefStreams(ctx, sizes, qi=QI, strength=3, write=write)
            for gi in range(2):  # the first group opens the streams
                grp = [f[gi * g:(gi + 1) * g] for f in frames]
                ctx.synchronize()
                t = time.perf_counter()
                pk = streams.encode_group(grp, proposer=prop, psnr=write)
                ctx.synchronize()
                dt = time.perf_counter() - t
            if not write:
                res[mode] = {"group_s": round(dt, 3), "mbs_per_s_wall": round(mbs_group / dt, 1)}
                continue
            by_res = {}
            for (w, h), packets in zip(sizes, pk):
                d = by_res.setdefault("%dx%d" % (w, h), {"bytes": 0, "psnr": []})
                d["bytes"] += sum(len(q["bytes"]) for q in packets if q["bytes"] is not None)
                d["psnr"] += [q["psnr_y"] for q in packets if "psnr_y" in q]
            res[mode]["by_res"] = by_res
            del streams
    out = {}
    for r in res["plain"]["by_res"]:
        a, b = res["plain"]["by_res"][r], res["learned"]["by_res"][r]
        out[r] = {"plain_bytes": a["bytes"], "learned_bytes": b["bytes"],
                  "byte_delta_pct": round(100.0 * (b["bytes"] - a["bytes"]) / a["bytes"], 3),
                  "plain_psnr_y": round(float(np.mean(a["psnr"])), 3), "learned_psnr_y": round(float(np.mean(b["psnr"])), 3),
                  "psnr_delta_db": round(float(np.mean(b["psnr"]) - np.mean(a["psnr"])), 3)}
    return {"per_resolution": out, "plain_group_s": res["plain"]["group_s"],
            "learned_group_s": res["learned"]["group_s"],
            "plain_mbs_per_s_wall": res["plain"]["mbs_per_s_wall"],
            "learned_mbs_per_s_wall": res["learned"]["mbs_per_s_wall"],
            "fallback_rate": round(float(np.mean(fbs)), 4) if fbs else None,
            "net": {"labels": tstats["labels"], "top4_label_hit": round(tstats["top4"], 4)},
            "note": "one group after the opening one; wall time with the writer off; the proposals are not "
                    "fused into the batched analysis launch (one learned search per frame and reference)"}


def stream_arm(args):
    """The lagged altref stream path of the survey's config 5: 8 streams at
    3840x2160 and 8 at 1280x720 in lockstep, 15-frame lookahead groups, each
    group an invisible ARNR anchor (centre = the group's last frame) coded
    against LAST / GOLDEN / ALTREF and then its P frames, all with the
    automatic loop-filter pick and the filtered pictures as the next
    references (vp8a.stream.AltrefStreams: every stage of all 16 streams one
    batched call). Timed: groups after the first (the first opens the
    streams), device time per group with inputs resident; MB/s counts every
    coded MB (anchors and P frames). Bytes and PSNR come from one further
    group with the host bitstream writer on, untimed."""
    import torch

    import vp8a
    from vp8a import synth
    from vp8a.stream import AltrefStreams

    sizes = STREAM_SIZES[: args.streams] if args.streams < len(STREAM_SIZES) else STREAM_SIZES
    g = STREAM_GROUP
    n_groups = 2 + args.steps
    need = g * n_groups
    seqs = {}
    for (w, h) in sorted(set(sizes)):
        seqs[(w, h)], _ = synth.make_sequence(w, h, need + 7, SEED + w, pieces=4, occluders=4)
    ctx = vp8a.Context(0)
    dev = torch.device("cuda", 0)
    frames = []
    for i, (w, h) in enumerate(sizes):
        off = i % 8
        frames.append([tuple(torch.from_numpy(np.ascontiguousarray(p)).to(dev) for p in f)
                       for f in seqs[(w, h)][off:off + need]])
    torch.cuda.synchronize()
    streams = AltrefStreams(ctx, sizes, qi=QI, strength=3, write=False)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    mbs_group = sum(((w + 15) // 16) * ((h + 15) // 16) for w, h in sizes) * g  # anchor + (g - 1) P frames
    ts = []
    for gi in range(n_groups - 1):
        grp = [f[gi * g:(gi + 1) * g] for f in frames]
        ctx.synchronize()
        s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_.record(stream)
        streams.encode_group(grp)
        e_.record(stream)
        e_.synchronize()
        ts.append(s_.elapsed_time(e_))
    timed = ts[1:]  # the first group opens the streams (no anchor context before it)
    ms = float(np.median(timed))
    # Bytes and luma PSNR of one more group, writer on.
    streams.write = True
    gi = n_groups - 1
    grp = [f[gi * g:(gi + 1) * g] for f in frames]
    packets = streams.encode_group(grp)
    by_res = {}
    for (w, h), pk in zip(sizes, packets):
        d = by_res.setdefault("%dx%d" % (w, h), {"streams": 0, "bytes_per_group": 0, "levels": []})
        d["streams"] += 1
        d["bytes_per_group"] += sum(len(p["bytes"]) for p in pk if p["bytes"] is not None)
        d["levels"] += [p["level"] for p in pk]
    for d in by_res.values():
        d["bytes_per_group"] //= d["streams"]
        d["mean_level"] = round(float(np.mean(d.pop("levels"))), 2)
    learned_res = stream_learned(ctx, torch, sizes, frames, g, args.train_steps) if args.stream_learned else None
    ctx.close()
    return {"case": "stream", "unit": "MB/s", "streams": len(sizes), "sizes": sorted(set("%dx%d" % s for s in sizes)),
            "group": g, "qi": QI, "value": round(mbs_group / (ms / 1e3), 1), "ms_per_group": round(ms, 2),
            "mbs_per_group": mbs_group, "group_ms": [round(x, 2) for x in ts], "per_resolution": by_res,
            "config": {"workload": "8x3840x2160 + 8x1280x720 altref streams, 15-frame groups: ARNR anchor + 14 P "
                                   "frames per group, exhaustive 3-ref analysis, qi-44 reconstruction, auto-LF "
                                   "(reference walk) and filter on every coded frame", "seed": SEED,
                       "timed": "device time per group after the first, inputs resident"}, "learned": learned_res}


def rd_arm(args):
    """The RD-effort inter search (decide_mb_rd's search, the stream
    encoder's per-MB inter search) over the bench's 1080p P frame against
    LAST / GOLDEN / ALTREF, census neighbours from the plain analysis's
    decisions, qi 44: device time per effort level (CUDA events on the
    context stream, every buffer device-resident, L2 flushed between
    calls) and MB/s."""
    import torch

    import vp8a
    from vp8a import abi

    ctx = vp8a.Context(0)
    frames, _ = make_inputs(SEED)
    gs = GpuStep(ctx, frames, vp8a.load(), torch, 0)
    ctx.synchronize()
    dec = np.frombuffer(gs.dec.cpu().numpy().tobytes(), abi.MB_DECISION_DTYPE).reshape(MB_ROWS, MB_COLS)
    nb = vp8a.neighbours_from_decisions(dec)
    with torch.cuda.stream(gs.stream):
        dnb = torch.from_numpy(nb.view(np.uint8).copy()).cuda()
        out = torch.zeros(N_MB * abi.RD_INTER_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    ctx.synchronize()
    y1_ac = vp8a.dequant_factors(gs.quant)[1]
    f = vp8a.i420(*gs.cur)
    pl = (abi.Planes * 3)(vp8a.planes(*gs.last), vp8a.planes(*gs.golden), vp8a.planes(*gs.alt))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    res = {}
    for effort, name in enumerate(("fastest", "fast", "balanced", "thorough")):
        def call():
            st = ctx._lib.vp8a_rd_inter_search(ctx.handle, C.byref(f), C.cast(pl, C.c_void_p), gs.host_ids.ctypes.data,
                                               3, C.byref(gs.ctxs), gs.lam, y1_ac, effort, dnb.data_ptr(),
                                               out.data_ptr())
            assert st == 0, vp8a.load().vp8a_last_error()
        for _ in range(args.warmup):
            call()
        ctx.synchronize()
        ts = []
        for _ in range(args.steps):
            with torch.cuda.stream(gs.stream):
                flush.fill_(1)
            s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_.record(gs.stream)
            call()
            e_.record(gs.stream)
            e_.synchronize()
            ts.append(s_.elapsed_time(e_))
        ms = float(np.median(ts))
        o = np.frombuffer(out.cpu().numpy().tobytes(), abi.RD_INTER_DTYPE)
        res[name] = {"ms": round(ms, 4), "mbs_per_s": round(N_MB / (ms / 1e3), 1),
                     "mean_refs_searched": round(float(o["n_searched"].mean()), 3),
                     "mean_sad": round(float(o["sad"].mean()), 1)}
    ms_plain = None
    ts = []
    for _ in range(args.steps):
        with torch.cuda.stream(gs.stream):
            flush.fill_(1)
        s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_.record(gs.stream)
        gs.run_analysis()
        e_.record(gs.stream)
        e_.synchronize()
        ts.append(s_.elapsed_time(e_))
    ms_plain = float(np.median(ts))
    del out, dnb, flush
    ctx.close()
    return {"case": "rd", "size": "%dx%d" % (W, H), "unit": "MB/s", "qi": QI, "y1_ac": int(y1_ac), "refs": 3,
            "efforts": res, "exhaustive_analysis_ms": round(ms_plain, 4),
            "note": "RD-effort inter search per MB given its census neighbours (one warp per MB, no wavefront); "
                    "the exhaustive analysis (the metric's search) timed beside it"}


def psnr_y(a, b):
    d = a.astype(np.float64) - b.astype(np.float64)
    mse = float(np.mean(d * d))
    return 99.0 if mse == 0 else 10.0 * np.log10(255.0 * 255.0 / mse)


def learned_rd(ctx, net, head, sample, n_seq=2):
    """Bytes and PSNR of whole P-frame encodes (analysis, qi reconstruction,
    automatic loop filter, bitstream) with and without the learned
    proposals, on held-out 1080p frames (seeds not used in training: frame
    8 against LAST = 7, GOLDEN = 0 and the ARNR anchor of frames 9-15) at
    qi 24 / 44 / 64. "learned" passes each reference's learned-search vector
    as a second NEWMV candidate to the exhaustive decision. Also: whether
    the learned loop-filter window holds the plain path's level on those
    frames, counting the frames whose plain level is not 0."""
    import torch

    import vp8a
    from vp8a import abi, learned, synth

    held = []
    for sidx in range(n_seq):
        fr, _ = synth.make_sequence(W, H, 16, SEED + 5000 + sidx, pieces=4, occluders=4)
        anchor = vp8a.build_arnr_altref_planes(ctx, [fr[9 + i] for i in range(LOOKAHEAD)], 3, 3)
        held.append((fr[8], [pad_planes(fr[7]), pad_planes(fr[0]), anchor]))
    xy = learned.all_mbs(MB_COLS, MB_ROWS)
    props, t_learn = [], []
    for cur, refs in held:
        with learned.on_ctx_stream(ctx):
            src = torch.from_numpy(cur[0]).cuda()
            rts = [torch.from_numpy(r[0]).cuda() for r in refs]
        ctx.synchronize()
        t0 = time.perf_counter()
        res = [learned.learned_search(ctx, net, src, r, xy) for r in rts]
        t_learn.append(time.perf_counter() - t0)
        p = np.zeros((N_MB, 3), abi.MV_DTYPE)
        for k, (mv, _, _) in enumerate(res):
            p["row"][:, k] = mv[:, 0]
            p["col"][:, k] = mv[:, 1]
        props.append(p)
    out = {}
    window_hits, window_n = 0, 0
    for qi in (24, 44, 64):
        acc = {m: {"bytes": 0, "psnr": [], "levels": []} for m in ("plain", "learned")}
        for (cur, refs), p in zip(held, props):
            for mode, pr in (("plain", None), ("learned", p)):
                bits, filt, det = vp8a.encode_p_frame(ctx, cur, refs, [1, 2, 3], qi, proposals=pr)
                acc[mode]["bytes"] += len(bits)
                acc[mode]["psnr"].append(psnr_y(filt[0][:H, :W], cur[0]))
                acc[mode]["levels"].append(int(det["level"]))
                if mode == "plain" and det["level"] != 0:
                    with learned.on_ctx_stream(ctx):
                        s_t = torch.from_numpy(cur[0]).cuda()
                        r_t = torch.from_numpy(refs[0][0]).cuda()
                    sums, count = head.features(net, s_t, r_t, sample, qi)
                    lo, hi = head.window(sums, count)
                    window_n += 1
                    window_hits += int(lo <= det["level"] <= hi)
        pb, lb = acc["plain"]["bytes"], acc["learned"]["bytes"]
        out["qi%d" % qi] = {
            "plain_bytes": pb, "learned_bytes": lb, "byte_delta_pct": round(100.0 * (lb - pb) / pb, 3),
            "plain_psnr_y": round(float(np.mean(acc["plain"]["psnr"])), 3),
            "learned_psnr_y": round(float(np.mean(acc["learned"]["psnr"])), 3),
            "psnr_delta_db": round(float(np.mean(acc["learned"]["psnr"]) - np.mean(acc["plain"]["psnr"])), 3),
            "levels_plain": acc["plain"]["levels"], "levels_learned": acc["learned"]["levels"]}
    out["frames"] = len(held)
    out["learned_search_s_per_frame"] = round(float(np.mean(t_learn)), 4)
    out["lf_window_hits_on_nonzero_plain_levels"] = [window_hits, window_n]
    return out


def batched_predict(ctx, vp8a, torch, split):
    """vp8a_predict_inter_mb (or _split_mv) over 8 frames' worth of MBs at
    random positions of random MB-padded reference planes of the --size grid,
    vectors within +-16 px: the batched entry points at a size that fills
    the GPU."""
    from vp8a.frames import planes

    rng = np.random.default_rng(SEED)
    shapes = [(MB_ROWS * 16, MB_COLS * 16), (MB_ROWS * 8, MB_COLS * 8), (MB_ROWS * 8, MB_COLS * 8)]
    ref = [torch.from_numpy(rng.integers(0, 256, s, dtype=np.uint8)).cuda() for s in shapes]
    n = 8 * N_MB
    xy = np.stack([rng.integers(0, MB_COLS, n), rng.integers(0, MB_ROWS, n)], 1).astype(np.uint32)
    mv = rng.integers(-64, 65, (n * (16 if split else 1), 2)).astype(np.int16)
    dxy, dmv = torch.from_numpy(xy.view(np.int32)).cuda(), torch.from_numpy(mv).cuda()
    out = torch.empty(n * 384, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    p = planes(*ref)
    call = ctx._lib.vp8a_predict_split_mv if split else ctx._lib.vp8a_predict_inter_mb

    def fn():
        st = call(ctx.handle, C.byref(p), dxy.data_ptr(), dmv.data_ptr(), n, 0, 0, out.data_ptr())
        assert st == 0, vp8a.load().vp8a_last_error()

    fn.keep = (ref, dxy, dmv, out, p)
    return fn


def lp_conv_arm(args):
    """One 32 -> 32 layer of the proposal net over `--images` 32 x 32 maps
    (8160 = one reference of a 1080p frame) through vp8a_lp_conv_forward:
    the tcgen05 path (BF16 out) beside the mma.sync path (FP32 out), CUDA
    events on the context stream, inputs larger than L2."""
    import torch

    import vp8a

    ctx = vp8a.Context(0)
    lib = ctx._lib
    n = args.images
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.relu(torch.randn(n, 32, 32, 32, device="cuda", generator=g)).to(torch.bfloat16)
    w = (torch.randn(32 * 9 * 32, device="cuda", generator=g) * 0.2).to(torch.bfloat16)
    b = torch.randn(32, device="cuda", generator=g) * 0.1
    y = torch.empty(n, 32, 32, 32, dtype=torch.bfloat16, device="cuda")
    yf = torch.empty(n, 32, 32, 32, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream)
    out = {}
    for name, yb, yff in (("tcgen05_bf16_out", y.data_ptr(), None), ("mma_sync_f32_out", None, yf.data_ptr())):
        call = lambda: lib.vp8a_lp_conv_forward(ctx.handle, x.data_ptr(), 32, w.data_ptr(), b.data_ptr(), 32, n,  # noqa: E731
                                                1, yb, yff)
        for _ in range(args.warmup):
            assert call() == 0
        assert lib.vp8a_ctx_synchronize(ctx.handle) == 0
        ts = []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            assert call() == 0
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        assert lib.vp8a_ctx_synchronize(ctx.handle) == 0
        ms = sorted(ts)[len(ts) // 2]
        flops = 2.0 * n * 1024 * 32 * 288
        out[name] = {"ms": round(ms, 4), "tflops": round(flops / ms / 1e9, 1),
                     "gbs_in_out": round(n * 1024 * 32 * (2 + (2 if yb else 4)) / ms / 1e6, 1)}
    out["max_abs_diff"] = float((y.float() - yf).abs().max())
    del x, y, yf, w, b, stream
    ctx.close()
    return {"case": "lp_conv", "images": n, "layer": "3x3 conv 32 -> 32 on 32 x 32 maps", **out}


def lp_net_arm(args):
    """The whole proposal net (vp8a_lp_net_propose: four layers and the top
    4 cells in one launch) over `--images` 32 x 32 maps, beside the same net
    layer by layer (four vp8a_lp_conv_forward launches and a torch top-k),
    CUDA events on the context stream. 24480 maps = the three references
    of a 1080p frame."""
    import torch

    import vp8a
    from vp8a import learned

    ctx = vp8a.Context(0)
    n = args.images
    net = learned.ProposalNet(ctx, seed=1)
    g = torch.Generator(device="cuda").manual_seed(5)
    with learned.on_ctx_stream(ctx):
        x = (torch.relu(torch.randn(n, 32, 32, 2, device="cuda", generator=g)) * 40).to(torch.bfloat16)
    ctx.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream)

    def fused():
        return net.propose(x, 4)

    def layered():
        with learned.on_ctx_stream(ctx):
            return torch.topk(net.forward(x), 4, dim=1).indices

    out = {}
    for name, fn in (("fused", fused), ("layered", layered)):
        for _ in range(args.warmup):
            fn()
        ctx.synchronize()
        ts = []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = sorted(ts)[len(ts) // 2]
        # Algorithmic FLOPs of the four 3 x 3 layers over the 32 x 32 map.
        flops = 2.0 * n * 1024 * 9 * (2 * 32 + 32 * 32 + 32 * 32 + 32 * 1)
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        out[name] = {"ms": round(ms, 4), "tflops": round(flops / ms / 1e9, 1),
                     "us_per_map_per_sm": round(ms * 1e3 * sms / n, 3)}
    with learned.on_ctx_stream(ctx):
        same = float((fused() == layered().to(torch.int32)).all(1).float().mean())
    out["top4_rows_equal_to_layered"] = round(same, 4)
    del x, stream, net
    ctx.close()
    return {"case": "lp_net", "images": n, **out}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vp8a", choices=["vp8a", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the step's parity check against the oracle")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--case", choices=["arnr", "analysis", "lf", "recon", "predict", "predict_mb", "predict_split",
                                       "batch", "learned", "lp_conv", "lp_net", "rd", "stream", "trellis", "me", "lp_windows",
                                       "lp_bwd"],
                    help="profile one stage alone, or (batch) the batched many-stream path")
    ap.add_argument("--streams", type=int, default=48, help="streams of the batch case")
    ap.add_argument("--train-steps", type=int, default=300, help="training steps of the learned case")
    ap.add_argument("--stream-learned", action="store_true",
                    help="stream case: also run the learned proposal through the stream path against the plain path")
    ap.add_argument("--size", default="1920x1080", help="frame size for --case")
    ap.add_argument("--images", type=int, default=8160, help="32 x 32 maps of the lp_conv and lp_net cases")
    ap.add_argument("--subpel-planes", type=int, default=0, help="analysis sub-pel planes on/off (single-stage cases)")
    ap.add_argument("--lf-layout", default="", help="passes,threads,prefetch: force the sweep's launch shape (cases)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl != "reference":
        log("note: fewer than 3 warm-up steps")
    if args.case == "batch":
        res = batch_arm(args)
    elif args.case == "learned":
        res = learned_arm(args)
    elif args.case == "lp_conv":
        res = lp_conv_arm(args)
    elif args.case == "lp_net":
        res = lp_net_arm(args)
    elif args.case == "rd":
        res = rd_arm(args)
    elif args.case == "stream":
        res = stream_arm(args)
    elif args.case:
        res = case_arm(args)
    else:
        res = reference_arm(args) if args.impl == "reference" else gpu_arm(args)
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
