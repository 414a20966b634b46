"""The lagged altref stream path of many streams at once on one GPU.

`AltrefStreams` mirrors the encoder-analysis side of
`Vp8AltrefStreamEncoder::flush_group` (src/stream.rs:2806-2957) for a set of
independent streams of any sizes, one lookahead group at a time:

1. the group's invisible anchor: `build_arnr_altref` over the group with
   the last frame as the centre (src/stream.rs:2890-2895), coded as an inter
   frame against LAST / GOLDEN / ALTREF and, once reconstructed and loop
   filtered, the new ALTREF (`encode_invisible_altref_update_full`);
2. every visible P frame of the group in order: the exhaustive inter
   analysis against LAST / GOLDEN / ALTREF, the §14 reconstruction of the
   chosen modes, the §9.4 automatic (level, sharpness) search
   (select_filter_params, the reference's full walk), the §15 filter pass,
   and the filtered picture as the next LAST (the `refresh_last` ladder).

Each stage of all streams is one batched device call
(vp8a_build_arnr_altrefs_planes, vp8a_analyse_inter_frames,
vp8a_reconstruct_inter_frames, vp8a_select_filter_params_batch); the
filter pass runs per stream. Reference planes stay on the device between
frames and groups. The frame bitstreams (`write`) come from the host
writer, vp8a_write_inter_frame, with the decisions and coefficients read
back.

What the device path does not do, as in the rest of this library: the key
frame that opens a stream is intra coding, so the first group's first
frame stands in as its own reconstruction (LAST = GOLDEN = ALTREF = that
frame, MB-padded) and is not coded; intra picking is off. The §13 trellis
runs at `trellis_strength` (the reference's KeyframeParams default, 1.0,
unless given; it is set on the context). Rate control, scene cuts and
golden promotion are control plane and keep their defaults (fixed
quantiser, no promotion).
"""
import ctypes as C

import numpy as np

from . import abi
from .frames import i420, planes, source
from .lib import check, load

REF_IDS = (abi.REF_LAST, abi.REF_GOLDEN, abi.REF_ALTREF)


def _mb_padded(torch, h, w, dev):
    mbr, mbc = (h + 15) // 16, (w + 15) // 16
    return [torch.zeros((mbr * 16, mbc * 16), dtype=torch.uint8, device=dev),
            torch.zeros((mbr * 8, mbc * 8), dtype=torch.uint8, device=dev),
            torch.zeros((mbr * 8, mbc * 8), dtype=torch.uint8, device=dev)]


def pad_into(torch, dst, frame):
    """Edge-replicate a visible (y, u, v) device picture into MB-padded
    device planes `dst` (the layout of a reference)."""
    for d, p in zip(dst, frame):
        h, w = p.shape
        d[:h, :w] = p
        if d.shape[1] > w:
            d[:h, w:] = p[:, w - 1:w]
        if d.shape[0] > h:
            d[h:, :] = d[h - 1:h, :]


class _Stream:
    def __init__(self, torch, w, h, dev):
        self.w, self.h = w, h
        self.mb_cols, self.mb_rows = (w + 15) // 16, (h + 15) // 16
        self.n_mb = self.mb_cols * self.mb_rows
        self.last = _mb_padded(torch, h, w, dev)
        self.golden = _mb_padded(torch, h, w, dev)
        self.altref = _mb_padded(torch, h, w, dev)
        self.recon = _mb_padded(torch, h, w, dev)
        self.anchor = _mb_padded(torch, h, w, dev)
        self.dec = torch.zeros(self.n_mb * abi.MB_DECISION_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.lf = torch.zeros(self.n_mb * abi.MB_LF_INFO_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.coeffs = torch.zeros(self.n_mb * 400, dtype=torch.int16, device=dev)
        self.flags = torch.zeros(self.n_mb, dtype=torch.uint8, device=dev)
        self.started = False


class AltrefStreams:
    """Streams of sizes `sizes` [(width, height), ...] coded in lockstep, one
    lookahead group per `encode_group` call. `qi` is the fixed quantiser
    index, `strength` the ARNR strength. With `write` the frames'
    bitstreams are produced (host writer) and returned."""

    def __init__(self, ctx, sizes, qi=44, strength=3, write=True, n_partitions=1, trellis_strength=1.0):
        import torch

        from .api import rd_lambda

        self.torch, self.ctx, self.lib = torch, ctx, load()
        self.dev = torch.device("cuda", ctx.device)
        self.stream = torch.cuda.ExternalStream(ctx.stream, device=self.dev)
        self.qi, self.strength, self.write, self.n_partitions = qi, strength, write, n_partitions
        self.quant = abi.quant_indices(qi)
        self.lam = rd_lambda(qi)
        self.ctxs = abi.default_mv_contexts()
        self.ids = np.array(REF_IDS, np.uint8)
        ctx.set_trellis_strength(trellis_strength)
        with torch.cuda.stream(self.stream):
            self.s = [_Stream(torch, w, h, self.dev) for w, h in sizes]
        self.keep = []

    # ------------------------------------------------------------ stages
    def _frames_i420(self, frames):
        return [i420(*f) for f in frames]

    def _analyse(self, srcs, props=None):
        """Exhaustive analysis of srcs[k] (visible (y, u, v) device planes)
        for stream k against its LAST / GOLDEN / ALTREF; `props` (optional)
        gives per stream its proposal vectors (3 MV_DTYPE vectors per MB, a
        device tensor or a contiguous numpy array, or None), the second
        NEWMV candidate of vp8a_analyse_inter_frames_proposals."""
        jobs, keep = [], []
        for st, src in zip(self.s, srcs):
            refs = (abi.Planes * 3)(planes(*st.last), planes(*st.golden), planes(*st.altref))
            keep.append(refs)
            jobs.append(abi.AnalysisJob(i420(*src), C.cast(refs, C.c_void_p), self.ids.ctypes.data, 3,
                                        C.cast(C.pointer(self.ctxs), C.c_void_p), self.lam, st.dec.data_ptr(), None))
        arr = (abi.AnalysisJob * len(jobs))(*jobs)
        if props is not None and any(p is not None for p in props):
            ptrs = [None if p is None else (p.data_ptr() if hasattr(p, "data_ptr") else p.ctypes.data) for p in props]
            parr = (C.c_void_p * len(props))(*ptrs)
            keep += [parr, props]
            check(self.lib.vp8a_analyse_inter_frames_proposals(self.ctx.handle, C.cast(arr, C.c_void_p), len(jobs),
                                                               C.cast(parr, C.c_void_p)),
                  "vp8a_analyse_inter_frames_proposals")
        else:
            check(self.lib.vp8a_analyse_inter_frames(self.ctx.handle, C.cast(arr, C.c_void_p), len(jobs)),
                  "vp8a_analyse_inter_frames")
        return keep

    def _reconstruct(self, srcs):
        jobs, keep = [], []
        for st, src in zip(self.s, srcs):
            refs = (abi.Planes * 3)(planes(*st.last), planes(*st.golden), planes(*st.altref))
            keep.append(refs)
            jobs.append(abi.ReconJob(i420(*src), C.cast(refs, C.c_void_p), self.ids.ctypes.data, 3, 0,
                                     st.dec.data_ptr(), self.quant, None, None, 0, abi.FILTER_SIXTAP,
                                     planes(*st.recon), st.coeffs.data_ptr(), st.flags.data_ptr(),
                                     st.lf.data_ptr()))
        arr = (abi.ReconJob * len(jobs))(*jobs)
        check(self.lib.vp8a_reconstruct_inter_frames(self.ctx.handle, C.cast(arr, C.c_void_p), len(jobs)),
              "vp8a_reconstruct_inter_frames")
        return keep

    def _loop_filter(self, srcs, levels=None):
        """The automatic (level, sharpness) pick of every stream's
        reconstruction (one batched walk) and the §15 pass in place.
        `levels` (optional) replaces the pick: one (level, sharpness) per
        stream."""
        if levels is None:
            jobs = [abi.SweepJob(planes(*st.recon), st.lf.data_ptr(), abi.filter_config(0, 0), source(*src), 0,
                                 None) for st, src in zip(self.s, srcs)]
            arr = (abi.SweepJob * len(jobs))(*jobs)
            lv = np.zeros(len(jobs), np.uint8)
            sh = np.zeros(len(jobs), np.uint8)
            check(self.lib.vp8a_select_filter_params_batch(self.ctx.handle, C.cast(arr, C.c_void_p), len(jobs),
                                                           lv.ctypes.data, sh.ctypes.data),
                  "vp8a_select_filter_params_batch")
            levels = [(int(a), int(b)) for a, b in zip(lv, sh)]
        for st, (level, sharp) in zip(self.s, levels):
            if level:
                cfg = abi.filter_config(level, sharp)
                p = planes(*st.recon)
                check(self.lib.vp8a_filter_frame(self.ctx.handle, C.byref(p), st.lf.data_ptr(), C.byref(cfg)),
                      "vp8a_filter_frame")
        return levels

    def _bitstreams(self, levels, **hdr):
        """Each stream's frame bytes from its decisions and coefficients."""
        from .api import write_inter_frame

        self.ctx.synchronize()
        out = []
        for st, (level, sharp) in zip(self.s, levels):
            dec = np.frombuffer(st.dec.cpu().numpy().tobytes(), abi.MB_DECISION_DTYPE)
            cf = st.coeffs.cpu().numpy().reshape(st.n_mb, 400)
            h = abi.frame_header(st.w, st.h, self.quant, n_partitions=self.n_partitions, loop_filter_level=level,
                                 sharpness_level=sharp, pick_intra=False, **hdr)
            out.append(write_inter_frame(h, dec, cf))
        return out

    def _code_frame(self, srcs, levels=None, props=None, **hdr):
        """Analyse, reconstruct and loop-filter srcs[k] for every stream k;
        the filtered picture is left in each stream's `recon` planes."""
        keep = self._analyse(srcs, props)
        keep += self._reconstruct(srcs)
        levels = self._loop_filter(srcs, levels)
        bits = self._bitstreams(levels, **hdr) if self.write else [None] * len(self.s)
        self.keep = keep
        return levels, bits

    # ------------------------------------------------------------- group
    def encode_group(self, groups, lf_levels=None, proposer=None, psnr=False):
        """`groups[k]` = the lookahead group of stream k: a list of visible
        (y, u, v) device pictures (every stream the same length). Returns
        per stream the list of packets, each a dict with `kind` ("key", the
        uncoded stand-in, "altref" or "inter"), `level`, `sharpness` and
        `bytes` (None without `write`). `lf_levels`, when given, is a
        function (stage index, streams) -> list of (level, sharpness)
        replacing the automatic pick (the learned window's hook);
        `proposer`, when given, is a function (streams, srcs) -> per stream
        the proposal vectors of each coded frame (see _analyse), called
        before the frame's analysis with its references in place (the
        learned proposal's hook). With `psnr` each inter packet also
        carries `psnr_y`, the luma PSNR of the filtered picture against its
        source."""
        torch = self.torch
        n = len(groups[0])
        assert all(len(g) == n for g in groups), "every stream's group must have the same length"
        packets = [[] for _ in self.s]
        first_p = 0
        with torch.cuda.stream(self.stream):
            if not self.s[0].started:
                # Key frame stand-in: the first frame as its own reconstruction.
                for st, g in zip(self.s, groups):
                    pad_into(torch, st.last, g[0])
                    for d, s_ in zip(st.golden, st.last):
                        d.copy_(s_)
                    for d, s_ in zip(st.altref, st.last):
                        d.copy_(s_)
                    st.started = True
                first_p = 1
                for p in packets:
                    p.append({"kind": "key", "level": 0, "sharpness": 0, "bytes": None})
        stage = 0
        if n - first_p > 0 and n >= 2:
            # The invisible anchor: ARNR over the group, centre = its last frame.
            jobs, keep = [], []
            for st, g in zip(self.s, groups):
                arr = (abi.I420 * n)(*self._frames_i420(g))
                keep.append(arr)
                jobs.append(abi.ArnrPlanesJob(C.cast(arr, C.c_void_p), n, n - 1, self.strength, planes(*st.anchor)))
            jarr = (abi.ArnrPlanesJob * len(jobs))(*jobs)
            check(self.lib.vp8a_build_arnr_altrefs_planes(self.ctx.handle, C.cast(jarr, C.c_void_p), len(jobs)),
                  "vp8a_build_arnr_altrefs_planes")
            srcs = [(st.anchor[0][:st.h, :st.w], st.anchor[1][:(st.h + 1) // 2, :(st.w + 1) // 2],
                     st.anchor[2][:(st.h + 1) // 2, :(st.w + 1) // 2]) for st in self.s]
            levels, bits = self._code_frame(srcs, lf_levels(stage, self) if lf_levels else None,
                                            proposer(self, srcs) if proposer else None,
                                            refresh_last=0, refresh_alternate_frame=1)
            stage += 1
            for st, p, (lv, sh), b in zip(self.s, packets, levels, bits):
                st.altref, st.recon = st.recon, st.altref
                p.append({"kind": "altref", "level": lv, "sharpness": sh, "bytes": b})
        for j in range(first_p, n):
            srcs = [g[j] for g in groups]
            levels, bits = self._code_frame(srcs, lf_levels(stage, self) if lf_levels else None,
                                            proposer(self, srcs) if proposer else None)
            stage += 1
            for st, p, (lv, sh), b, src in zip(self.s, packets, levels, bits, srcs):
                st.last, st.recon = st.recon, st.last
                pk = {"kind": "inter", "level": lv, "sharpness": sh, "bytes": b}
                if psnr:
                    with torch.cuda.stream(self.stream):
                        d = st.last[0][:st.h, :st.w].float() - src[0].float()
                        mse = float((d * d).mean())
                    pk["psnr_y"] = 99.0 if mse == 0.0 else 10.0 * float(np.log10(255.0 * 255.0 / mse))
                p.append(pk)
        return packets

    def references(self, k):
        """Stream k's (LAST, GOLDEN, ALTREF) MB-padded device planes."""
        st = self.s[k]
        return st.last, st.golden, st.altref
