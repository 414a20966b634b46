"""Parity of the batched altref stream path (vp8a.stream.AltrefStreams, the
device side of Vp8AltrefStreamEncoder::flush_group, src/stream.rs:2806-2957)
against the same group walk run with the oracle on the CPU: for every
stream and every packet (the invisible ARNR anchor and each P frame) the
chosen (level, sharpness) and the frame's bytes, and after every group the
LAST / GOLDEN / ALTREF reference planes, must be identical."""
import numpy as np
import pytest

import vp8a
from vp8a import abi, synth
from vp8a.stream import AltrefStreams

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

QI, STRENGTH = 44, 3
TRELLIS = 1.0


class OracleStream:
    """The group walk of AltrefStreams restated with the oracle."""

    def __init__(self, oracle):
        self.o = oracle
        self.refs = None

    def code(self, frame, **hdr):
        o = self.o
        lam = o.rd_lambda(QI)
        dec = o.analyse_inter_frame(frame, self.refs, [1, 2, 3], lam, threads=8)
        recon = tuple(np.zeros_like(p) for p in self.refs[0])
        lf = np.zeros(dec.size, abi.MB_LF_INFO_DTYPE)
        cf, fl, _ = o.reconstruct_inter_frame(frame, self.refs, [1, 2, 3], dec, abi.quant_indices(QI), recon,
                                              lf_info=lf, threads=8, trellis_strength=TRELLIS)
        level, sharp = o.select_filter_params(recon, lf, abi.filter_config(0, 0), frame, threads=8)
        out = o.filter_frame(recon, lf, abi.filter_config(level, sharp)) if level else recon
        h, w = frame[0].shape
        hdr_ = abi.frame_header(w, h, abi.quant_indices(QI), loop_filter_level=level, sharpness_level=sharp,
                                pick_intra=False, **hdr)
        return out, level, sharp, vp8a.write_inter_frame(hdr_, dec.reshape(-1), cf)

    def group(self, frames):
        packets = []
        first_p = 0
        if self.refs is None:
            p = vp8a.pad_to_mb(*frames[0])
            self.refs = [p, tuple(x.copy() for x in p), tuple(x.copy() for x in p)]
            first_p = 1
            packets.append(("key", 0, 0, None))
        n = len(frames)
        if n - first_p > 0 and n >= 2:
            anchor = self.o.build_arnr_altref(frames, n - 1, STRENGTH, threads=8)
            out, lv, sh, b = self.code(anchor, refresh_last=0, refresh_alternate_frame=1)
            self.refs[2] = out
            packets.append(("altref", lv, sh, b))
        for j in range(first_p, n):
            out, lv, sh, b = self.code(frames[j])
            self.refs[0] = out
            packets.append(("inter", lv, sh, b))
        return packets


def test_altref_streams_match_the_oracle_walk(oracle):
    ctx = vp8a.Context(0)  # its own context: the pipeline sets the trellis strength on it
    sizes = [(96, 64), (64, 48), (80, 40)]
    group, n_groups = 4, 2
    seqs = [synth.make_sequence(w, h, group * n_groups, seed=70 + i, pieces=3, occluders=2)[0]
            for i, (w, h) in enumerate(sizes)]
    dev = lambda f: tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f)  # noqa: E731
    streams = AltrefStreams(ctx, sizes, qi=QI, strength=STRENGTH, trellis_strength=TRELLIS)
    oracles = [OracleStream(oracle) for _ in sizes]
    kinds_seen, levels_seen = set(), set()
    for gi in range(n_groups):
        frames = [s[gi * group:(gi + 1) * group] for s in seqs]
        torch.cuda.synchronize()
        got = streams.encode_group([[dev(f) for f in fr] for fr in frames])
        for k, (fr, orc) in enumerate(zip(frames, oracles)):
            want = orc.group(fr)
            assert len(got[k]) == len(want)
            for g, (kind, lv, sh, b) in zip(got[k], want):
                assert (g["kind"], g["level"], g["sharpness"]) == (kind, lv, sh), (gi, k, g["kind"])
                assert g["bytes"] == b, (gi, k, g["kind"])
                kinds_seen.add(kind)
                levels_seen.add(lv)
            ctx.synchronize()
            for dref, oref in zip(streams.references(k), orc.refs):
                assert all(np.array_equal(d.cpu().numpy(), o) for d, o in zip(dref, oref)), (gi, k)
    ctx.close()
    assert kinds_seen == {"key", "altref", "inter"}
    assert len(levels_seen) > 1
