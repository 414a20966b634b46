"""Learned motion proposal (no counterpart in the reference).

A 4-layer 3x3 conv net (2 -> 32 -> 32 -> 32 -> 1 channels, ReLU between,
BF16 weights and activations, FP32 accumulation) scores a 32 x 32 grid of
whole-pel vectors, 2 px apart, from an MB's coarse cost volume against a
reference (`vp8a_lp_windows`: at each grid vector the half-resolution SAD of
the MB and the reference's texture), so each score sees the matching cost
of its own vector and its neighbours'. Training
runs every layer on the library's hand-written tensor-core kernels
(`vp8a_lp_conv_forward` / `vp8a_lp_conv_backward`), the loss and the
optimiser on its own kernels (`vp8a_lp_softmax_ce`, `vp8a_lp_adam`);
inference runs the whole net and the top-k in one launch
(`vp8a_lp_net_propose`); torch only holds the device buffers. Training
labels are the plain search's own whole-pel results (`labels_from_search`).

The net only proposes: `learned_search` takes its best cells as seeds of an
exact local search (`vp8a_lp_seeded_search`: every whole-pel position within
+-2 px of each seed, the first smallest SAD, then the reference's half- and
quarter-pel refinement),
with the plain descent from the zero vector as the fallback for MBs whose
refined SAD exceeds 1.25 x the frame's median. Every returned vector and SAD
is exact; the net decides only where to look.
"""
import ctypes as C

import numpy as np

from . import abi
from .frames import luma_ref, ptr
from .lib import check

GRID = 32            # cells per side; cell (i, j) = (2 (i - 16), 2 (j - 16)) px

_streams = {}


def on_ctx_stream(ctx):
    """A torch stream context on the library context's CUDA stream: torch
    work inside it is ordered with the library's calls (every function here
    runs its torch ops under it; callers building inputs with torch should
    too)."""
    import torch

    key = ctx.stream
    if key not in _streams:
        _streams[key] = torch.cuda.ExternalStream(ctx.stream)
    return torch.cuda.stream(_streams[key])
PIX = GRID * GRID
LAYERS = [(2, 32, True), (32, 32, True), (32, 32, True), (32, 1, False)]


def cell_of_mv(mv_row, mv_col):
    """Label cell of a quarter-pel vector (nearest 2-px cell), or -1 when it
    falls outside the grid."""
    r = np.rint(np.asarray(mv_row, np.float64) / 8.0).astype(np.int64) + 16
    c = np.rint(np.asarray(mv_col, np.float64) / 8.0).astype(np.int64) + 16
    ok = (r >= 0) & (r < GRID) & (c >= 0) & (c < GRID)
    return np.where(ok, r * GRID + c, -1).astype(np.int32)


def mv_of_cell(cell):
    """Quarter-pel (row, col) of a cell's vector."""
    cell = np.asarray(cell, np.int64)
    return (cell // GRID - 16) * 8, (cell % GRID - 16) * 8


def _ordered(fn):
    """Run a ProposalNet method with torch on the library's stream."""

    def wrapped(self, *a, **k):
        with on_ctx_stream(self.ctx):
            return fn(self, *a, **k)

    wrapped.__doc__ = fn.__doc__
    wrapped.__name__ = fn.__name__
    return wrapped


class ProposalNet:
    """The net's parameters (FP32 master copies, BF16 working copies, Adam
    moments) and activations, on the context's GPU."""

    def __init__(self, ctx, seed=0):
        import torch

        self.torch, self.ctx, self.dev = torch, ctx, torch.device("cuda")
        g = torch.Generator().manual_seed(seed)
        self.layers = []
        for cin, cout, relu in LAYERS:
            std = (2.0 / (9 * cin)) ** 0.5 * (0.5 if not relu else 1.0)
            w = (torch.randn(cout * 9 * cin, generator=g) * std).to(self.dev)
            b = torch.zeros(cout, device=self.dev)
            self.layers.append({
                "cin": cin, "cout": cout, "relu": relu, "w": w, "b": b,
                "wh": w.to(torch.bfloat16),
                "mw": torch.zeros_like(w), "vw": torch.zeros_like(w),
                "mb": torch.zeros_like(b), "vb": torch.zeros_like(b),
                "gw": torch.zeros_like(w), "gb": torch.zeros_like(b),
                "bh": b.to(torch.bfloat16),  # the bias stays FP32 in the forward pass
            })
        self.step_count = 0
        self._acts = None

    def _lib(self):
        return self.ctx._lib

    @_ordered
    def forward(self, x, keep=False):
        """x: [n, 32, 32, 2] bf16 device tensor. Returns FP32 scores [n, 1024]
        (and keeps the activations for `backward` when `keep`)."""
        torch = self.torch
        n = x.shape[0]
        acts = [x]
        h = x
        for li, L in enumerate(self.layers):
            last = li == len(self.layers) - 1
            if last:
                out = torch.empty((n, PIX), dtype=torch.float32, device=self.dev)
                y, yf = None, out
            else:
                out = torch.empty((n, GRID, GRID, L["cout"]), dtype=torch.bfloat16, device=self.dev)
                y, yf = out, None
            check(self._lib().vp8a_lp_conv_forward(self.ctx.handle, ptr(h), L["cin"], ptr(L["wh"]), ptr(L["b"]),
                                                   L["cout"], n, int(L["relu"]), ptr(y), ptr(yf)),
                  "vp8a_lp_conv_forward")
            h = out
            acts.append(out)
        if keep:
            self._acts = acts
        return h

    @_ordered
    def loss_and_grad(self, logits, labels):
        """Softmax cross-entropy of `labels` (int32 device tensor, -1 = none);
        returns (mean loss, BF16 d(logits))."""
        torch = self.torch
        n = logits.shape[0]
        d = torch.empty((n, PIX), dtype=torch.bfloat16, device=self.dev)
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        check(self._lib().vp8a_lp_softmax_ce(self.ctx.handle, ptr(logits), ptr(labels), n, ptr(d), ptr(loss), None),
              "vp8a_lp_softmax_ce")
        valid = max(int((labels >= 0).sum().item()), 1)
        return loss, d, valid

    @_ordered
    def backward(self, dlogits):
        """Accumulates every layer's gradients from d(scores)."""
        torch = self.torch
        acts = self._acts
        n = acts[0].shape[0]
        dy = dlogits.view(n, GRID, GRID, 1)
        for li in range(len(self.layers) - 1, -1, -1):
            L = self.layers[li]
            x = acts[li]
            dx = None if li == 0 else torch.empty_like(x)
            check(self._lib().vp8a_lp_conv_backward(self.ctx.handle, ptr(x), L["cin"], ptr(L["wh"]), L["cout"], n,
                                                    ptr(dy), int(li > 0), ptr(dx), ptr(L["gw"]), ptr(L["gb"])),
                  "vp8a_lp_conv_backward")
            dy = dx

    @_ordered
    def zero_grad(self):
        for L in self.layers:
            L["gw"].zero_()
            L["gb"].zero_()

    @_ordered
    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        for L in self.layers:
            for w, g, m, v, wh in ((L["w"], L["gw"], L["mw"], L["vw"], L["wh"]),
                                   (L["b"], L["gb"], L["mb"], L["vb"], L["bh"])):
                check(self._lib().vp8a_lp_adam(self.ctx.handle, ptr(w), ptr(g), ptr(m), ptr(v), w.numel(), lr, beta1,
                                               beta2, eps, self.step_count, ptr(wh)), "vp8a_lp_adam")

    @_ordered
    def train_step(self, x, labels, lr=1e-3):
        """One forward / backward / Adam step on a batch; returns the mean
        cross-entropy over the batch's labelled items (of the forward pass
        before the update) as a Python float. The loss is read back on the
        library's stream, after the kernel that wrote it."""
        self.zero_grad()
        logits = self.forward(x, keep=True)
        loss, d, valid = self.loss_and_grad(logits, labels)
        # d(logits) is normalised by the batch size, the loss by the labelled
        # items.
        self.backward(d)
        self.adam(lr)
        return float((loss / valid).item())

    @_ordered
    def propose(self, x, k=4, logits=None):
        """Top-k cells per item, best first ([n, k] int32 device tensor; the
        first cell among equal scores): the whole net in one fused launch
        (vp8a_lp_net_propose), activations on chip. `logits` (optional
        [n, 1024] FP32 device tensor) receives the scores."""
        torch = self.torch
        n = x.shape[0]
        cells = torch.empty((n, k), dtype=torch.int32, device=self.dev)
        L = self.layers
        check(self._lib().vp8a_lp_net_propose(self.ctx.handle, ptr(x), n, ptr(L[0]["wh"]), ptr(L[0]["b"]),
                                              ptr(L[1]["wh"]), ptr(L[1]["b"]), ptr(L[2]["wh"]), ptr(L[2]["b"]),
                                              ptr(L[3]["wh"]), ptr(L[3]["b"]), k, ptr(cells),
                                              ptr(logits) if logits is not None else None),
              "vp8a_lp_net_propose")
        return cells


def windows(ctx, src_y, ref_y, mb_xy):
    """The net's input for the MBs `mb_xy` ([n, 2] uint32 device tensor of
    (col, row)) of a source / reference luma pair (device uint8 planes of one
    size). Returns [n, 32, 32, 2] bf16."""
    import torch

    n = mb_xy.shape[0]
    for t, what in ((src_y, "source"), (ref_y, "reference"), (mb_xy, "mb_xy")):
        assert t.is_cuda, f"{what} must be a CUDA tensor"
    assert mb_xy.dim() == 2 and mb_xy.shape[1] == 2 and mb_xy.dtype == torch.int32 and mb_xy.is_contiguous()
    with on_ctx_stream(ctx):
        out = torch.empty((n, GRID, GRID, 2), dtype=torch.bfloat16, device=mb_xy.device)
        s, r = luma_ref(src_y), luma_ref(ref_y)
        check(ctx._lib.vp8a_lp_windows(ctx.handle, C.byref(s), C.byref(r), ptr(mb_xy), n, ptr(out)),
              "vp8a_lp_windows")
    return out


def all_mbs(mb_cols, mb_rows, device="cuda"):
    import torch

    r, c = np.meshgrid(np.arange(mb_rows), np.arange(mb_cols), indexing="ij")
    xy = np.stack([c.reshape(-1), r.reshape(-1)], 1).astype(np.uint32)
    return torch.from_numpy(xy.view(np.int32)).to(device)


def labels_from_search(ctx, frame, ref_padded, lam):
    """Labels of one frame: the plain search's quarter-pel result against
    `ref_padded` (the exhaustive analysis' per-reference trace, reference
    LAST), as cells (-1 where the vector leaves the grid)."""
    from .api import analyse_inter_frame

    _, tr = analyse_inter_frame(ctx, frame, [ref_padded], [abi.REF_LAST], lam, trace=True)
    q = tr[..., 0]["quarter"]["mv"].reshape(-1)
    return cell_of_mv(q["row"], q["col"]), tr[..., 0]["quarter"]["sad"].reshape(-1)


def learned_search(ctx, net, src_y, ref_y, mb_xy, k=4, radius=2, fallback=1.25, seeds=None, timings=None):
    """The learned path for one (source, reference) luma pair: proposal,
    exact +-`radius` px whole-pel search around each of the k seeds, half-
    and quarter-pel refinement of the best, and the plain descent from the
    zero vector for MBs whose SAD exceeds `fallback` x the median. `seeds`
    ([n, k] cells) replaces the net (the ablation). `timings` (a dict),
    when given, accumulates each stage's device milliseconds (CUDA events
    on the library stream): cost volumes, net, seeded whole-pel search,
    sub-pel refinement, fallback. Returns (mv [n, 2] quarter-pel int16, sad
    [n] uint32, fell_back [n] bool) as numpy."""
    import torch

    with on_ctx_stream(ctx):
        return _learned_search(ctx, net, src_y, ref_y, mb_xy, k, radius, fallback, seeds, timings)


def _learned_search(ctx, net, src_y, ref_y, mb_xy, k, radius, fallback, seeds, timings=None):
    import torch

    marks = []

    def mark(name):
        if timings is not None:
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            marks.append((name, e))

    n = mb_xy.shape[0]
    h, w = src_y.shape[0], src_y.shape[1]
    mark("start")
    if seeds is None:
        x = windows(ctx, src_y, ref_y[:h, :w], mb_xy)
        mark("cost_volumes")
        seeds = net.propose(x, k)
        mark("net")
    mbr, mbc = (h + 15) // 16, (w + 15) // 16
    # Source MBs (16x16 luma, edge-replicated) for every item.
    src_mbs = _source_mbs(src_y, mb_xy, h, w)
    ref = luma_ref(ref_y, width=mbc * 16, height=mbr * 16)
    lib = ctx._lib
    # Every whole-pel vector within +-radius px of each seed, first smallest
    # SAD in seed, row, column order (one fused kernel).
    seeds32 = seeds.to(torch.int32).contiguous()
    found = torch.empty((n, 2), dtype=torch.int32, device=seeds.device)  # search_result: mv (2 x i16) + sad
    check(lib.vp8a_lp_seeded_search(ctx.handle, C.byref(ref), ptr(src_mbs), ptr(mb_xy), ptr(seeds32), k, radius, n,
                                    ptr(found)), "vp8a_lp_seeded_search")
    mark("seeded_search")
    whole = found[:, 0].contiguous().view(torch.int16).view(n, 2)
    sr_out = torch.empty((n, 2), dtype=torch.int32, device=seeds.device)  # search_result: mv (2 x i16) + sad
    half = torch.empty((n, 2), dtype=torch.int32, device=seeds.device)
    check(lib.vp8a_half_pixel_refine_luma(ctx.handle, C.byref(ref), ptr(src_mbs), ptr(mb_xy), ptr(whole), n,
                                          ptr(half)), "vp8a_half_pixel_refine_luma")
    hmv = half[:, 0].contiguous().view(torch.int16).view(n, 2)
    check(lib.vp8a_quarter_pixel_refine_luma(ctx.handle, C.byref(ref), ptr(src_mbs), ptr(mb_xy), ptr(hmv.contiguous()),
                                             n, ptr(sr_out)), "vp8a_quarter_pixel_refine_luma")
    out_mv = sr_out[:, 0].contiguous().view(torch.int16).view(n, 2).clone()
    out_sad = sr_out[:, 1].clone()
    mark("subpel")
    # Fallback: the plain descent from the zero vector (8 rounds + sub-pel)
    # for the MBs whose SAD exceeds `fallback` x the median, kept where it
    # wins. The flags stay on the device: the masked descent skips the other
    # items, so no count or index list crosses to the host.
    med = out_sad.to(torch.float32).median()
    fb = out_sad.to(torch.float32) > fallback * med
    zero = torch.zeros((n, 2), dtype=torch.int16, device=seeds.device)
    w_o = torch.empty((n, 2), dtype=torch.int32, device=seeds.device)
    h_o = torch.empty_like(w_o)
    q_o = torch.zeros_like(w_o)
    fb8 = fb.to(torch.uint8)
    check(lib.vp8a_motion_descent_masked(ctx.handle, C.byref(ref), ptr(src_mbs), ptr(mb_xy), ptr(zero), 8, n,
                                         ptr(fb8), ptr(w_o), ptr(h_o), ptr(q_o)),
          "vp8a_motion_descent_masked")
    better = fb & (q_o[:, 1] < out_sad)
    out_sad = torch.where(better, q_o[:, 1], out_sad)
    out_mv = torch.where(better[:, None], q_o[:, 0].contiguous().view(torch.int16).view(n, 2), out_mv)
    mark("fallback")
    ctx.synchronize()
    for (_, a), (name, b) in zip(marks, marks[1:]):
        timings[name] = timings.get(name, 0.0) + a.elapsed_time(b)
    return out_mv.cpu().numpy(), out_sad.cpu().numpy().astype(np.uint32), fb.cpu().numpy()


def _source_mbs(src_y, mb_xy, h, w):
    """[n, 256] uint8: the 16x16 luma of each listed MB, edge-replicated
    (I420Frame::extract_mb)."""
    import torch

    xy = mb_xy.view(torch.int32).to(torch.int64)
    oy = torch.arange(16, device=src_y.device)
    ys = (xy[:, 1:2] * 16 + oy[None, :]).clamp(max=h - 1)
    xs = (xy[:, 0:1] * 16 + oy[None, :]).clamp(max=w - 1)
    return src_y[ys[:, :, None], xs[:, None, :]].reshape(-1, 256).contiguous()


LF_LEVELS = 64
LF_WINDOW = 9


class LfWindowHead:
    """The proposal's loop-filter level window: a linear head over the
    net's layer-3 features averaged over a sample of the frame's MBs, plus
    the frame's quantiser index (qi / 127), scoring the 64 levels; the
    window is the 9 levels around the best score. Trained with the frame's
    level chosen by the plain search (vp8a_lp_lf_head, Adam)."""

    C = 33  # 32 pooled channels + qi

    def __init__(self, ctx, seed=0):
        import torch

        self.torch, self.ctx = torch, ctx
        g = torch.Generator().manual_seed(seed)
        self.w = (torch.randn(LF_LEVELS * self.C, generator=g) * 0.05).cuda()
        self.b = torch.zeros(LF_LEVELS, device="cuda")
        self.state = {k: torch.zeros_like(v) for k, v in (("mw", self.w), ("vw", self.w), ("mb", self.b),
                                                          ("vb", self.b), ("gw", self.w), ("gb", self.b))}
        self.wh = self.w.to(torch.bfloat16)
        self.bh = self.b.to(torch.bfloat16)
        self.steps = 0

    def features(self, net, src_y, ref_y, mb_xy, qi):
        """(sums [33] FP32 device tensor, count) of one frame: the layer-3
        channel sums over the sampled MBs' 32x32 maps, and qi / 127 x count."""
        torch = self.torch
        with on_ctx_stream(self.ctx):
            h, w = src_y.shape[0], src_y.shape[1]
            x = windows(self.ctx, src_y, ref_y[:h, :w], mb_xy)
            net.forward(x, keep=True)
            a3 = net._acts[3]
            sums = torch.zeros(self.C, dtype=torch.float32, device="cuda")
            check(self.ctx._lib.vp8a_lp_pool(self.ctx.handle, ptr(a3), 32, a3.shape[0], ptr(sums)), "vp8a_lp_pool")
            count = float(a3.shape[0] * PIX)
            sums[32] = qi / 127.0 * count
        return sums, count

    def train_step(self, frames, lr=1e-2):
        """frames: list of (sums, count, level). Returns the summed loss."""
        torch = self.torch
        with on_ctx_stream(self.ctx):
            self.state["gw"].zero_()
            self.state["gb"].zero_()
            loss = torch.zeros(1, device="cuda")
            for sums, count, level in frames:
                check(self.ctx._lib.vp8a_lp_lf_head(self.ctx.handle, ptr(sums), count, self.C, ptr(self.w),
                                                    ptr(self.b), LF_LEVELS, int(level), None, ptr(self.state["gw"]),
                                                    ptr(self.state["gb"]), ptr(loss)), "vp8a_lp_lf_head")
            self.steps += 1
            for w, g, m, v, wh in ((self.w, self.state["gw"], self.state["mw"], self.state["vw"], self.wh),
                                   (self.b, self.state["gb"], self.state["mb"], self.state["vb"], self.bh)):
                check(self.ctx._lib.vp8a_lp_adam(self.ctx.handle, ptr(w), ptr(g), ptr(m), ptr(v), w.numel(), lr, 0.9,
                                                 0.999, 1e-8, self.steps, ptr(wh)), "vp8a_lp_adam")
            return float(loss.item())

    def window(self, sums, count):
        """(lo, hi): the 9 levels around the best-scored level, inside 0..63."""
        torch = self.torch
        with on_ctx_stream(self.ctx):
            z = torch.empty(LF_LEVELS, device="cuda")
            check(self.ctx._lib.vp8a_lp_lf_head(self.ctx.handle, ptr(sums), count, self.C, ptr(self.w), ptr(self.b),
                                                LF_LEVELS, -1, ptr(z), None, None, None), "vp8a_lp_lf_head")
            c = int(torch.argmax(z).item())
        lo = max(0, min(c - LF_WINDOW // 2, LF_LEVELS - LF_WINDOW))
        return lo, lo + LF_WINDOW - 1


def sample_mbs(mb_cols, mb_rows, n=256, seed=0, device="cuda"):
    """n MB positions spread over the frame (seeded)."""
    import torch

    rng = np.random.default_rng(seed)
    total = mb_cols * mb_rows
    idx = np.sort(rng.choice(total, size=min(n, total), replace=False))
    xy = np.stack([idx % mb_cols, idx // mb_cols], 1).astype(np.uint32)
    return torch.from_numpy(xy.view(np.int32)).to(device)
