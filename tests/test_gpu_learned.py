"""The learned motion proposal's kernels against an FP32 numpy reference
(gradient check), its training, and the seeded exact search with the
ablation (net seeds against the same search seeded at the zero vector).

Reference semantics: the conv layers compute, in FP32 over BF16 inputs and
weights, out[y][x][co] = b[co] + sum over taps and ci of
x[y + dy][x + dx][ci] w[co][tap][ci] (zero outside the 32 x 32 image);
their gradients are the exact sums below; the GPU's differ only by the
FP32 accumulation order (and BF16 rounding of the activations it stores),
which the tolerances state."""
import numpy as np
import pytest

import vp8a
from util import windows_ref
from vp8a import abi, learned, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def bf16(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).float().numpy()


def conv_ref(x, w, b, relu):
    n, s, _, cin = x.shape
    cout = w.shape[0]
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((n, s, s, cout), np.float64) + b
    for tap in range(9):
        dy, dx = tap // 3 - 1, tap % 3 - 1
        out += np.einsum("nyxc,oc->nyxo", xp[:, 1 + dy:1 + dy + s, 1 + dx:1 + dx + s, :], w[:, tap, :])
    return np.maximum(out, 0) if relu else out


def conv_bwd_ref(x, w, dy_, x_relu):
    n, s, _, cin = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dyp = np.pad(dy_, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dw = np.zeros(w.shape, np.float64)
    dx = np.zeros(x.shape, np.float64)
    for tap in range(9):
        ty, tx = tap // 3 - 1, tap % 3 - 1
        dw[:, tap, :] = np.einsum("nyxo,nyxc->oc", dy_, xp[:, 1 + ty:1 + ty + s, 1 + tx:1 + tx + s, :])
        dx += np.einsum("nyxo,oc->nyxc", dyp[:, 1 - ty:1 - ty + s, 1 - tx:1 - tx + s, :], w[:, tap, :])
    if x_relu:
        dx = dx * (x > 0)
    return dw, dy_.sum(axis=(0, 1, 2)), dx


def dev_bf16(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).cuda()


@pytest.mark.parametrize("cin,cout,relu", [(2, 32, True), (32, 32, True), (32, 1, False)])
def test_conv_forward_and_gradients_match_fp32_reference(ctx, cin, cout, relu):
    rng = np.random.default_rng(cin * 100 + cout)
    n = 3
    x = bf16(rng.standard_normal((n, 32, 32, cin)))
    if cin == 32:
        x = np.maximum(x, 0)  # an activation out of a ReLU
    w = bf16(rng.standard_normal((cout, 9, cin)) * 0.2)
    b = rng.standard_normal(cout).astype(np.float32) * 0.1
    lib = ctx._lib
    dx_, dw_, db_ = dev_bf16(x), dev_bf16(w.reshape(-1)), torch.from_numpy(b).cuda()
    yf = torch.empty((n, 32, 32, cout), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()  # inputs in place before the library's stream reads them
    assert lib.vp8a_lp_conv_forward(ctx.handle, dx_.data_ptr(), cin, dw_.data_ptr(), db_.data_ptr(), cout, n,
                                    int(relu), None, yf.data_ptr()) == abi.OK
    ctx.synchronize()
    want = conv_ref(x, w, b, relu)
    got = yf.cpu().numpy()
    # FP32 accumulation of BF16 products: the order differs, nothing else.
    assert np.abs(got - want).max() <= 1e-4 * max(1.0, np.abs(want).max())
    # Gradients for a BF16 upstream gradient.
    dy = bf16(rng.standard_normal((n, 32, 32, cout)) * 0.05)
    gw = torch.zeros(cout * 9 * cin, device="cuda")
    gb = torch.zeros(cout, device="cuda")
    gx = torch.empty((n, 32, 32, cin), dtype=torch.bfloat16, device="cuda")
    x_relu = int(cin == 32)
    ddy = dev_bf16(dy)
    torch.cuda.synchronize()
    assert lib.vp8a_lp_conv_backward(ctx.handle, dx_.data_ptr(), cin, dw_.data_ptr(), cout, n, ddy.data_ptr(),
                                     x_relu, gx.data_ptr(), gw.data_ptr(), gb.data_ptr()) == abi.OK
    ctx.synchronize()
    rdw, rdb, rdx = conv_bwd_ref(x, w, dy, x_relu)
    assert np.abs(gw.cpu().numpy().reshape(rdw.shape) - rdw).max() <= 1e-4 * max(1.0, np.abs(rdw).max())
    assert np.abs(gb.cpu().numpy() - rdb).max() <= 1e-4 * max(1.0, np.abs(rdb).max())
    # dX is stored as BF16: within half an ulp of BF16 (2^-8 relative).
    gxn = gx.float().cpu().numpy()
    assert np.all(np.abs(gxn - rdx) <= np.abs(rdx) * 2.0 ** -8 + 1e-6)


@pytest.mark.parametrize("relu", [True, False])
def test_tensor_core_conv_32_to_32_matches_fp32_reference(ctx, relu):
    # BF16 output of a 32 -> 32 layer: the tcgen05 path (TMEM accumulators,
    # shared-memory descriptors). FP32 accumulation in another order, then
    # one BF16 rounding: within half a BF16 ulp of the FP32 reference plus
    # the accumulation slack.
    rng = np.random.default_rng(77 + relu)
    n = 7
    x = np.maximum(bf16(rng.standard_normal((n, 32, 32, 32))), 0)
    w = bf16(rng.standard_normal((32, 9, 32)) * 0.2)
    b = rng.standard_normal(32).astype(np.float32) * 0.1
    lib = ctx._lib
    dx_, dw_, db_ = dev_bf16(x), dev_bf16(w.reshape(-1)), torch.from_numpy(b).cuda()
    y = torch.full((n, 32, 32, 32), float("nan"), dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    assert lib.vp8a_lp_conv_forward(ctx.handle, dx_.data_ptr(), 32, dw_.data_ptr(), db_.data_ptr(), 32, n,
                                    int(relu), y.data_ptr(), None) == abi.OK
    assert lib.vp8a_ctx_synchronize(ctx.handle) == abi.OK
    want = conv_ref(x, w, b, relu)
    got = y.float().cpu().numpy()
    assert np.isfinite(got).all()
    slack = 1e-4 * max(1.0, np.abs(want).max())
    assert np.all(np.abs(got - want) <= np.abs(want) * 2.0 ** -8 + slack)


def test_softmax_cross_entropy_and_adam(ctx):
    rng = np.random.default_rng(3)
    n = 5
    z = (rng.standard_normal((n, 1024)) * 3).astype(np.float32)
    lab = np.array([0, 1023, 517, -1, 44], np.int32)
    dz = torch.from_numpy(z).cuda()
    dl = torch.from_numpy(lab).cuda()
    g = torch.empty((n, 1024), dtype=torch.bfloat16, device="cuda")
    loss = torch.zeros(1, device="cuda")
    prob = torch.zeros(n, device="cuda")
    torch.cuda.synchronize()
    assert ctx._lib.vp8a_lp_softmax_ce(ctx.handle, dz.data_ptr(), dl.data_ptr(), n, g.data_ptr(), loss.data_ptr(),
                                       prob.data_ptr()) == abi.OK
    ctx.synchronize()
    p = np.exp(z - z.max(1, keepdims=True))
    p /= p.sum(1, keepdims=True)
    want_loss = -sum(np.log(p[i, lab[i]]) for i in range(n) if lab[i] >= 0)
    assert abs(loss.item() - want_loss) <= 1e-4 * abs(want_loss)
    onehot = np.zeros_like(p)
    for i in range(n):
        if lab[i] >= 0:
            onehot[i, lab[i]] = 1
    want_g = np.where((lab >= 0)[:, None], (p - onehot) / n, 0)
    assert np.all(np.abs(g.float().cpu().numpy() - want_g) <= np.abs(want_g) * 2.0 ** -8 + 1e-7)
    # Adam against its definition.
    w = rng.standard_normal(1000).astype(np.float32)
    gr = rng.standard_normal(1000).astype(np.float32)
    m = np.zeros_like(w)
    v = np.zeros_like(w)
    dw_, dg, dm, dv = (torch.from_numpy(a.copy()).cuda() for a in (w, gr, m, v))
    wb = torch.empty(1000, dtype=torch.bfloat16, device="cuda")
    torch.cuda.synchronize()
    for step in (1, 2):
        assert ctx._lib.vp8a_lp_adam(ctx.handle, dw_.data_ptr(), dg.data_ptr(), dm.data_ptr(), dv.data_ptr(), 1000,
                                     1e-3, 0.9, 0.999, 1e-8, step, wb.data_ptr()) == abi.OK
        m = 0.9 * m + 0.1 * gr
        v = 0.999 * v + 0.001 * gr * gr
        w = w - 1e-3 * (m / (1 - 0.9 ** step)) / (np.sqrt(v / (1 - 0.999 ** step)) + 1e-8)
    ctx.synchronize()
    assert np.abs(dw_.cpu().numpy() - w).max() <= 1e-6
    # The BF16 copy is the rounding of the FP32 master weights.
    assert torch.equal(wb, dw_.to(torch.bfloat16))


def moving_sequence(w, h, seed, n=6):
    frames, _ = synth.make_sequence(w, h, n, seed=seed, pieces=4, occluders=3)
    return frames


def dataset(ctx, sizes_seeds, lam):
    with learned.on_ctx_stream(ctx):
        x, y = _dataset(ctx, sizes_seeds, lam)
    ctx.synchronize()
    return x, y


def _dataset(ctx, sizes_seeds, lam):
    xs, ys = [], []
    for (w, h, seed) in sizes_seeds:
        frames = moving_sequence(w, h, seed)
        for k in range(1, len(frames)):
            ref = vp8a.pad_to_mb(*frames[k - 1])
            lab, _ = learned.labels_from_search(ctx, frames[k], ref, lam)
            mbr, mbc = (h + 15) // 16, (w + 15) // 16
            xy = learned.all_mbs(mbc, mbr)
            src = torch.from_numpy(frames[k][0]).cuda()
            refy = torch.from_numpy(ref[0]).cuda()
            xs.append(learned.windows(ctx, src, refy[:h, :w], xy))
            ys.append(torch.from_numpy(lab).cuda())
    return torch.cat(xs), torch.cat(ys)


def test_training_reduces_loss_and_finds_the_search_vectors(ctx):
    lam = vp8a.rd_lambda(44)
    x, y = dataset(ctx, [(320, 240, 11), (320, 240, 12), (176, 144, 13)], lam)
    net = learned.ProposalNet(ctx, seed=1)
    n = x.shape[0]
    g = torch.Generator(device="cpu").manual_seed(0)

    def top4(net_):
        cells = net_.propose(x, 4)
        with learned.on_ctx_stream(ctx):
            return float(((cells == y[:, None].long()).any(1) & (y >= 0)).float().sum() / (y >= 0).sum())

    before = top4(net)
    losses = []
    first_ref = None
    for it in range(150):
        with learned.on_ctx_stream(ctx):
            idx = torch.randint(0, n, (256,), generator=g).cuda()
            xb, yb = x[idx].contiguous(), y[idx].contiguous()
        if it == 0:
            # The definition on this batch, in float64 numpy from the net's
            # own FP32 scores: mean over labelled items of
            # logsumexp(scores) - scores[label].
            scores = net.forward(xb)
            with learned.on_ctx_stream(ctx):
                sc = scores.double().cpu().numpy()
                lab = yb.cpu().numpy()
            keep = lab >= 0
            m = sc.max(1, keepdims=True)
            lse = (m[:, 0] + np.log(np.exp(sc - m).sum(1)))
            first_ref = float(np.mean((lse - sc[np.arange(sc.shape[0]), np.maximum(lab, 0)])[keep]))
        losses.append(net.train_step(xb, yb, lr=2e-3))
    after = top4(net)
    # A fresh net's scores are near-uniform over the 1024 cells: the first
    # loss is close to ln 1024 and equals the definition on its batch.
    assert abs(losses[0] - first_ref) <= 1e-3 * first_ref, (losses[0], first_ref)
    assert 0.5 * np.log(1024) < losses[0] < 2.0 * np.log(1024), losses[0]
    assert all(v > 0.0 for v in losses), min(losses)
    assert np.mean(losses[-20:]) < 0.7 * np.mean(losses[:10]), (losses[:10], losses[-20:])
    assert after > before + 0.2, (before, after)


def test_learned_search_is_exact_and_beats_zero_seeds(ctx, oracle):
    lam = vp8a.rd_lambda(44)
    x, y = dataset(ctx, [(320, 240, 21), (320, 240, 22)], lam)
    net = learned.ProposalNet(ctx, seed=2)
    g = torch.Generator(device="cpu").manual_seed(1)
    for it in range(150):
        with learned.on_ctx_stream(ctx):
            idx = torch.randint(0, x.shape[0], (256,), generator=g).cuda()
            xb, yb = x[idx].contiguous(), y[idx].contiguous()
        net.train_step(xb, yb, lr=2e-3)
    frames = moving_sequence(320, 240, 29)
    ref = vp8a.pad_to_mb(*frames[2])
    src = frames[3]
    xy = learned.all_mbs(20, 15)
    srcd = torch.from_numpy(src[0]).cuda()
    refd = torch.from_numpy(ref[0]).cuda()
    mv, sad, fb = learned.learned_search(ctx, net, srcd, refd, xy)
    # Exact: every SAD is the plain search's SAD at the returned vector.
    xyh = xy.cpu().numpy().view(np.uint32)
    src_mbs = learned._source_mbs(srcd, xy, 240, 320).cpu().numpy()
    want = oracle.mb_luma_sad_at_mv(ref[0], src_mbs, xyh, mv)
    assert np.array_equal(sad, np.asarray(want, np.uint32))
    # The ablation: the same search seeded at the zero vector only.
    zero = torch.full((xy.shape[0], 4), 16 * 32 + 16, dtype=torch.int64, device="cuda")
    _, sad0, _ = learned.learned_search(ctx, net, srcd, refd, xy, seeds=zero)
    assert sad.mean() < sad0.mean(), (sad.mean(), sad0.mean())
    # And the plain exhaustive search's per-MB result for reference.
    _, plain_sad = learned.labels_from_search(ctx, src, ref, lam)
    assert sad.mean() <= 1.15 * plain_sad.mean(), (sad.mean(), plain_sad.mean())


@pytest.mark.parametrize("k,radius", [(4, 2), (1, 4), (3, 1)])
def test_seeded_search_is_the_first_smallest_sad(ctx, oracle, k, radius):
    # vp8a_lp_seeded_search against its definition: every whole-pel vector
    # within +-radius px of each seed cell, SADs from the plain search's
    # SAD (the oracle), first smallest in seed, row, column order. Seeds
    # near the grid's edges put windows across the reference's border.
    import ctypes as C

    frames = moving_sequence(176, 144, 13)
    ref = vp8a.pad_to_mb(*frames[2])
    src = frames[3]
    n_mb = 11 * 9
    xy = learned.all_mbs(11, 9)
    srcd = torch.from_numpy(src[0]).cuda()
    refd = torch.from_numpy(np.ascontiguousarray(ref[0])).cuda()
    src_mbs = learned._source_mbs(srcd, xy, 144, 176)
    rng = np.random.default_rng(k * 10 + radius)
    cells = rng.integers(0, 1024, (n_mb, k)).astype(np.int32)
    cells[0] = 0
    cells[1] = 1023
    dseeds = torch.from_numpy(cells).cuda()
    out = torch.empty((n_mb, 2), dtype=torch.int32, device="cuda")
    lib = vp8a.load()
    r = vp8a.frames.luma_ref(refd, width=176, height=144)
    with learned.on_ctx_stream(ctx):
        st = lib.vp8a_lp_seeded_search(ctx.handle, C.byref(r), src_mbs.data_ptr(), xy.data_ptr(),
                                       dseeds.data_ptr(), k, radius, n_mb, out.data_ptr())
    assert st == 0, lib.vp8a_last_error()
    ctx.synchronize()
    got = out.cpu().numpy()
    mv = got[:, 0].copy().view(np.int16).reshape(n_mb, 2)
    sad = got[:, 1].view(np.uint32)
    offs = [(dr, dc) for dr in range(-radius, radius + 1) for dc in range(-radius, radius + 1)]
    cand = np.array([[((c // 32 - 16) * 8 + 4 * dr, (c % 32 - 16) * 8 + 4 * dc) for c in row for dr, dc in offs]
                     for row in cells], np.int16)
    ncand = cand.shape[1]
    xyh = np.repeat(xy.cpu().numpy().view(np.uint32), ncand, axis=0)
    sm = np.repeat(src_mbs.cpu().numpy(), ncand, axis=0)
    all_sad = np.asarray(oracle.mb_luma_sad_at_mv(ref[0], sm, xyh, cand.reshape(-1, 2)), np.uint32).reshape(n_mb, ncand)
    best = all_sad.argmin(axis=1)
    assert np.array_equal(sad, all_sad[np.arange(n_mb), best])
    assert np.array_equal(mv, cand[np.arange(n_mb), best])
    # Out-of-range arguments are errors.
    with learned.on_ctx_stream(ctx):
        st = lib.vp8a_lp_seeded_search(ctx.handle, C.byref(r), src_mbs.data_ptr(), xy.data_ptr(),
                                       dseeds.data_ptr(), 4, 3, n_mb, out.data_ptr())
    assert st == abi.E_INVALID_ARGUMENT


def test_filter_sweep_window_matches_the_full_table(ctx, oracle):
    from test_gpu_lf import lf_case

    src, recon, m = lf_case(160, 96, seed=4)
    base = abi.filter_config(0, 2, delta_enabled=1, ref_delta_last=3)
    full = vp8a.filter_sweep(ctx, recon, m, base, src)
    win = vp8a.filter_sweep_window(ctx, recon, m, base, src, 20, 28)
    inside = np.zeros((64, 8), bool)
    inside[0] = True
    inside[20:29] = True
    assert np.array_equal(win[inside], full[inside])
    assert (win[~inside] == np.uint64(2 ** 64 - 1)).all()


def test_lf_head_matches_its_definition(ctx):
    rng = np.random.default_rng(8)
    c, levels = 33, 64
    sums = (rng.standard_normal(c) * 100).astype(np.float32)
    count = 50.0
    w = (rng.standard_normal(levels * c) * 0.1).astype(np.float32)
    b = (rng.standard_normal(levels) * 0.1).astype(np.float32)
    d = {k: torch.from_numpy(v).cuda() for k, v in (("s", sums), ("w", w), ("b", b))}
    z = torch.empty(levels, device="cuda")
    gw = torch.zeros(levels * c, device="cuda")
    gb = torch.zeros(levels, device="cuda")
    loss = torch.zeros(1, device="cuda")
    torch.cuda.synchronize()
    assert ctx._lib.vp8a_lp_lf_head(ctx.handle, d["s"].data_ptr(), count, c, d["w"].data_ptr(), d["b"].data_ptr(),
                                    levels, 17, z.data_ptr(), gw.data_ptr(), gb.data_ptr(), loss.data_ptr()) == abi.OK
    ctx.synchronize()
    f = sums / count
    zz = w.reshape(levels, c) @ f + b
    p = np.exp(zz - zz.max())
    p /= p.sum()
    g = p.copy()
    g[17] -= 1
    assert np.allclose(z.cpu().numpy(), zz, rtol=1e-5, atol=1e-5)
    assert np.allclose(gb.cpu().numpy(), g, rtol=1e-4, atol=1e-6)
    assert np.allclose(gw.cpu().numpy().reshape(levels, c), np.outer(g, f), rtol=1e-4, atol=1e-6)
    assert abs(loss.item() + np.log(p[17])) < 1e-4


@pytest.mark.parametrize("k", [1, 4, 16])
def test_fused_net_matches_the_layered_net(ctx, k):
    # vp8a_lp_net_propose (the four layers in one launch, activations on
    # chip) against the layer-by-layer forward of the same net: the same
    # sums over BF16 activations in another FP32 accumulation order, so an
    # activation may round to the neighbouring BF16 value; the scores agree
    # within 2^-6 of their range. The cells are exactly the first-index
    # top k of the fused scores. 300 images: more than one per CTA.
    rng = np.random.default_rng(k)
    frames = moving_sequence(176, 144, 21)
    srcd = torch.from_numpy(frames[3][0]).cuda()
    refd = torch.from_numpy(frames[2][0]).cuda()
    xw = learned.windows(ctx, srcd, refd, learned.all_mbs(11, 9))
    xr = dev_bf16(rng.standard_normal((300 - xw.shape[0], 32, 32, 2)) * 40)
    with learned.on_ctx_stream(ctx):
        x = torch.cat([xw, xr]).contiguous()
    net = learned.ProposalNet(ctx, seed=3 + k)
    want = net.forward(x)
    logits = torch.full((300, 1024), float("nan"), dtype=torch.float32, device="cuda")
    cells = net.propose(x, k, logits=logits)
    ctx.synchronize()
    got, want, cells = logits.cpu().numpy(), want.cpu().numpy(), cells.cpu().numpy()
    assert np.isfinite(got).all()
    scale = np.abs(want).max(axis=1, keepdims=True) + 1e-3
    assert np.all(np.abs(got - want) <= scale * 2.0 ** -6)
    assert cells.dtype == np.int32 and cells.shape == (300, k)
    assert np.array_equal(cells, np.argsort(-got, axis=1, kind="stable")[:, :k])


def test_fused_net_arguments(ctx):
    net = learned.ProposalNet(ctx, seed=1)
    x = torch.zeros((2, 32, 32, 2), dtype=torch.bfloat16, device="cuda")
    L = net.layers
    lib = ctx._lib
    cells = torch.zeros((2, 17), dtype=torch.int32, device="cuda")
    args = [x.data_ptr(), 2] + [v for li in L for v in (li["wh"].data_ptr(), li["b"].data_ptr())]
    for bad_k in (0, 17):
        assert lib.vp8a_lp_net_propose(ctx.handle, *args, bad_k, cells.data_ptr(), None) == abi.E_INVALID_ARGUMENT
    assert lib.vp8a_lp_net_propose(ctx.handle, x.data_ptr(), 0, *args[2:], 4, None, None) == abi.OK
    ctx.synchronize()


@pytest.mark.parametrize("w,h", [(176, 144), (72, 40)])
def test_windows_match_their_definition(ctx, w, h):
    # vp8a_lp_windows bit for bit against the numpy definition, frames whose
    # windows cross every edge of the planes.
    frames = moving_sequence(w, h, 17)
    srcd = torch.from_numpy(np.ascontiguousarray(frames[3][0])).cuda()
    refd = torch.from_numpy(np.ascontiguousarray(frames[2][0])).cuda()
    mbc, mbr = (w + 15) // 16, (h + 15) // 16
    xy = learned.all_mbs(mbc, mbr)
    got = learned.windows(ctx, srcd, refd, xy)
    ctx.synchronize()
    want = bf16(windows_ref(frames[3][0], frames[2][0], xy.cpu().numpy().view(np.uint32)))
    assert np.array_equal(got.float().cpu().numpy(), want)
