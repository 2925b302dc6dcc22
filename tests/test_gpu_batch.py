"""Batched (multi-image) path on the GPU: every image of a batch renders
exactly as it does alone, gradients equal the per-image fused-L2 gradients,
the batched loss reduces like the single-image one, the persistent tile walk
equals one CTA per tile, the guarded Adam matches torch's Adam and skips
overflowed steps, and a captured fit equals the eager one."""
import pytest
import torch

from lig_b200 import _lib, ops
from lig_b200.batch import BatchedFit, BatchLayout, autotune, uneven_batch
from lig_b200.fused import render_l2_loss
from tests._scene import np_, rel_err

pytestmark = pytest.mark.gpu

SHAPES = [(64, 96), (130, 77), (16, 16), (200, 150), (33, 250)]


def _targets(shapes, seed=11):
    g = torch.Generator().manual_seed(seed)
    return [torch.rand(h, w, 3, generator=g).cuda() for h, w in shapes]


def _fit(shapes, counts, block=16, persistent=False, graph=False, **kw):
    return BatchedFit(_targets(shapes), counts, block=block, persistent=persistent, graph=graph,
                      diag=(0.5, 5.0), **kw)


def _single(means, chol, rgbs, H, W, B):
    """Single-image projection + binning + forward through the ops layer
    (which, unlike the drop-in API, also takes B = 32).  -> (img, wsum, fin,
    binning)."""
    with torch.no_grad():
        xys, ext, con, cnt = ops.project_fwd(chol, means, None, H, W, B, True)
        b, outs = ops.bin_gaussians(xys, ext, cnt, H, W, B, after_enqueue=lambda bb: ops.raster_fwd(
            H, W, B, bb.gaussian_ids_sorted, bb.tile_bins, bb.total, xys, con, rgbs, None, False))
    return outs[0], outs[1], outs[5], b


@pytest.mark.parametrize("block", [8, 16, 32])
@pytest.mark.parametrize("persistent", [False, True])
def test_batch_images_equal_single_renders(block, persistent):
    counts = [900, 1200, 0, 3000, 700]  # image 2 has no Gaussians: white
    fit = _fit(SHAPES, counts, block=block, persistent=persistent)
    img = fit.render()
    torch.cuda.synchronize()
    L = fit.L
    for i, (h, w) in enumerate(SHAPES):
        got = L.image(img, i)
        got_w = L.image(fit.wsum.view(-1, 1), i)[..., 0]
        got_f = L.image(fit.fin.view(-1, 1), i)[..., 0]
        if counts[i] == 0:
            assert torch.all(got == 1) and torch.all(got_w == 0) and torch.all(got_f == 0)
            continue
        mu, ch, co = fit.params_of(i)
        s_img, s_w, s_fin, _ = _single(mu.clone(), ch.clone(), co.clone(), h, w, block)
        assert torch.equal(got, s_img), f"image {i}"
        assert torch.equal(got_w, s_w), f"wsum {i}"
        # final indices are global list positions: the image's own + its offset
        off = int(fit.cnt[:L.g_off[i]].long().sum())
        ok = (got_f == s_fin + off) | ((got_f == 0) & (s_fin == 0))
        assert bool(ok.all()), f"final_idx {i}"


def test_batch_sorted_ids_and_bins_match_single():
    block = 16
    counts = [500, 800, 300]
    shapes = SHAPES[:2] + [SHAPES[3]]
    fit = _fit(shapes, counts, block=block)
    fit.render()
    torch.cuda.synchronize()
    L = fit.L
    m_off = 0
    for i, (h, w) in enumerate(shapes):
        mu, ch, co = fit.params_of(i)
        b = _single(mu.clone(), ch.clone(), co.clone(), h, w, block)[3]
        m = b.num_intersects
        got_ids = fit.gids[m_off:m_off + m] - L.g_off[i]
        assert torch.equal(got_ids, b.gaussian_ids_sorted[:m])
        bins = fit.bins[L.tile_off[i]:L.tile_off[i + 1]]
        single = b.tile_bins.view(-1, 2)
        nonempty = single[:, 1] > single[:, 0]
        assert torch.equal(bins[nonempty] - m_off, single[nonempty])
        m_off += m
    assert int(fit.total.item()) == m_off


def test_batch_fused_l2_gradients_match_single():
    counts = [900, 1200, 400, 3000, 700]
    fit = _fit(SHAPES, counts)
    fit._enqueue_step()  # one eager iteration: gradients in fit.grad, then Adam
    torch.cuda.synchronize()
    # recompute with the pre-step parameters: undo is not possible, so rebuild
    fit2 = _fit(SHAPES, counts)
    L = fit2.L
    targets = _targets(SHAPES)
    fit2._render(fit2._stream())
    torch.cuda.synchronize()
    st = fit2._stream()
    l_ws = torch.empty(_lib.lib.lig_l2_batch_workspace_bytes(L.n), dtype=torch.uint8,
                       device="cuda")
    ops.call("lig_l2_clamped_loss_batch", _lib.LIG_F32, *L.hw_args(), ops._p(fit2.img),
             ops._p(fit2.target), ops._p(fit2.loss), ops._p(fit2.per_image), ops._p(l_ws),
             l_ws.numel(), st)
    ops.call("lig_raster_bwd_l2_batch", _lib.LIG_F32, *L.args(), L.block, ops._p(fit2.gids),
             ops._p(fit2.bins), ops._p(fit2.total), ops._p(fit2.cum), ops._p(fit2.xys),
             ops._p(fit2.con), ops._p(fit2.rgbs), None, ops._p(fit2.fin), ops._p(fit2.img),
             ops._p(fit2.target), ops._p(fit2.one), 0.0, 0, ops._p(fit2.work),
             ops._p(fit2.r_ws), fit2.r_ws.numel(), ops._p(fit2.v_xy), ops._p(fit2.v_abs),
             ops._p(fit2.v_con), ops._p(fit2.g_rgbs), None, st)
    ops.call("lig_project_bwd_batch", _lib.LIG_F32, *L.args(), 1, ops._p(fit2.chol),
             ops._p(fit2.means), None, L.block, ops._p(fit2.v_xy), 2, ops._p(fit2.v_con), 3,
             ops._p(fit2.g_chol), ops._p(fit2.g_means), st)
    torch.cuda.synchronize()
    total = 0.0
    for i, (h, w) in enumerate(SHAPES):
        mu, ch, co = [t.clone().requires_grad_() for t in fit2.params_of(i)]
        loss = render_l2_loss(ch, mu, co, None, targets[i], h, w, 16)
        loss.backward()
        total += loss.item()
        assert abs(fit2.per_image[i].item() - loss.item()) <= 1e-6 * loss.item()
        gm = L.points_of(fit2.g_means, i)
        gc = L.points_of(fit2.g_chol, i)
        gr = L.points_of(fit2.g_rgbs, i)
        assert rel_err(np_(gm), np_(mu.grad)) <= 1e-5
        assert rel_err(np_(gc), np_(ch.grad)) <= 1e-5
        assert rel_err(np_(gr), np_(co.grad)) <= 1e-5
    assert abs(fit2.loss.item() - total) <= 1e-5 * total
    # the first fit's step (fused-L2 forward, backward from its difference)
    # gives the same loss and gradients
    assert abs(fit.loss.item() - fit2.loss.item()) <= 1e-6 * fit2.loss.item()
    assert torch.allclose(fit.per_image, fit2.per_image, rtol=1e-6, atol=0)
    assert rel_err(np_(fit.grad), np_(fit2.grad)) <= 1e-5


def test_batch_of_one_loss_bit_exact():
    h, w = 120, 130
    g = torch.Generator().manual_seed(5)
    img = (torch.rand(h * w, 3, generator=g) * 1.4 - 0.2).cuda()
    tgt = torch.rand(h * w, 3, generator=g).cuda()
    single = ops.l2_clamped_loss(img, tgt)
    L = BatchLayout([h], [w], [0], 16)
    out = torch.zeros((), device="cuda")
    per = torch.zeros(1, device="cuda")
    ws = torch.empty(_lib.lib.lig_l2_batch_workspace_bytes(1), dtype=torch.uint8, device="cuda")
    ops.call("lig_l2_clamped_loss_batch", _lib.LIG_F32, *L.hw_args(), ops._p(img), ops._p(tgt),
             ops._p(out), ops._p(per), ops._p(ws), ws.numel(),
             ops._stream(torch.device("cuda")))
    assert torch.equal(out, single.reshape(()))
    assert torch.equal(per[0], single.reshape(()))


def test_adam_matches_torch_adam():
    n = 10_003
    g = torch.Generator().manual_seed(3)
    p0 = torch.randn(n, generator=g).cuda()
    grads = [torch.randn(n, generator=g).cuda() for _ in range(5)]
    ref = p0.clone().requires_grad_()
    opt = torch.optim.Adam([ref], lr=1e-2)
    for gr in grads:
        ref.grad = gr.clone()
        opt.step()
    p = p0.clone()
    m, v = torch.zeros_like(p), torch.zeros_like(p)
    step = torch.zeros(1, dtype=torch.int32, device="cuda")
    sc = torch.empty(64, dtype=torch.uint8, device="cuda")
    st = ops._stream(torch.device("cuda"))
    for gr in grads:
        ops.call("lig_adam_step", n, ops._p(p), ops._p(gr), ops._p(m), ops._p(v), 1e-2, 0.9,
                 0.999, 1e-8, None, ops._p(step), None, ops._p(sc), st)
    assert int(step.item()) == 5
    assert rel_err(np_(p - p0), np_(ref.detach() - p0)) <= 1e-5


def test_adam_skips_on_overflow_status():
    n = 1000
    p = torch.randn(n, device="cuda")
    p0 = p.clone()
    gr = torch.randn(n, device="cuda")
    m, v = torch.zeros_like(p), torch.zeros_like(p)
    step = torch.zeros(1, dtype=torch.int32, device="cuda")
    skipped = torch.zeros(1, dtype=torch.int32, device="cuda")
    status = torch.tensor([_lib.LIG_STATUS_OVERFLOW], dtype=torch.int32, device="cuda")
    sc = torch.empty(64, dtype=torch.uint8, device="cuda")
    st = ops._stream(torch.device("cuda"))
    ops.call("lig_adam_step", n, ops._p(p), ops._p(gr), ops._p(m), ops._p(v), 1e-2, 0.9, 0.999,
             1e-8, ops._p(status), ops._p(step), ops._p(skipped), ops._p(sc), st)
    assert torch.equal(p, p0) and int(step.item()) == 0 and int(skipped.item()) == 1
    assert torch.all(m == 0) and torch.all(v == 0)


def test_overflow_is_skipped_and_redone():
    """Capacity far below the intersection count: the overflowed steps are
    skipped on the device, the capacity grows, and exactly `iters` steps end
    up applied — the same parameters as a fit that never overflowed."""
    shapes, counts = SHAPES[:4], [900, 1200, 400, 3000]
    a = _fit(shapes, counts, graph=True)
    a._size_capacity(1000)  # << M: every step overflows until recovery
    a.slack = 1.25
    st = a.fit(5)
    assert st.skipped >= 1
    assert bool((a.steps == 5).all())
    b = _fit(shapes, counts, graph=True)
    b.fit(5)
    assert bool((b.steps == 5).all()) and b.stats.skipped == 0
    assert rel_err(np_(a.flat), np_(b.flat)) <= 1e-5


def test_graph_fit_matches_eager_fit():
    shapes, counts = SHAPES, [900, 1200, 400, 3000, 700]
    a = _fit(shapes, counts, graph=True)
    b = _fit(shapes, counts, graph=False)
    a.fit(6)
    b.fit(6)
    assert a.graph is not None and b.graph is None
    assert rel_err(np_(a.flat), np_(b.flat)) <= 1e-5


def test_batched_fit_reduces_every_image_loss():
    targets, counts = uneven_batch(n_img=6, size_scale=0.08)
    fit = BatchedFit(targets, counts, lr=1e-2, graph=True)
    p0 = fit.psnr()
    fit.fit(40)
    p1 = fit.psnr()
    assert all(b > a for a, b in zip(p0, p1)), (p0, p1)


def test_autotune_returns_a_measured_choice():
    targets, counts = uneven_batch(n_img=4, size_scale=0.05)
    res = autotune(targets, counts, blocks=(8, 16), walks=(False, True), iters=2)
    assert res["block"] in (8, 16) and res["persistent"] in (False, True)
    assert len(res["table"]) == 4 and all(r["s_per_iter"] > 0 for r in res["table"])


def test_batched_adam_per_image_steps_match_single_adam():
    """lig_adam_step_batch with per-image step counts == lig_adam_step run on
    each image's parameters alone (images at different steps)."""
    counts = [5, 0, 7, 3]
    N = sum(counts)
    g = torch.Generator().manual_seed(4)
    p0 = torch.randn(8 * N, generator=g).cuda()
    grads = [torch.randn(8 * N, generator=g).cuda() for _ in range(3)]
    start = [0, 4, 2, 9]  # images already at different Adam steps
    L = BatchLayout([8] * 4, [8] * 4, counts, 16)
    st = ops._stream(torch.device("cuda"))
    p = p0.clone()
    m, v = torch.zeros_like(p), torch.zeros_like(p)
    steps = torch.tensor(start, dtype=torch.int32, device="cuda")
    sc = torch.empty(_lib.lib.lig_adam_batch_scratch_bytes(4), dtype=torch.uint8, device="cuda")
    for gr in grads:
        ops.call("lig_adam_step_batch", 4, L.args()[3], ops._p(p), ops._p(gr), ops._p(m),
                 ops._p(v), 1e-2, 0.9, 0.999, 1e-8, None, ops._p(steps), None, ops._p(sc),
                 sc.numel(), st)
    assert steps.tolist() == [s + 3 for s in start]

    def parts(flat, i):  # image i's 8 n_i values, in (means, chol, rgb) order
        a, b = L.g_off[i], L.g_off[i + 1]
        return torch.cat([flat[2 * a:2 * b], flat[2 * N + 3 * a:2 * N + 3 * b],
                          flat[5 * N + 3 * a:5 * N + 3 * b]])

    for i, n in enumerate(counts):
        if n == 0:
            continue
        q = parts(p0, i).clone()
        mq, vq = torch.zeros_like(q), torch.zeros_like(q)
        s1 = torch.tensor([start[i]], dtype=torch.int32, device="cuda")
        sc1 = torch.empty(64, dtype=torch.uint8, device="cuda")
        for gr in grads:
            ops.call("lig_adam_step", q.numel(), ops._p(q), ops._p(parts(gr, i).contiguous()),
                     ops._p(mq), ops._p(vq), 1e-2, 0.9, 0.999, 1e-8, None, ops._p(s1), None,
                     ops._p(sc1), st)
        assert torch.allclose(parts(p, i), q, rtol=1e-6, atol=1e-7)


def test_levelfit_graph_engine_matches_autograd_engine():
    """LevelFit's CUDA-graph engine (one-image BatchedFit, flat Adam) follows
    the autograd engine (drop-in API + torch Adam); alternating two target
    buffers replays one graph per buffer with the same results."""
    from lig_b200.fit import LevelFit
    H, W, n = 96, 112, 1500
    g = torch.Generator().manual_seed(12)
    target = torch.rand(H, W, 3, generator=g).cuda()
    a = LevelFit(n, H, W, lr=1e-2, diag=(0.5, 4.0), engine="graph")
    b = LevelFit(n, H, W, lr=1e-2, diag=(0.5, 4.0), engine="autograd")
    c = LevelFit(n, H, W, lr=1e-2, diag=(0.5, 4.0), engine="graph")
    bufs = [target.clone(), target.clone()]
    la, lb = [], []
    for k in range(8):
        la.append(float(a.step(target)))
        lb.append(float(b.step(target)))
        c.step(bufs[k % 2])
    assert a._batch.graph is not None and len(c._batch._graphs) == 2
    for x, y in zip(la, lb):
        assert abs(x - y) <= 1e-4 * abs(y)
    for p, q in zip((a.means, a.chol, a.rgbs), (b.means, b.chol, b.rgbs)):
        d = (p - q.detach()).abs()
        assert float((d > 1e-4).float().mean()) < 0.01 and float(d.median()) <= 1e-6
    for p, q in zip((a.means, a.chol, a.rgbs), (c.means, c.chol, c.rgbs)):
        d = (p - q).abs()
        assert float((d > 1e-4).float().mean()) < 0.01 and float(d.median()) <= 1e-6


def test_uint8_targets_equal_their_float_conversion():
    """A batch fitted to 8-bit targets (lig_raster_fwd_l2_u8_batch) sees
    exactly the masked difference and losses of the same batch
    fitted to the float targets byte / 255 (torchvision's ToTensor division,
    done on the host as train.py's image loading does); the fits then follow
    each other (the backward's atomic sums differ only in order)."""
    counts = [900, 1200, 0, 3000, 700]
    g = torch.Generator().manual_seed(12)
    u8 = [torch.randint(0, 256, (h, w, 3), generator=g, dtype=torch.uint8) for h, w in SHAPES]
    f32 = [(t.float() / 255).cuda() for t in u8]
    a = BatchedFit([t.cuda() for t in u8], counts, graph=False, diag=(0.5, 5.0))
    b = BatchedFit(f32, counts, graph=False, diag=(0.5, 5.0))
    assert a.target.dtype == torch.uint8 and b.target.dtype == torch.float32
    a.step()
    b.step()
    torch.cuda.synchronize()
    assert torch.equal(a.img, b.img)
    assert torch.equal(a.loss, b.loss) and torch.equal(a.per_image, b.per_image)
    a.fit(5)
    b.fit(5)
    assert rel_err(np_(a.flat), np_(b.flat)) <= 1e-5
    pa, pb = a.psnr(), b.psnr()
    assert all(abs(x - y) <= 1e-4 for x, y in zip(pa, pb))


def test_levelfit_uint8_upload_buffers():
    """LevelFit.step on 8-bit target buffers (the per-step upload of the
    end-to-end bench) equals the step on their float conversion, for the
    graph engine (bytes read in the loss kernel) and the autograd engine
    (converted before the drop-in call)."""
    from lig_b200.fit import LevelFit
    H, W, n = 96, 112, 1500
    g = torch.Generator().manual_seed(13)
    u8 = torch.randint(0, 256, (H, W, 3), generator=g, dtype=torch.uint8)
    f32 = (u8.float() / 255).cuda()
    bufs = [u8.cuda(), u8.cuda()]
    for engine in ("graph", "autograd"):
        a = LevelFit(n, H, W, lr=1e-2, diag=(0.5, 4.0), engine=engine)
        b = LevelFit(n, H, W, lr=1e-2, diag=(0.5, 4.0), engine=engine)
        la = [float(a.step(bufs[k % 2])) for k in range(4)]
        lb = [float(b.step(f32)) for _ in range(4)]
        assert la[0] == lb[0], engine
        for x, y in zip(la, lb):
            assert abs(x - y) <= 1e-5 * abs(y), engine


def test_uint8_target_every_byte_value():
    """Every byte value b reads as the correctly rounded b / 255 (the host's
    division, as ToTensor): with no Gaussians the render is white, so the
    masked difference is exactly 1 - t."""
    g = torch.Generator().manual_seed(14)
    vals = torch.stack([torch.randperm(256, generator=g) for _ in range(3)], 1).to(torch.uint8)
    u8 = vals.reshape(16, 16, 3)
    ref = 1 - u8.float() / 255
    other = torch.randint(0, 256, (64, 64, 3), generator=g, dtype=torch.uint8)
    a = BatchedFit([u8.cuda(), other.cuda()], [0, 200], graph=False)  # image 0: no Gaussians
    a.step()
    torch.cuda.synchronize()
    assert torch.equal(a.L.image(a.img, 0).cpu(), ref)
