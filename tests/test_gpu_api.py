"""The drop-in gsplat2d API on the GPU: end-to-end equality with the reference
pipeline, empty-list branch, error behaviour, absgrad, the `_C` table,
align-corners upscaler, and a LIG-style training step."""
import numpy as np
import pytest
import torch

import lig_b200
from lig_b200 import gsplat2d, ops, upscaler_torch
from lig_b200.gsplat2d import cuda as C
from oracle import oracle as O
from oracle import ref
from tests._scene import chol_to_cov, np_, rel_err, scene

pytestmark = pytest.mark.gpu


def test_install_gsplat2d_aliases():
    lig_b200.install_gsplat2d()
    import gsplat2d as g2
    from gsplat2d.project_gaussians import project_gaussians
    from gsplat2d.rasterize import rasterize_gaussians
    from upscaler_torch import torch_gradient_aware_upscale
    assert g2.project_gaussians_2d is project_gaussians
    assert g2.rasterize_gaussians_sum is rasterize_gaussians
    assert torch_gradient_aware_upscale is upscaler_torch.torch_gradient_aware_upscale


def test_gaussianlig_style_forward_backward_matches_reference():
    """gaussianlig.Gaussian2D.forward + L2 backward, raw cov2d ~ U[0,1)^3
    (non-PD allowed), no opacities, B=16."""
    H, W, B, n = 120, 136, 16, 1500
    g = torch.Generator().manual_seed(2)
    means = (torch.rand(n, 2, generator=g) * torch.tensor([W, H])).cuda()
    cov = torch.rand(n, 3, generator=g).cuda()
    rgbs = torch.rand(n, 3, generator=g).cuda()
    gt = torch.rand(1, 3, H, W, generator=g).cuda()

    def step(project, raster):
        p = [means.clone().requires_grad_(), cov.clone().requires_grad_(),
             rgbs.clone().requires_grad_()]
        xys, ext, con, cnt = project(p[1], p[0], H, W, B)
        img = raster(xys, ext, con, cnt, p[2], None, H, W, B)[0][..., :3]
        img = torch.clamp(img, 0, 1).view(-1, H, W, 3).permute(0, 3, 1, 2).contiguous()
        loss = torch.nn.functional.mse_loss(img, gt)
        loss.backward()
        return img.detach(), [q.grad for q in p]

    img, grads = step(gsplat2d.project_gaussians, gsplat2d.rasterize_gaussians)
    # reference pipeline with the reference kernels; gradients via the same chain rule
    r = ref.render(cov, means, rgbs, None, H, W, B, chol=False)
    rimg = torch.clamp(r["img"], 0, 1).permute(2, 0, 1).unsqueeze(0)
    assert (img - rimg).abs().max().item() <= 1e-5
    v_img = (2.0 / img.numel()) * (rimg - gt) * ((r["img"].permute(2, 0, 1).unsqueeze(0) >= 0) &
                                                  (r["img"].permute(2, 0, 1).unsqueeze(0) <= 1))
    v_img = v_img.squeeze(0).permute(1, 2, 0).contiguous()
    rg = ref.raster_bwd(H, W, B, r["binning"], r["xys"], r["conics"], rgbs, None, r["final_idx"],
                        v_img, torch.zeros(H, W, device="cuda"))
    v_cov, v_mean = ref.project_bwd(r["extents"], cov, r["conics"], rg["v_xy"], rg["v_conic"],
                                    chol=False)
    assert rel_err(np_(grads[0]), np_(v_mean)) <= 1e-4
    assert rel_err(np_(grads[1]), np_(v_cov)) <= 1e-4
    assert rel_err(np_(grads[2]), np_(rg["v_rgb"])) <= 1e-4


def test_empty_list_white_image_and_zero_grads():
    H, W, B = 32, 48, 16
    means = torch.tensor([[-500.0, -500.0], [900.0, 10.0]], device="cuda", requires_grad=True)
    chol = torch.tensor([[1.0, 0.0, 1.0], [1.0, 0.0, 1.0]], device="cuda", requires_grad=True)
    cols = torch.rand(2, 3, device="cuda", requires_grad=True)
    xys, ext, con, cnt = gsplat2d.project_gaussians_cholesky(chol, means, H, W, B)
    assert int(cnt.sum()) == 0
    img, wsum, dx, dy, dxy = gsplat2d.rasterize_gaussians(xys, ext, con, cnt, cols, None, H, W, B,
                                                          compute_upscale_gradients=True)
    assert torch.all(img == 1) and torch.all(wsum == 0) and torch.all(dx == 0)
    (img.sum() + wsum.sum()).backward()
    assert torch.all(cols.grad == 0) and torch.all(means.grad == 0)


def test_errors_and_uint8_and_absgrad():
    H, W, B = 64, 64, 16
    means, L, colors, op = scene(200, H, W)
    xys, ext, con, cnt = gsplat2d.project_gaussians_cholesky(L, means, H, W, B, op)
    with pytest.raises(AssertionError):
        gsplat2d.rasterize_gaussians(xys, ext, con, cnt, colors, op, H, W, 32)
    with pytest.raises(ValueError):
        gsplat2d.rasterize_gaussians(xys[:, :1], ext, con, cnt, colors, op, H, W, B)
    with pytest.raises(ValueError):
        gsplat2d.rasterize_gaussians(xys, ext, con, cnt, colors[:, 0], op, H, W, B)
    with pytest.raises(ValueError):
        gsplat2d.project_gaussians_cholesky(L[:, :2], means, H, W, B)
    c8 = (colors * 255).to(torch.uint8)
    a = gsplat2d.rasterize_gaussians(xys, ext, con, cnt, c8, op, H, W, B)[0]
    b = gsplat2d.rasterize_gaussians(xys, ext, con, cnt, c8.float() / 255, op, H, W, B)[0]
    assert torch.equal(a, b)
    x = xys.detach().clone().requires_grad_()
    img = gsplat2d.rasterize_gaussians(x, ext, con, cnt, colors, op, H, W, B)[0]
    img.sum().backward()
    assert hasattr(x, "absgrad") and x.absgrad.shape == x.shape
    assert torch.all(x.absgrad >= x.grad.abs() - 1e-6)


def test_c_table_matches_reference():
    H, W, B = 90, 100, 16
    means, L, colors, op = scene(700, H, W, opac=(0.05, 1.0))
    cov = chol_to_cov(L)
    n = cov.shape[0]
    for a, b in zip(C.project_gaussians_forward(n, cov, means, op, H, W, B),
                    ref.project_fwd(cov, means, op, H, W, B, False)):
        assert torch.equal(a, b)
    xys, ext, con, cnt = C.project_gaussians_forward_cholesky(n, L, means, op, H, W, B)
    m, cum = gsplat2d.compute_cumulative_intersects(cnt)
    tb = ((W + B - 1) // B, (H + B - 1) // B, 1)
    depths = torch.zeros(n, device="cuda")
    out = gsplat2d.bin_and_sort_gaussians(n, m, xys, depths, ext, cum, tb, B)
    rb = ref.bin_and_sort(xys, ext, cnt, H, W, B)
    for a, b in zip(out, (rb.isect_ids, rb.gaussian_ids, rb.isect_ids_sorted,
                          rb.gaussian_ids_sorted, rb.tile_bins)):
        assert torch.equal(a, b)
    fwd = C.rasterize_forward(tb, (B, B, 1), (W, H, 1), out[3], out[4], xys, con, colors, op, True)
    rf = ref.raster_fwd(H, W, B, rb, xys, con, colors, op, True)
    assert torch.equal(fwd[5], rf["final_idx"])
    assert (fwd[0] - rf["img"]).abs().max().item() <= 1e-5
    c2, e2 = C.compute_cov2d_bounds(n, cov, op)
    rc, re_ = ref.cov2d_bounds(cov, op)
    assert torch.equal(c2, rc) and torch.equal(e2, re_)


def test_align_corners_upscaler_matches_oracle():
    h, w, nh, nw = 40, 52, 101, 157
    g = torch.Generator().manual_seed(8)
    planes = [torch.randn(h, w, 3, generator=g, dtype=torch.float64) for _ in range(4)]
    got = upscaler_torch.torch_gradient_aware_upscale(*[p.cuda() for p in planes], nh, nw)
    exp = O.upscale_fwd(*[p.numpy() for p in planes], nh, nw, mode=1, dtype=np.float64)
    assert np.abs(np_(got) - exp).max() <= 1e-12
    gout = torch.randn(nh, nw, 3, generator=g, dtype=torch.float64)
    x = [p.cuda().requires_grad_() for p in planes]
    upscaler_torch.torch_gradient_aware_upscale(*x, nh, nw).backward(gout.cuda())
    eg = O.upscale_bwd(gout.numpy(), h, w, mode=1, dtype=np.float64)
    for a, b in zip(x, eg):
        assert rel_err(np_(a.grad), b) <= 1e-12


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_single_channel_upscaler_is_one_channel_of_the_rgb_form(dtype):
    """torch_gradient_aware_upscale_single_channel runs the one-channel
    kernel: value and gradients equal channel k of the 3-channel upscale of
    planes whose channel k holds the single-channel input (half-pixel ROI
    path through ops too)."""
    h, w, nh, nw = 37, 45, 90, 131
    g = torch.Generator().manual_seed(18)
    planes = [torch.randn(h, w, generator=g, dtype=dtype).cuda() for _ in range(4)]
    gout = torch.randn(nh, nw, generator=g, dtype=dtype).cuda()
    x1 = [p.clone().requires_grad_() for p in planes]
    y1 = upscaler_torch.torch_gradient_aware_upscale_single_channel(*x1, nh, nw)
    y1.backward(gout)
    rgb = [torch.stack([torch.zeros_like(p), p, torch.zeros_like(p)], -1) for p in planes]
    x3 = [p.clone().requires_grad_() for p in rgb]
    y3 = upscaler_torch.torch_gradient_aware_upscale(*x3, nh, nw)
    y3.backward(torch.stack([torch.zeros_like(gout), gout, torch.zeros_like(gout)], -1))
    assert y1.shape == (nh, nw) and torch.equal(y1, y3[..., 1])
    for a, b in zip(x1, x3):
        assert torch.equal(a.grad, b.grad[..., 1])
    roi = (3.0, 2.5, 40.0, 30.0)
    o1 = ops.upscale_fwd(*[p.unsqueeze(-1) for p in planes], nh, nw, roi=roi, mode=0)
    o3 = ops.upscale_fwd(*rgb, nh, nw, roi=roi, mode=0)
    assert torch.equal(o1[..., 0], o3[..., 1])


@pytest.mark.parametrize("H,W,B,n", [(150, 170, 16, 3000),
                                     # >= 4096 tiles: 0.017 Gaussians per pixel, 8x16 regions
                                     (1040, 1100, 16, 20000),
                                     # >= 4096 tiles: 0.052 Gaussians per pixel, 8x8 regions
                                     (1040, 1100, 16, 60000),
                                     (97, 203, 12, 2500)])
def test_dropin_backward_image_loss_matches_reference(H, W, B, n):
    """The drop-in backward for an image-only loss without opacities (LIG's
    own training loop, gaussianlig.py:70-111) runs the lean walk with the
    per-pixel |v_xy| sums: v_xy, xys.absgrad, v_conic and v_rgb against the
    reference kernel fed the same cotangent (1e-4 relative)."""
    means, L, colors, _ = scene(n, H, W, diag=(0.5, 5.0), seed=19)
    g = torch.Generator().manual_seed(20)
    w = torch.randn(H, W, 3, generator=g).cuda()
    xys, ext, con, cnt = gsplat2d.project_gaussians_cholesky(L, means, H, W, B)
    xys = xys.detach().requires_grad_()
    con = con.detach().requires_grad_()
    col = colors.clone().requires_grad_()
    img = gsplat2d.rasterize_gaussians(xys, ext, con, cnt, col, None, H, W, B)[0]
    (img * w).sum().backward()
    rb = ref.bin_and_sort(xys.detach(), ext, cnt, H, W, B)
    rf = ref.raster_fwd(H, W, B, rb, xys.detach(), con.detach(), colors, None)
    gr = ref.raster_bwd(H, W, B, rb, xys.detach(), con.detach(), colors, None,
                        rf["final_idx"], w, torch.zeros(H, W, device="cuda"))
    assert rel_err(np_(xys.grad), np_(gr["v_xy"])) <= 1e-4
    assert rel_err(np_(xys.absgrad), np_(gr["v_xy_abs"])) <= 1e-4
    assert rel_err(np_(con.grad), np_(gr["v_conic"])) <= 1e-4
    assert rel_err(np_(col.grad), np_(gr["v_rgb"])) <= 1e-4


def test_no_device_wait_gave_up():
    """No bounded device-side wait (bulk-staged backward) has timed out in
    this process (the counter stays 0 in normal operation)."""
    from lig_b200 import _lib
    H, W, B, n = 150, 170, 16, 3000
    means, L, colors, _ = scene(n, H, W, diag=(0.5, 5.0), seed=21)
    target = torch.rand(H, W, 3, generator=torch.Generator().manual_seed(22)).cuda()
    from lig_b200.fused import render_l2_loss
    p = [t.clone().requires_grad_() for t in (means, L, colors)]
    render_l2_loss(p[1], p[0], p[2], None, target, H, W, B).backward()
    torch.cuda.synchronize()
    assert _lib.lib.lig_wait_timeouts() == 0


def test_lig_training_step_decreases_loss():
    H, W, B, n = 96, 96, 16, 2000
    means, L, colors, _ = scene(n, H, W, diag=(0.5, 3.0), seed=2)
    gt_means, gt_L, gt_col, _ = scene(1500, H, W, diag=(0.5, 3.0), seed=0)
    with torch.no_grad():
        x, e, c, k = gsplat2d.project_gaussians_cholesky(gt_L, gt_means, H, W, B)
        gt = torch.clamp(gsplat2d.rasterize_gaussians(x, e, c, k, gt_col, None, H, W, B)[0], 0, 1)
    params = [means.requires_grad_(), L.requires_grad_(), colors.requires_grad_()]
    opt = torch.optim.Adam(params, lr=1e-2)
    losses = []
    for _ in range(30):
        x, e, c, k = gsplat2d.project_gaussians_cholesky(params[1], params[0], H, W, B)
        img = torch.clamp(gsplat2d.rasterize_gaussians(x, e, c, k, params[2], None, H, W, B)[0],
                          0, 1)
        loss = torch.nn.functional.mse_loss(img, gt)
        opt.zero_grad()
        loss.backward()
        opt.step()
        losses.append(loss.item())
    assert losses[-1] < 0.7 * losses[0]


@pytest.mark.parametrize("H,W,B,n", [(150, 170, 16, 3000),
                                     # >= 4096 tiles: the 8x16 and the 8x8 backward walks
                                     (1040, 1100, 16, 20000),
                                     (1040, 1100, 16, 60000)])
def test_fused_render_l2_matches_unfused_chain(H, W, B, n):
    """lig_b200.fused.render_l2_loss == project + rasterize + clamp + mse_loss,
    value and gradients (the fused backward forms dL/dimg in-kernel)."""
    from lig_b200.fused import render_l2_loss
    means, L, colors, _ = scene(n, H, W, diag=(0.5, 5.0), seed=4)
    g = torch.Generator().manual_seed(9)
    target = torch.rand(H, W, 3, generator=g).cuda()

    def unfused(p):
        xys, ext, con, cnt = gsplat2d.project_gaussians_cholesky(p[1], p[0], H, W, B)
        img = gsplat2d.rasterize_gaussians(xys, ext, con, cnt, p[2], None, H, W, B)[0]
        return torch.nn.functional.mse_loss(torch.clamp(img, 0, 1), target)

    p1 = [t.clone().requires_grad_() for t in (means, L, colors)]
    p2 = [t.clone().requires_grad_() for t in (means, L, colors)]
    l1 = unfused(p1)
    l1.backward()
    l2 = render_l2_loss(p2[1], p2[0], p2[2], None, target, H, W, B)
    l2.backward()
    assert abs(l1.item() - l2.item()) <= 1e-6 * abs(l1.item())
    for a, b in zip(p2, p1):
        assert rel_err(np_(a.grad), np_(b.grad)) <= 1e-5


def test_fused_l2_forward_nonfinite_colours():
    """Gaussians with infinite or NaN colours: the fused forward's masked
    difference and final indices equal the plain forward's exactly (the
    packed four-pixel loop hands such Gaussians to its scalar path)."""
    H, W, B, n = 1040, 1100, 16, 20000
    means, L, colors, _ = scene(n, H, W, diag=(0.5, 5.0), seed=16)
    bad = torch.arange(0, n, n // 24, device="cuda")[:24]
    vals = torch.tensor([float("inf"), -float("inf"), float("nan")], device="cuda")
    colors = colors.clone()
    colors[bad, torch.arange(24, device="cuda") % 3] = vals[torch.arange(24, device="cuda") % 3]
    g = torch.Generator().manual_seed(17)
    target = torch.rand(H, W, 3, generator=g).cuda()
    xys, ext, con, cnt = ops.project_fwd(L, means, None, H, W, B, True)
    b = ops.bin_gaussians(xys, ext, cnt, H, W, B)
    img, _, _, _, _, fin = ops.raster_fwd(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total,
                                          xys, con, colors, None, False)
    diff, fin2, _ = ops.raster_fwd_l2(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total,
                                      xys, con, colors, None, target)
    assert not torch.isfinite(img).all()
    exp = torch.where((img >= 0) & (img <= 1), torch.clamp(img, 0, 1) - target,
                      torch.zeros_like(img))
    assert torch.equal(diff, exp) and torch.equal(fin2, fin)


@pytest.mark.parametrize("H,W,B,n", [(150, 170, 16, 3000),
                                     (1040, 1100, 16, 20000),  # >= 4096 tiles: four pixels per lane
                                     (600, 560, 8, 8000),      # >= 4096 tiles, 8x8 tiles
                                     (2048, 2080, 32, 60000),  # >= 4096 tiles, 32x32 tiles
                                     (97, 203, 12, 2500),
                                     (130, 90, 32, 2000)])
def test_fused_l2_forward_diff_and_loss(H, W, B, n):
    """lig_raster_fwd_l2: diff = mask * (clamp(x) - t) bit-exact against the
    plain forward's image, loss against the separate loss kernel (different
    summation order: 1e-6 relative), final_idx identical; and the backward
    from diff equals the backward from (image, target)."""
    means, L, colors, _ = scene(n, H, W, diag=(0.5, 5.0), seed=6)
    g = torch.Generator().manual_seed(10)
    target = torch.rand(H, W, 3, generator=g).cuda()
    xys, ext, con, cnt = ops.project_fwd(L, means, None, H, W, B, True)
    b = ops.bin_gaussians(xys, ext, cnt, H, W, B)
    img, _, _, _, _, fin = ops.raster_fwd(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total,
                                          xys, con, colors, None, False)
    diff, fin2, loss = ops.raster_fwd_l2(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total,
                                         xys, con, colors, None, target)
    exp = torch.where((img >= 0) & (img <= 1), torch.clamp(img, 0, 1) - target,
                      torch.zeros_like(img))
    assert torch.equal(diff, exp) and torch.equal(fin2, fin)
    ref_loss = ops.l2_clamped_loss(img, target)
    assert abs(loss.item() - ref_loss.item()) <= 1e-6 * ref_loss.item()
    one = torch.ones((), device="cuda")
    ga = ops.raster_bwd_l2(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total, xys, con,
                           colors, None, fin, img, target, one)
    gb = ops.raster_bwd_diff(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total, xys, con,
                             colors, None, fin2, diff, one)
    for x, y in zip(ga[:4], gb[:4]):
        assert rel_err(np_(x), np_(y)) <= 1e-5
    # without opacities these fused backwards skip |v_xy| and the opacity
    # gradient; the rest equals the general backward fed the same cotangent
    assert torch.all(gb[1] == 0)
    v_img = diff * (2.0 / (3 * H * W))
    full = ops.raster_bwd(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total, xys, con, colors,
                          None, fin, v_img, None, None, None, None)
    for i in (0, 2, 3):
        assert rel_err(np_(gb[i]), np_(full[i])) <= 1e-5


@pytest.mark.parametrize("H,W,B,n", [(150, 170, 16, 3000),
                                     (1040, 1100, 16, 20000)])  # >= 4096 tiles
def test_fused_l2_without_final_indices(H, W, B, n):
    """final_idx = NULL (the fit loop without opacities): the fused forward
    gives the same masked difference and loss bit for bit without tracking or
    writing the per-pixel last index, and the backward from the difference,
    which then reads no final indices, gives the same gradients."""
    means, L, colors, _ = scene(n, H, W, diag=(0.5, 5.0), seed=41)
    g = torch.Generator().manual_seed(42)
    target = torch.rand(H, W, 3, generator=g).cuda()
    xys, ext, con, cnt = ops.project_fwd(L, means, None, H, W, B, True)
    b = ops.bin_gaussians(xys, ext, cnt, H, W, B)
    args = (H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total, xys, con, colors, None)
    diff, fin, loss = ops.raster_fwd_l2(*args, target)
    diff0, fin0, loss0 = ops.raster_fwd_l2(*args, target, want_final_idx=False)
    assert fin0 is None and fin is not None
    assert torch.equal(diff0, diff) and torch.equal(loss0, loss)
    one = torch.ones((), device="cuda")
    ga = ops.raster_bwd_diff(*args, fin, diff, one)
    gb = ops.raster_bwd_diff(*args, None, diff0, one)
    for x, y in zip(ga[:4], gb[:4]):   # float atomics: the order of additions differs
        assert rel_err(np_(x), np_(y)) <= 1e-5


@pytest.mark.parametrize("seed,diag,offdiag", [(21, (0.3, 8.0), 4.0),    # thin, tilted
                                              (22, (0.2, 1.0), 0.05),   # small, axis-aligned
                                              (23, (2.0, 20.0), 8.0)])  # large, tilted
def test_fused_l2_forward_row_blocks_exact(seed, diag, offdiag):
    """The fused forward with four pixels per lane (>= 4096 tiles) evaluates
    only the 4-row blocks of its 8x16 region that a Gaussian can reach; on
    thin, small and large tilted Gaussians the masked difference and the
    final indices stay equal to the plain forward's, bit for bit."""
    H, W, B, n = 1024, 1040, 16, 12000
    means, L, colors, _ = scene(n, H, W, diag=diag, seed=seed, offdiag_std=offdiag)
    g = torch.Generator().manual_seed(seed)
    target = torch.rand(H, W, 3, generator=g).cuda()
    xys, ext, con, cnt = ops.project_fwd(L, means, None, H, W, B, True)
    b = ops.bin_gaussians(xys, ext, cnt, H, W, B)
    img, _, _, _, _, fin = ops.raster_fwd(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total,
                                          xys, con, colors, None, False)
    diff, fin2, _ = ops.raster_fwd_l2(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total,
                                      xys, con, colors, None, target)
    exp = torch.where((img >= 0) & (img <= 1), torch.clamp(img, 0, 1) - target,
                      torch.zeros_like(img))
    assert torch.equal(diff, exp) and torch.equal(fin2, fin)


@pytest.mark.parametrize("H,W,B,n,dtype", [(150, 170, 16, 3000, torch.float32),
                                           (1024, 1040, 16, 12000, torch.float32),
                                           (97, 130, 12, 1500, torch.float64)])
def test_fused_l2_forward_uint8_target(H, W, B, n, dtype):
    """lig_raster_fwd_l2_u8: an 8-bit target gives the masked difference,
    final indices and loss of the float target byte / 255 (ToTensor's
    division on the host), bit for bit, in float and double."""
    means, L, colors, _ = scene(n, H, W, diag=(0.5, 5.0), seed=8, dtype=dtype)
    g = torch.Generator().manual_seed(18)
    u8 = torch.randint(0, 256, (H, W, 3), generator=g, dtype=torch.uint8)
    tf = (u8.to(dtype) / 255).cuda()
    xys, ext, con, cnt = ops.project_fwd(L, means, None, H, W, B, True)
    b = ops.bin_gaussians(xys, ext, cnt, H, W, B)
    args = (H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total, xys, con, colors, None)
    d1, f1, l1 = ops.raster_fwd_l2(*args, u8.cuda())
    d2, f2, l2 = ops.raster_fwd_l2(*args, tf)
    assert d1.dtype == dtype
    assert torch.equal(d1, d2) and torch.equal(f1, f2) and torch.equal(l1, l2)


def test_binning_grows_sort_shared_memory_between_calls():
    """A process whose first binning needs 9-bit radix digits and whose next
    one needs 10-bit digits (more shared memory in the downsweep) must opt
    the kernel into the larger size (fresh process: the opt-in is cached)."""
    import subprocess
    import sys
    code = r"""
import torch
from lig_b200 import ops
from tests._scene import scene
for (H, W, B) in ((4096, 8192, 16), (8192, 8192, 8)):
    means, L, colors, _ = scene(2000, H, W, diag=(0.5, 3.0), seed=3)
    xys, ext, con, cnt = ops.project_fwd(L, means, None, H, W, B, True)
    b = ops.bin_gaussians(xys, ext, cnt, H, W, B)
    torch.cuda.synchronize()
    assert b.num_intersects == int(cnt.sum())
print("ok")
"""
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-2000:]


def test_alpha_cut_is_the_step_of_the_alpha_test():
    """Over every non-negative float sigma (bit patterns up to +inf) the
    rasterizers' alpha >= 1/255 decision is one step in sigma's bit pattern,
    and the warp search the pack kernel runs finds its edge:
    out = [search cut, first failing pattern, last passing pattern]."""
    from lig_b200 import _lib
    out = torch.zeros(3, dtype=torch.int32, device="cuda")
    assert _lib.lib.lig_alpha_cut(ops._p(out), ops._stream(out.device)) == _lib.LIG_OK
    o = out.cpu().numpy().view(np.uint32)
    assert o[0] == o[1] and o[2] + 1 == o[1], o
    cut = float(o[:1].view(np.float32)[0])
    assert 5.5 < cut < 5.6 and abs(cut - np.log(255.0)) < 1e-5


@pytest.mark.parametrize("H,W,B,n", [(150, 170, 16, 3000),
                                     (1040, 1100, 16, 20000)])  # four pixels per lane
def test_alpha_cut_paths_with_degenerate_gaussians(H, W, B, n):
    """In the fused forward, chunks that hold a Gaussian without culling data
    take the float alpha test, the rest the cut's compare.  Mixed in:
    non-positive-definite
    conics; negative-definite ones centred exactly on a pixel centre (sigma
    is -0 there: the reference passes it with alpha = clamp); conics whose
    entries times the squared cull reach come near the float range (no
    culling data by that guard); NaN conics (sigma is NaN: the reference
    passes it with alpha = clamp).  The
    fused forward's masked difference and final indices equal the plain
    forward's bit for bit, and the lean backward's colour gradients (an
    all-positive cotangent, so one flipped alpha decision would move a
    Gaussian's sum by at least 0.5 / 255) equal the general backward's per
    Gaussian."""
    means, L, colors, _ = scene(n, H, W, diag=(0.5, 5.0), seed=31)
    xys, ext, con, cnt = ops.project_fwd(L, means, None, H, W, B, True)
    xys, con = xys.clone(), con.clone()
    idx = torch.arange(7, n, 53, device="cuda")
    kind = torch.arange(idx.numel(), device="cuda") % 4
    bad = {0: [1.0, 2.0, 1.0], 1: [-0.3, -0.1, -0.5], 2: [1e35, -0.99e35, 1e35],
           3: [float("nan"), 0.0, 1.0]}
    for k, v in bad.items():
        sel = idx[kind == k]
        con[sel] = torch.tensor(v, device="cuda")
        if k == 1:
            xys[sel] = torch.floor(xys[sel]) + 0.5
    g = torch.Generator().manual_seed(32)
    target = torch.rand(H, W, 3, generator=g).cuda()
    b = ops.bin_gaussians(xys, ext, cnt, H, W, B)
    img, _, _, _, _, fin = ops.raster_fwd(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total,
                                          xys, con, colors, None, False)
    diff, fin2, _ = ops.raster_fwd_l2(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total,
                                      xys, con, colors, None, target)
    assert torch.isfinite(img).all()
    exp = torch.where((img >= 0) & (img <= 1), torch.clamp(img, 0, 1) - target,
                      torch.zeros_like(img))
    assert torch.equal(diff, exp) and torch.equal(fin2, fin)
    v = 0.5 + 0.5 * torch.rand(H, W, 3, generator=g).cuda()
    lean = ops.raster_bwd(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total, xys, con,
                          colors, None, fin, v, None)
    full = ops.raster_bwd(H, W, B, b.gaussian_ids_sorted, b.tile_bins, b.total, xys, con,
                          colors, None, fin, v, torch.zeros(H, W, device="cuda"))
    a, r = np_(lean[3]).astype(np.float64), np_(full[3]).astype(np.float64)
    assert np.isfinite(r).all()
    assert (np.abs(a - r) <= 1e-6 * np.abs(r) + 1e-5).all()
    assert (r[np_(idx)].sum(1) > 0).any()   # the planted Gaussians were rendered
