"""FP64 instantiation of the same kernels against the FP64 CPU oracle, and the
autograd chain (project -> gradient-aware raster -> upscale) against FP64
central finite differences (h = 1e-6)."""
import numpy as np
import pytest
import torch

import lig_b200
from lig_b200 import ops
from lig_b200.gsplat2d import gradient_aware_upscale, project_gaussians_cholesky, rasterize_gaussians
from oracle import oracle as O
from tests._scene import np_, rel_err, scene

pytestmark = pytest.mark.gpu

F64 = torch.float64


@pytest.mark.parametrize("n,H,W,B,opac", [(400, 96, 112, 16, None), (300, 70, 61, 8, (0.1, 0.99)),
                                          (250, 50, 50, 12, (0.0, 1.0))])
@pytest.mark.parametrize("ga", [False, True])
def test_fp64_forward_vs_dense_oracle(n, H, W, B, opac, ga):
    means, L, colors, op = scene(n, H, W, diag=(0.5, 4.0), opac=opac, dtype=F64)
    xys, ext, con, cnt = ops.project_fwd(L, means, op, H, W, B, True)
    o_xys, o_ext, o_con, o_cnt = O.project_fwd(np_(L), np_(means), np_(op), H, W, B, chol=True,
                                               dtype=np.float64)
    assert np.array_equal(np_(cnt), o_cnt)
    assert np.array_equal(np_(ext), o_ext)
    assert rel_err(np_(con), o_con) <= 1e-13
    mb = ops.bin_gaussians(xys, ext, cnt, H, W, B)
    img, wsum, dx, dy, dxy, fin = ops.raster_fwd(H, W, B, mb.gaussian_ids_sorted, mb.tile_bins,
                                                 mb.total, xys, con, colors, op, ga)
    d = O.dense_fwd_f64(H, W, B, o_xys, o_ext, o_cnt, o_con, np_(colors), np_(op), grad_aware=ga)
    assert np.abs(np_(img) - d["img"]).max() <= 1e-9
    assert np.abs(np_(wsum) - d["wsum"]).max() <= 1e-9
    if ga:
        for a, k in zip((dx, dy, dxy), ("dx", "dy", "dxy")):
            assert np.abs(np_(a) - d[k]).max() <= 1e-9, k


@pytest.mark.parametrize("ga", [False, True])
def test_fp64_backward_vs_oracle(ga):
    n, H, W, B = 300, 80, 72, 16
    means, L, colors, op = scene(n, H, W, diag=(0.5, 4.0), opac=(0.1, 0.95), dtype=F64)
    xys, ext, con, cnt = ops.project_fwd(L, means, op, H, W, B, True)
    mb = ops.bin_gaussians(xys, ext, cnt, H, W, B)
    img, wsum, dx, dy, dxy, fin = ops.raster_fwd(H, W, B, mb.gaussian_ids_sorted, mb.tile_bins,
                                                 mb.total, xys, con, colors, op, ga)
    g = torch.Generator().manual_seed(3)
    cot = [torch.randn(s, generator=g, dtype=F64).cuda()
           for s in [(H, W, 3), (H, W), (H, W, 3), (H, W, 3), (H, W, 3)]]
    vd = cot[2:] if ga else [None] * 3
    got = ops.raster_bwd(H, W, B, mb.gaussian_ids_sorted, mb.tile_bins, mb.total, xys, con,
                         colors, op, fin, cot[0], cot[1], *vd)
    bn = O.bin_and_sort(np_(xys), np_(ext), np_(cnt), H, W, B, dtype=np.float64)
    exp = O.raster_bwd(H, W, B, bn, np_(xys), np_(con), np_(colors), np_(op), np_(fin),
                       np_(cot[0]), np_(cot[1]), *[np_(v) for v in vd], dtype=np.float64)
    for a, k in zip(got, ["v_xy", "v_xy_abs", "v_conic", "v_rgb", "v_opacity"]):
        assert rel_err(np_(a), exp[k]) <= 1e-10, k


def _loss_fn(H, W, B, up, w_out):
    def f(means, chol, colors, op):
        xys, ext, con, cnt = project_gaussians_cholesky(chol, means, H, W, B, op)
        img, wsum, dx, dy, dxy = rasterize_gaussians(xys, ext, con, cnt, colors, op, H, W, B,
                                                     compute_upscale_gradients=True)
        out = gradient_aware_upscale(img, dx, dy, dxy, up * H, up * W)
        return (out * w_out).sum()
    return f


def test_autograd_vs_finite_differences():
    """Config 3, part 1: 128x128, 500 Gaussians, opacities 0.9 (the 0.999 clamp
    never fires), 2x gradient-aware upscale.  Parameters whose +-h evaluations
    cross a culling threshold are excluded (FD at h and 2h disagree)."""
    H = W = 128
    B, n, up = 16, 500, 2
    means, L, colors, _ = scene(n, H, W, diag=(0.8, 5.0), dtype=F64)
    op = torch.full((n,), 0.9, dtype=F64, device="cuda")
    g = torch.Generator().manual_seed(3)
    w_out = torch.randn(up * H, up * W, 3, generator=g, dtype=F64).cuda()
    f = _loss_fn(H, W, B, up, w_out)
    params = [means.clone().requires_grad_(), L.clone().requires_grad_(),
              colors.clone().requires_grad_()]
    loss = f(*params, op)
    grads = torch.autograd.grad(loss, params)
    rng = np.random.default_rng(0)
    h = 1e-6
    checked = 0
    with torch.no_grad():
        for pi, name in enumerate(["means", "cholesky", "colors"]):
            base = [p.detach().clone() for p in params]
            for _ in range(25):
                idx = tuple(int(rng.integers(0, s)) for s in base[pi].shape)

                def at(delta):
                    args = [b.clone() for b in base]
                    args[pi][idx] += delta
                    return f(*args, op).item()

                fd1 = (at(h) - at(-h)) / (2 * h)
                fd2 = (at(2 * h) - at(-2 * h)) / (4 * h)
                if abs(fd1 - fd2) > 1e-4 * (abs(fd1) + 1e-3):
                    continue  # culling threshold crossed inside the stencil
                an = grads[pi][idx].item()
                assert abs(an - fd1) <= 1e-5 * (abs(fd1) + 1e-2), (name, idx, an, fd1)
                checked += 1
    assert checked >= 60
