"""The LIG level fit and two-level pipeline driven by the reference's kernels
(the checker side of the PSNR-parity tests and of tests/perf_vs_reference.py).

Same seeded init, target, Adam settings and level hand-over as
lig_b200/fit.py; every kernel is the reference's (oracle/_ref, compiled from
the reference sources), with its torch glue restated in oracle/ref.py —
cumsum + .item(), torch.sort + gather — and the clamp/L2 gradient computed as
autograd would for clamp(render, 0, 1) + F.mse_loss (gaussianlig.py:95-101).
"""
import torch

from lig_b200 import synthetic
from lig_b200.fit import downsample, psnr
from oracle import ref


class RefFit:
    """One level: n Cholesky-parameterised Gaussians fitted with Adam."""

    def __init__(self, n, H, W, diag, lr=1e-3, B=16, seed=synthetic.SEED_INIT,
                 rgb_init="uniform"):
        means, chol, colors = synthetic.gaussians(n, H, W, diag=diag, seed=seed)
        if rgb_init == "zeros":
            colors = torch.zeros_like(colors)
        self.means = means.cuda().requires_grad_()
        self.chol = chol.cuda().requires_grad_()
        self.rgbs = colors.cuda().requires_grad_()
        self.H, self.W, self.B = H, W, B
        self.opt = torch.optim.Adam([self.rgbs, self.means, self.chol], lr=lr, fused=True)

    def render(self, grad_aware=False):
        with torch.no_grad():
            return ref.render(self.chol, self.means, self.rgbs, None, self.H, self.W, self.B,
                              True, grad_aware)

    def step(self, target):
        H, W, B = self.H, self.W, self.B
        with torch.no_grad():
            r = ref.render(self.chol, self.means, self.rgbs, None, H, W, B)
            img = r["img"]
            c = torch.clamp(img, 0, 1)
            diff = c - target
            loss = (diff * diff).mean()
            v_img = (2.0 / img.numel()) * diff * ((img >= 0) & (img <= 1))
            v_w = torch.zeros(H, W, device=img.device)
            g = ref.raster_bwd(H, W, B, r["binning"], r["xys"], r["conics"], self.rgbs, None,
                               r["final_idx"], v_img, v_w)
            v_chol, v_mean = ref.project_bwd(r["extents"], self.chol, r["conics"], g["v_xy"],
                                             g["v_conic"], chol=True)
        self.means.grad, self.chol.grad, self.rgbs.grad = v_mean, v_chol, g["v_rgb"]
        self.opt.step()
        self.opt.zero_grad(set_to_none=True)
        return loss


def iters_per_s(fit, target, iters):
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(iters):
        fit.step(target)
    e.record()
    torch.cuda.synchronize()
    return iters / (s.elapsed_time(e) / 1e3)


def ref_two_level(gt, n1, n2, iters, lr=1e-3, factor=4, diag=(0.5, 6.0), rgb_init="uniform"):
    """lig_b200.fit.fit_two_level with every kernel replaced by the
    reference's: level fits, the gradient-aware render and upscale."""
    H, W, _ = gt.shape
    t1 = downsample(gt, factor)
    h1, w1 = t1.shape[:2]
    lvl1 = RefFit(n1, h1, w1, diag, lr=lr, rgb_init=rgb_init)
    ips1 = iters_per_s(lvl1, t1, iters)
    with torch.no_grad():
        r = lvl1.render(grad_aware=True)
        p1 = psnr(torch.clamp(r["img"], 0, 1), t1)
        up = torch.clamp(ref.upscale_fwd(r["img"], r["dx"], r["dy"], r["dxy"], H, W), 0, 1)
        pu = psnr(up, gt)
        resid = gt - up + 0.5
        lo, hi = resid.min(), resid.max()
        t2 = ((resid - lo) / (hi - lo)).contiguous()
    del lvl1
    lvl2 = RefFit(n2, H, W, diag, lr=lr, seed=synthetic.SEED_INIT + 1, rgb_init=rgb_init)
    ips2 = iters_per_s(lvl2, t2, iters)
    with torch.no_grad():
        r2 = torch.clamp(lvl2.render()["img"], 0, 1)
        p2 = psnr(r2, t2)
        out = torch.clamp(r2 * (hi - lo) + up - 0.5 + lo, 0, 1)
        pf = psnr(out, gt)
    return {"psnr": pf, "level_psnr": [p1, p2], "up_psnr": pu, "iters_per_s": [ips1, ips2]}
