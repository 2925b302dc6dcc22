"""LIG fitting on the lig_b200 kernels: one level (a Gaussian2D fit) and the
two-level pipeline of train.py:93-158.

A level fits Cholesky-parameterised Gaussians (means, [l11, l21, l22], rgb) to
an HWC target with L2 on the clamped render and Adam, the loop of
gaussianlig.Gaussian2D.train_iter (gaussianlig.py:99-111) with the
parameterisation of the fit configurations.  The iteration runs either as a
captured CUDA graph of the library's fused entry points (LevelFit's default
engine, through lig_b200.batch) or through the drop-in gsplat2d API under
autograd; renders between levels use the drop-in API
(project_gaussians_cholesky + rasterize_gaussians + gradient_aware_upscale).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import torch
import torch.nn.functional as F

from . import synthetic
from .fused import render_l2_loss
from .gsplat2d import gradient_aware_upscale, project_gaussians_cholesky, rasterize_gaussians


class LevelFit:
    """One LIG level: N Gaussians fitted to an [H, W, 3] target — fp32, or
    uint8 (an RGB image as stored, read as byte / 255 the way torchvision's
    ToTensor converts it in train.py; the graph engine reads the bytes in the
    loss kernel, so uploading a new target each step moves a quarter of the
    bytes).

    rgb_init "uniform" draws colours U(0,1) (the fit configurations);
    "zeros" starts them at zero as gaussianlig.py:57 does.

    engine "graph" (default): the iteration runs as a one-image BatchedFit —
    fused-loss forward, backward from the masked difference, projection
    backward and the flat guarded Adam, captured as a CUDA graph (one per
    target buffer), no autograd and no per-step host work.  engine
    "autograd": the drop-in gsplat2d API under torch autograd with
    torch.optim.Adam (fused_loss selects the fused render + L2 node or the
    plain clamp + F.mse_loss chain)."""

    def __init__(self, n: int, H: int, W: int, device="cuda", lr: float = 1e-3, block: int = 16,
                 diag=(0.5, 6.0), seed: int = synthetic.SEED_INIT, fused_adam: bool = True,
                 fused_loss: bool = True, engine: str = "graph", rgb_init: str = "uniform"):
        if engine not in ("graph", "autograd"):
            raise ValueError("engine must be 'graph' or 'autograd'")
        if rgb_init not in ("uniform", "zeros"):
            raise ValueError("rgb_init must be 'uniform' or 'zeros'")
        self.H, self.W, self.block, self.lr = H, W, block, lr
        self.fused_loss = fused_loss
        self.engine = engine if fused_loss else "autograd"
        means, chol, colors = synthetic.gaussians(n, H, W, diag=diag, seed=seed)
        if rgb_init == "zeros":  # gaussianlig.py:57 initialises colours to zero
            colors = torch.zeros_like(colors)
        self.means = torch.nn.Parameter(means.to(device))
        self.chol = torch.nn.Parameter(chol.to(device))
        self.rgbs = torch.nn.Parameter(colors.to(device))
        self.params = [self.rgbs, self.means, self.chol]
        kw = {"fused": True} if fused_adam and torch.device(device).type == "cuda" else {}
        self.opt = torch.optim.Adam(self.params, lr=lr, **kw)
        self._batch = None

    @property
    def n(self) -> int:
        return self.means.shape[0]

    def render(self, grad_aware: bool = False):
        xys, ext, con, cnt = project_gaussians_cholesky(self.chol, self.means, self.H, self.W,
                                                        self.block)
        return rasterize_gaussians(xys, ext, con, cnt, self.rgbs, None, self.H, self.W,
                                   self.block, compute_upscale_gradients=grad_aware)

    def _graph_step(self, target_hwc: torch.Tensor) -> torch.Tensor:
        if self._batch is None:
            from .batch import BatchedFit
            with torch.no_grad():
                init = [(self.means.detach(), self.chol.detach(), self.rgbs.detach())]
            self._batch = BatchedFit([target_hwc], [self.n], block=self.block, lr=self.lr,
                                     init=init, graph=True)
            b = self._batch
            # the parameters now live in the batch's flat buffer
            self.means, self.chol, self.rgbs = b.means, b.chol, b.rgbs
            self.params = [self.rgbs, self.means, self.chol]
        self._batch.step_checked(target_hwc)
        return self._batch.loss

    def step(self, target_hwc: torch.Tensor) -> torch.Tensor:
        """One iteration: render, clamp, L2, backward, Adam.  Returns the loss
        as a device tensor (no host synchronisation; with the graph engine a
        buffer that the next step overwrites)."""
        if self.engine == "graph":
            return self._graph_step(target_hwc.contiguous())
        if target_hwc.dtype == torch.uint8:  # an 8-bit image, read as ToTensor does
            target_hwc = target_hwc.float() / 255
        if self.fused_loss:
            loss = render_l2_loss(self.chol, self.means, self.rgbs, None, target_hwc, self.H,
                                  self.W, self.block)
        else:
            img = torch.clamp(self.render()[0], 0, 1)
            loss = F.mse_loss(img, target_hwc)
        self.opt.zero_grad(set_to_none=True)
        loss.backward()
        self.opt.step()
        return loss.detach()


def psnr(a: torch.Tensor, b: torch.Tensor) -> float:
    mse = F.mse_loss(a.float(), b.float()).item()
    return 10 * math.log10(1.0 / max(mse, 1e-20))


def make_target(H: int, W: int, n_teacher: int, diag, noise: str = "white", noise_std=0.02,
                device="cuda", block: int = 16) -> torch.Tensor:
    """Teacher render (seed 0) + noise (seed 1), clipped to [0, 1]; [H, W, 3]."""
    means, chol, colors = synthetic.gaussians(n_teacher, H, W, diag=diag,
                                              seed=synthetic.SEED_TEACHER)
    with torch.no_grad():
        xys, ext, con, cnt = project_gaussians_cholesky(chol.to(device), means.to(device), H, W,
                                                        block)
        img = rasterize_gaussians(xys, ext, con, cnt, colors.to(device), None, H, W, block)[0]
        if noise == "white":
            img = img + synthetic.white_noise(H, W, noise_std).to(device)
        else:
            img = img + synthetic.spectral_noise(H, W, noise_std, device=device)
    return torch.clamp(img, 0, 1).contiguous()


def downsample(gt_hwc: torch.Tensor, factor: int) -> torch.Tensor:
    """Bicubic antialiased downsample (the level-1 target of the two-level fit)."""
    x = gt_hwc.permute(2, 0, 1).unsqueeze(0)
    y = F.interpolate(x, scale_factor=1.0 / factor, mode="bicubic", align_corners=False,
                      antialias=True)
    return y.squeeze(0).permute(1, 2, 0).contiguous()


@dataclass
class TwoLevelResult:
    psnr: float
    level_psnr: list = field(default_factory=list)
    up_psnr: float = 0.0        # upscaled level-1 render alone vs the full-resolution target
    iters_per_s: list = field(default_factory=list)
    store_min: float = 0.0
    store_max: float = 0.0


def fit_two_level(gt_hwc: torch.Tensor, n1: int, n2: int, iters: int, lr: float = 1e-3,
                  factor: int = 4, diag=(0.5, 6.0), block: int = 16,
                  log_every: Optional[int] = None, rgb_init: str = "uniform") -> TwoLevelResult:
    """The LIG level pipeline (train.py:93-158) with the gradient-aware upscale
    between levels: level 1 fits the factor-x downsampled image, its render is
    upscaled with gradient_aware_upscale and clamped to [0, 1] (the level
    estimate of train.py is a clamped render), level 2 fits the min-max
    normalised residual gt - up + 0.5, and the reconstruction is
    level2 * (max - min) + up - 0.5 + min (train.py:154)."""
    H, W, _ = gt_hwc.shape
    dev = gt_hwc.device
    res = TwoLevelResult(psnr=0.0)
    t1 = downsample(gt_hwc, factor)
    h1, w1 = t1.shape[:2]
    lvl1 = LevelFit(n1, h1, w1, dev, lr=lr, block=block, diag=diag, rgb_init=rgb_init)
    res.iters_per_s.append(_run(lvl1, t1, iters, log_every))
    with torch.no_grad():
        img, _, dx, dy, dxy = lvl1.render(grad_aware=True)
        res.level_psnr.append(psnr(torch.clamp(img, 0, 1), t1))
        # the level-1 estimate lies in [0, 1] as train.py's im_estim does
        # (Gaussian2D.forward clamps its render, gaussianlig.py:95); the
        # spline of an unclamped render can overshoot far outside it and
        # would stretch the residual's min-max range
        up = torch.clamp(gradient_aware_upscale(img, dx, dy, dxy, H, W), 0, 1)
        res.up_psnr = psnr(up, gt_hwc)
        resid = gt_hwc - up + 0.5
        lo, hi = resid.min(), resid.max()
        t2 = ((resid - lo) / (hi - lo)).contiguous()
    del lvl1
    lvl2 = LevelFit(n2, H, W, dev, lr=lr, block=block, diag=diag,
                    seed=synthetic.SEED_INIT + 1, rgb_init=rgb_init)
    res.iters_per_s.append(_run(lvl2, t2, iters, log_every))
    with torch.no_grad():
        r2 = torch.clamp(lvl2.render()[0], 0, 1)
        res.level_psnr.append(psnr(r2, t2))
        out = torch.clamp(r2 * (hi - lo) + up - 0.5 + lo, 0, 1)
        res.psnr = psnr(out, gt_hwc)
    res.store_min, res.store_max = float(lo), float(hi)
    return res


def _run(level: LevelFit, target: torch.Tensor, iters: int, log_every: Optional[int]) -> float:
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for it in range(1, iters + 1):
        loss = level.step(target)
        if log_every and it % log_every == 0:
            print(f"  iter {it}: loss {loss.item():.6f}")
    t1.record()
    torch.cuda.synchronize()
    return iters / (t0.elapsed_time(t1) / 1e3)
