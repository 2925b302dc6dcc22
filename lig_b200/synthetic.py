"""Seeded synthetic workloads standing in for the DIV2K / STimage images the
reference trains on (not available here): Gaussians drawn as in the fit
configurations (means uniform over the image, Cholesky diagonals uniform,
off-diagonal normal with std 0.5, colours uniform), a target rendered from a
"teacher" set plus noise.  All draws use a CPU torch.Generator per purpose so
CPU and GPU paths see identical bits.  Seeds: teacher 0, noise 1, fit-init 2,
cotangents 3."""
from __future__ import annotations

import math

import torch

SEED_TEACHER, SEED_NOISE, SEED_INIT, SEED_COT = 0, 1, 2, 3


def gaussians(n: int, H: int, W: int, diag=(0.5, 4.0), offdiag_std: float = 0.5,
              seed: int = SEED_TEACHER, dtype=torch.float32):
    """-> means [n,2] (x,y), cholesky [n,3] (l11,l21,l22), colors [n,3] on CPU."""
    g = torch.Generator().manual_seed(seed)
    means = torch.rand(n, 2, generator=g, dtype=torch.float64) * torch.tensor(
        [float(W), float(H)], dtype=torch.float64)
    lo, hi = diag
    l11 = lo + (hi - lo) * torch.rand(n, generator=g, dtype=torch.float64)
    l22 = lo + (hi - lo) * torch.rand(n, generator=g, dtype=torch.float64)
    l21 = offdiag_std * torch.randn(n, generator=g, dtype=torch.float64)
    chol = torch.stack([l11, l21, l22], 1)
    colors = torch.rand(n, 3, generator=g, dtype=torch.float64)
    return means.to(dtype), chol.to(dtype), colors.to(dtype)


def gaussians_on_device(n: int, H: int, W: int, device, diag=(0.5, 4.0),
                        offdiag_std: float = 0.5, seed: int = SEED_TEACHER):
    """The distribution of gaussians() drawn on the device with a device
    generator (a different random stream from the CPU one): no host work or
    host-to-device copies, for fit requests arriving at a running server."""
    g = torch.Generator(device=device).manual_seed(seed)
    kw = dict(generator=g, device=device, dtype=torch.float32)
    means = torch.rand(n, 2, **kw) * torch.tensor([float(W), float(H)], device=device)
    lo, hi = diag
    l11 = lo + (hi - lo) * torch.rand(n, **kw)
    l22 = lo + (hi - lo) * torch.rand(n, **kw)
    l21 = offdiag_std * torch.randn(n, **kw)
    chol = torch.stack([l11, l21, l22], 1)
    colors = torch.rand(n, 3, **kw)
    return means, chol, colors


def white_noise(H: int, W: int, std: float, seed: int = SEED_NOISE) -> torch.Tensor:
    g = torch.Generator().manual_seed(seed)
    return std * torch.randn(H, W, 3, generator=g)


def spectral_noise(H: int, W: int, std: float, seed: int = SEED_NOISE,
                   device="cpu") -> torch.Tensor:
    """1/f^2-power ("pink-2D") noise per channel: white N(0,1) -> FFT -> amplitude
    * 1/|f| (DC = 0) -> inverse FFT -> scaled to the given std.  [H, W, 3]."""
    g = torch.Generator().manual_seed(seed)
    white = torch.randn(3, H, W, generator=g).to(device)
    fy = torch.fft.fftfreq(H, device=device).view(H, 1)
    fx = torch.fft.rfftfreq(W, device=device).view(1, W // 2 + 1)
    f = torch.sqrt(fx * fx + fy * fy)
    amp = torch.where(f > 0, 1.0 / torch.clamp(f, min=1e-12), torch.zeros_like(f))
    spec = torch.fft.rfft2(white) * amp
    out = torch.fft.irfft2(spec, s=(H, W))
    out = out - out.mean(dim=(1, 2), keepdim=True)
    out = out * (std / out.std(dim=(1, 2), keepdim=True).clamp_min(1e-12))
    return out.permute(1, 2, 0).contiguous()


def fit_shapes(i: int, base_seed: int = 1000):
    """Image shape of item i of the batched uneven fit: height log-uniform in
    [256, 4096], width = round(H * U[0.5, 2]) clipped to [256, 4096]."""
    g = torch.Generator().manual_seed(base_seed + i)
    h = int(round(math.exp(math.log(256) + (math.log(4096) - math.log(256)) * torch.rand(1, generator=g).item())))
    w = int(round(h * (0.5 + 1.5 * torch.rand(1, generator=g).item())))
    return h, min(max(w, 256), 4096)
