"""Seeded test scenes shared by the parity tests."""
import numpy as np
import torch

from lig_b200 import synthetic


def scene(n, H, W, diag=(0.5, 4.0), seed=0, opac=None, dtype=torch.float32, device="cuda",
          offdiag_std=0.5):
    """means [n,2], cholesky [n,3], colors [n,3], opacities [n] or None."""
    means, chol, colors = synthetic.gaussians(n, H, W, diag=diag, offdiag_std=offdiag_std,
                                              seed=seed, dtype=dtype)
    op = None
    if opac is not None:
        g = torch.Generator().manual_seed(seed + 77)
        lo, hi = opac
        op = (lo + (hi - lo) * torch.rand(n, generator=g, dtype=torch.float64)).to(dtype)
    to = (lambda t: None if t is None else t.to(device))
    return to(means), to(chol), to(colors), to(op)


def chol_to_cov(chol):
    l11, l21, l22 = chol[:, 0], chol[:, 1], chol[:, 2]
    return torch.stack([l11 * l11, l11 * l21, l21 * l21 + l22 * l22], 1)


def np_(t):
    return None if t is None else t.detach().cpu().numpy()


def rel_err(a, b):
    """max |a-b| / (max |b| + tiny): scale-aware relative error of a vector."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / (np.abs(b).max() + 1e-30)) if a.size else 0.0
