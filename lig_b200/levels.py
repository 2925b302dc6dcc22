"""LIG level pipeline: the residual target between levels, the multi-level
compose of a decode, and the checkpoint format.

* ``residual_target(gt, up)`` -> (target, store_min, store_max): the next
  level's target of train.py:113-126 (gt - up + 0.5, min-max normalised),
  two device passes, bit-identical to the torch expression.
* ``compose(prev, render, store_min, store_max, last)``: one decode step of
  train.py:188-200 (bilinear resize of the running image + de-normalised
  level render, final clamp) in one pass.
* ``save_lig`` / ``load_lig``: the reference's checkpoint layout
  (train.py:172-176): {'state_dict': [per-level {'means', 'cov2d', 'rgbs'}],
  'store_max': [...], 'store_min': [...]}, readable by the reference's loader
  (train.py:58-67), which keeps only the keys its modules know; Cholesky
  levels also carry 'cholesky', and every level its 'H' / 'W'.
* ``decode_lig(model)``: render every level and compose (SimpleTrainer2d.test,
  train.py:181-200).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import torch

from . import ops
from .ops import call
from .serve import GaussianSet, render_view

_VP = ctypes.c_void_p


def _p(t):
    return None if t is None else _VP(t.data_ptr())


def _f32(t: torch.Tensor) -> torch.Tensor:
    if not t.is_cuda:
        raise RuntimeError("lig_b200: tensors must be CUDA tensors (no CPU fallback)")
    return t.to(torch.float32).contiguous()


def residual_target(gt_hwc: torch.Tensor, up_hwc: torch.Tensor):
    """-> (target [H,W,3], store_min, store_max as 0-d device tensors)."""
    gt, up = _f32(gt_hwc), _f32(up_hwc)
    if gt.shape != up.shape:
        raise ValueError("gt and up must have the same shape")
    out = torch.empty_like(gt)
    mm = torch.empty(2, dtype=torch.float32, device=gt.device)
    call("lig_level_residual", gt.numel(), _p(gt), _p(up), _p(out), _p(mm),
         ops._stream(gt.device))
    return out, mm[0], mm[1]


def compose(prev: Optional[torch.Tensor], render: torch.Tensor, store_min, store_max,
            last: bool, clamp_render: bool = True) -> torch.Tensor:
    """base + (clamp(render) * (max - min) - 0.5 + min), base = prev resized
    bilinearly to render's size (None: 0); clamped to [0, 1] when last.
    store_min / store_max: floats or 0-d device tensors."""
    render = _f32(render)
    H, W = render.shape[:2]
    if prev is not None:
        prev = _f32(prev)
    mm = None
    lo = hi = 0.0
    if torch.is_tensor(store_min):
        mm = torch.stack([store_min.reshape(()), store_max.reshape(())]).to(
            device=render.device, dtype=torch.float32).contiguous()
    else:
        lo, hi = float(store_min), float(store_max)
    out = torch.empty_like(render)
    ph, pw = (prev.shape[0], prev.shape[1]) if prev is not None else (0, 0)
    call("lig_level_compose", ph, pw, _p(prev), H, W, _p(render), _p(mm), lo, hi,
         int(clamp_render), int(last), _p(out), ops._stream(render.device))
    return out


# --------------------------------------------------------------- checkpoint
@dataclass
class LIGModel:
    levels: List[GaussianSet]
    store_min: List[float] = field(default_factory=list)
    store_max: List[float] = field(default_factory=list)


def _cov_from_chol(ch: torch.Tensor) -> torch.Tensor:
    l11, l21, l22 = ch[:, 0], ch[:, 1], ch[:, 2]
    return torch.stack([l11 * l11, l11 * l21, l21 * l21 + l22 * l22], 1)


def save_lig(path, levels: Sequence[GaussianSet], store_min: Sequence, store_max: Sequence):
    """Write the reference's multi-level checkpoint (train.py:172-176)."""
    sd = []
    for gs in levels:
        d = {"means": gs.means.detach().cpu(), "rgbs": gs.rgbs.detach().cpu(),
             "H": int(gs.H), "W": int(gs.W)}
        if gs.cholesky:
            d["cholesky"] = gs.chol.detach().cpu()
            d["cov2d"] = _cov_from_chol(gs.chol.detach()).cpu()
        else:
            d["cov2d"] = gs.chol.detach().cpu()
        if gs.opacities is not None:
            d["opacities"] = gs.opacities.detach().cpu()
        sd.append(d)
    torch.save({"state_dict": sd,
                "store_max": [float(x) for x in store_max],
                "store_min": [float(x) for x in store_min]}, path)


def level_sizes(H: int, W: int, n_scales: int):
    """Level image sizes of gaussianlig.LIG (gaussianlig.py:23-27)."""
    return [(int(H * pow(2.0, -n_scales + s + 1)), int(W * pow(2.0, -n_scales + s + 1)))
            for s in range(n_scales)]


def load_lig(path, device="cuda", image_hw: Optional[tuple] = None) -> LIGModel:
    """Read a multi-level checkpoint into resident sets.  Level sizes come
    from the file ('H'/'W') or, for the reference's own files, from
    image_hw and the level count as gaussianlig.LIG derives them."""
    ck = torch.load(path, map_location="cpu", weights_only=False)
    sds = ck["state_dict"]
    sizes = None
    if image_hw is not None:
        sizes = level_sizes(image_hw[0], image_hw[1], len(sds))
    levels = []
    for s, d in enumerate(sds):
        if "H" in d and "W" in d:
            H, W = int(d["H"]), int(d["W"])
        elif sizes is not None:
            H, W = sizes[s]
        else:
            raise ValueError("level sizes are not in the file: pass image_hw")
        chol = "cholesky" in d
        in3 = d["cholesky"] if chol else d["cov2d"]
        op = d.get("opacities")
        levels.append(GaussianSet(d["means"].to(device, torch.float32).contiguous(),
                                  in3.to(device, torch.float32).contiguous(),
                                  d["rgbs"].to(device, torch.float32).contiguous(), H, W,
                                  None if op is None else op.to(device, torch.float32),
                                  cholesky=chol))
    return LIGModel(levels, [float(x) for x in ck.get("store_min", [])],
                    [float(x) for x in ck.get("store_max", [])])


def decode_lig(model: LIGModel, block: int = 16) -> torch.Tensor:
    """Full-resolution decode: level 0's clamped render, then per level the
    bilinear resize of the running image plus the de-normalised clamped
    render of that level, clamped at the end (train.py:181-200)."""
    out = None
    n = len(model.levels)
    for s, gs in enumerate(model.levels):
        img = render_view(gs, gs.H, gs.W, block=block)[0]
        last = s == n - 1
        if s == 0:
            out = torch.clamp(img, 0, 1)  # Gaussian2D.forward clamps its render
        else:
            out = compose(out, img, model.store_min[s - 1], model.store_max[s - 1], last)
    return out
