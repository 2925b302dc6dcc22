"""Fused fit-loop operator: render + clamped L2 loss as one autograd node.

`render_l2_loss(chol, means, colors, opacities, target, H, W, block)` returns
mean((clamp(render, 0, 1) - target)^2), the loss of gaussianlig.py:95-102
(clamp -> loss_fn 'L2'), with the gradient flowing to the Gaussian
parameters exactly as project_gaussians_cholesky + rasterize_gaussians +
torch.clamp + F.mse_loss would give it — but without materialising the
render, its cotangent, the clamp mask or the unused wsum cotangent: the
forward rasterizer writes the masked difference clamp(x) - target and reduces
the loss from per-tile partials (lig_raster_fwd_l2), and the backward forms
the pixel cotangent from that difference (lig_raster_bwd_diff).
"""
from __future__ import annotations

from typing import Optional

import torch
from torch.autograd import Function

from . import ops


class _RenderL2(Function):
    @staticmethod
    def forward(ctx, chol, means, colors, opacities, target, H, W, block, alpha_clamp):
        xys, ext, con, cnt = ops.project_fwd(chol, means, opacities, H, W, block, True)
        target = target.reshape(H, W, 3)

        def enqueue(b):
            # the backward reads final indices only with opacities
            return ops.raster_fwd_l2(H, W, block, b.gaussian_ids_sorted, b.tile_bins, b.total,
                                     xys, con, colors, opacities, target,
                                     want_final_idx=opacities is not None)

        binning, (diff, fin, loss) = ops.bin_gaussians(xys, ext, cnt, H, W, block,
                                                       after_enqueue=enqueue)
        ctx.geom = (H, W, block)
        ctx.alpha_clamp = alpha_clamp
        ctx.save_for_backward(chol, means, colors, opacities, binning.gaussian_ids_sorted,
                              binning.tile_bins, binning.total, xys, con, diff, fin)
        return loss

    @staticmethod
    def backward(ctx, g):
        (chol, means, colors, opacities, gids, bins, total, xys, con, diff,
         fin) = ctx.saved_tensors
        H, W, block = ctx.geom
        clamp = ctx.alpha_clamp if ctx.alpha_clamp is not None else 0.0
        v_xy, v_abs, v_con, v_rgb, v_op = ops.raster_bwd_diff(
            H, W, block, gids, bins, total, xys, con, colors, opacities, fin, diff,
            g.to(diff.dtype), alpha_clamp=clamp)
        v_chol, v_mean = ops.project_bwd(chol, means, opacities, H, W, block, True, v_xy, v_con)
        return v_chol, v_mean, v_rgb, v_op, None, None, None, None, None


def render_l2_loss(chol: torch.Tensor, means: torch.Tensor, colors: torch.Tensor,
                   opacities: Optional[torch.Tensor], target: torch.Tensor, img_height: int,
                   img_width: int, block_width: int = 16,
                   alpha_clamp: Optional[float] = None) -> torch.Tensor:
    """Loss of one fit iteration (0-d tensor); target is [H, W, 3]."""
    if colors.dim() != 2 or colors.shape[1] != 3:
        raise ValueError("colors must be [N, 3]")
    return _RenderL2.apply(chol.contiguous(), means.contiguous(), colors.contiguous(),
                           opacities.contiguous() if opacities is not None else None,
                           target.contiguous(), int(img_height), int(img_width),
                           int(block_width), alpha_clamp)
