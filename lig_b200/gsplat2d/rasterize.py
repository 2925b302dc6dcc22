"""rasterize_gaussians: drop-in for gsplat2d/gsplat2d/rasterize.py:13-197.

Same signature, return tuple (img, wsum, dx, dy, dxy), errors, empty-list
branch (white image), uint8 colour scaling and ``xys.absgrad``.

Differences in mechanism, not in results:
  * binning is one device pipeline (prefix sum, emission, radix sort, tile
    ranges) with the intersection count checked after the rasterizer is
    already enqueued (see lig_b200.ops), instead of cumsum + .item() +
    torch.sort + gather;
  * kernels run on torch's current stream (the reference launches on the
    legacy default stream);
  * colors must have 3 channels in the forward too (the reference's forward
    kernel reads float3 whatever D is; its backward rejects D != 3).

``alpha_clamp`` (keyword, default None = the reference's clamps: 0.99 in the
sum backward, 0.999 in the gradient-aware one) selects the backward clamp;
0.999 makes the sum backward the exact derivative of its forward.
"""
from typing import Optional, Tuple

import torch
from torch import Tensor
from torch.autograd import Function

from .. import ops


def rasterize_gaussians(
    xys: Tensor,
    extents: Tensor,
    conics: Tensor,
    num_tiles_hit: Tensor,
    colors: Tensor,
    opacities: Optional[Tensor],
    img_height: int,
    img_width: int,
    block_width: int,
    compute_upscale_gradients: bool = False,
    alpha_clamp: Optional[float] = None,
) -> Tuple[Tensor, Tensor, Tensor, Tensor, Tensor]:
    assert block_width > 1 and block_width <= 16, "block_width must be between 2 and 16"
    if colors.dtype == torch.uint8:
        colors = colors.float() / 255

    if xys.ndimension() != 2 or xys.size(1) != 2:
        raise ValueError("xys must have dimensions (N, 2)")

    if colors.ndimension() != 2:
        raise ValueError("colors must have dimensions (N, D)")
    if colors.size(1) != 3:
        raise ValueError("colors must have 3 channels")

    return _RasterizeGaussians.apply(
        xys.contiguous(),
        extents.contiguous(),
        conics.contiguous(),
        num_tiles_hit.contiguous(),
        colors.contiguous(),
        opacities.contiguous() if opacities is not None else None,
        img_height,
        img_width,
        block_width,
        compute_upscale_gradients,
        alpha_clamp,
    )


class _RasterizeGaussians(Function):
    """Rasterizes 2D gaussians (weighted sum)."""

    @staticmethod
    def forward(ctx, xys, extents, conics, num_tiles_hit, colors, opacities, img_height,
                img_width, block_width, compute_upscale_gradients, alpha_clamp=None):
        def enqueue_raster(b):
            return ops.raster_fwd(img_height, img_width, block_width, b.gaussian_ids_sorted,
                                  b.tile_bins, b.total, xys, conics, colors, opacities,
                                  compute_upscale_gradients)

        binning, outs = ops.bin_gaussians(xys, extents, num_tiles_hit, img_height, img_width,
                                          block_width, after_enqueue=enqueue_raster)
        out_img, out_wsum, out_dx, out_dy, out_dxy, final_idx = outs
        if not compute_upscale_gradients:
            out_dx = out_dy = out_dxy = None
        ctx.set_materialize_grads(False)  # unused outputs (e.g. wsum) get no zero tensor
        ctx.img_width = img_width
        ctx.img_height = img_height
        ctx.num_intersects = binning.num_intersects
        ctx.block_width = block_width
        ctx.compute_upscale_gradients = compute_upscale_gradients
        ctx.alpha_clamp = alpha_clamp
        ctx.save_for_backward(binning.gaussian_ids_sorted, binning.tile_bins, binning.total, xys,
                              conics, colors, opacities, final_idx)
        return out_img, out_wsum, out_dx, out_dy, out_dxy

    @staticmethod
    def backward(ctx, v_out_img, v_out_wsum, v_out_dx, v_out_dy, v_out_dxy):
        (gaussian_ids_sorted, tile_bins, total, xys, conics, colors, opacities,
         final_idx) = ctx.saved_tensors
        h, w = ctx.img_height, ctx.img_width
        if v_out_img is None:
            v_out_img = torch.zeros((h, w, 3), dtype=xys.dtype, device=xys.device)
        # v_out_wsum None: the wsum output was unused; the kernel treats it as zero
        ga = ctx.compute_upscale_gradients
        if ga:
            z = None
            if v_out_dx is None or v_out_dy is None or v_out_dxy is None:
                z = torch.zeros((h, w, 3), dtype=xys.dtype, device=xys.device)
            v_out_dx = z if v_out_dx is None else v_out_dx
            v_out_dy = z if v_out_dy is None else v_out_dy
            v_out_dxy = z if v_out_dxy is None else v_out_dxy
        clamp = ctx.alpha_clamp if ctx.alpha_clamp is not None else 0.0
        v_xy, v_xy_abs, v_conic, v_colors, v_opacity = ops.raster_bwd(
            h, w, ctx.block_width, gaussian_ids_sorted, tile_bins, total, xys, conics, colors,
            opacities, final_idx, v_out_img, v_out_wsum,
            v_out_dx if ga else None, v_out_dy if ga else None, v_out_dxy if ga else None,
            alpha_clamp=clamp)
        xys.absgrad = v_xy_abs
        return (
            v_xy,       # xys
            None,       # extents
            v_conic,    # conics
            None,       # num_tiles_hit
            v_colors,   # colors
            v_opacity,  # opacities
            None,       # img_height
            None,       # img_width
            None,       # block_width
            None,       # compute_upscale_gradients
            None,       # alpha_clamp
        )
