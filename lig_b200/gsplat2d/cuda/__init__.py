"""The reference's `_C` function table (csrc/ext.cpp:4-17), same names,
argument order and return tuples, implemented on the lig_b200 C ABI.

Outputs are freshly allocated tensors as in the reference bindings
(csrc/bindings.cu); kernels run on torch's current stream."""
from typing import Optional, Tuple

import torch

from ... import ops


def _hw_from(img_size):
    return int(img_size[1]), int(img_size[0])


def rasterize_forward(tile_bounds, block, img_size, gaussian_ids_sorted, tile_bins, xys, conics,
                      colors, opacities: Optional[torch.Tensor],
                      compute_upscale_gradients: bool = True):
    """csrc/bindings.cu:303-401 -> (out_img, out_wsum, out_dx, out_dy, out_dxy, final_idx)."""
    h, w = _hw_from(img_size)
    b = int(block[0])
    m = int(gaussian_ids_sorted.numel())
    total = torch.full((1,), m, dtype=torch.int32, device=xys.device)
    img, wsum, dx, dy, dxy, fin = ops.raster_fwd(h, w, b, gaussian_ids_sorted.to(torch.int32),
                                                 tile_bins.to(torch.int32), total, xys, conics,
                                                 colors, opacities, compute_upscale_gradients)
    if m == 0:  # the reference kernel leaves zeros when no list is populated
        img.zero_()
    return img, wsum, dx, dy, dxy, fin


def rasterize_backward(img_height, img_width, block_width, gaussians_ids_sorted, tile_bins, xys,
                       conics, colors, final_idx, v_output, v_render_wsum,
                       opacities: Optional[torch.Tensor] = None,
                       v_output_dx: Optional[torch.Tensor] = None,
                       v_output_dy: Optional[torch.Tensor] = None,
                       v_output_dxy: Optional[torch.Tensor] = None):
    """csrc/bindings.cu:403-506 -> (v_xy, v_xy_abs, v_conic, v_colors, v_opacity)."""
    if xys.ndimension() != 2 or xys.size(1) != 2:
        raise RuntimeError("xys must have dimensions (num_points, 2)")
    if colors.ndimension() != 2 or colors.size(1) != 3:
        raise RuntimeError("colors must have 2 dimensions")
    m = int(gaussians_ids_sorted.numel())
    total = torch.full((1,), m, dtype=torch.int32, device=xys.device)
    return ops.raster_bwd(int(img_height), int(img_width), int(block_width),
                          gaussians_ids_sorted.to(torch.int32), tile_bins.to(torch.int32), total,
                          xys, conics, colors, opacities, final_idx, v_output, v_render_wsum,
                          v_output_dx, v_output_dy, v_output_dxy)


def project_gaussians_forward(num_points, cov2d, means2d, opacities, img_height, img_width,
                              block_width):
    """csrc/bindings.cu:68-117."""
    return ops.project_fwd(cov2d[:num_points], means2d[:num_points], opacities, img_height,
                           img_width, block_width, cholesky=False)


def project_gaussians_backward(num_points, extents, conics, v_xy, v_conic):
    """csrc/bindings.cu:119-151 -> (v_cov2d, v_mean2d)."""
    return ops.project_bwd_saved(extents[:num_points], None, conics, v_xy, v_conic,
                                 cholesky=False)


def project_gaussians_forward_cholesky(num_points, cholesky, means2d, opacities, img_height,
                                       img_width, block_width):
    """csrc/bindings.cu:153-202."""
    return ops.project_fwd(cholesky[:num_points], means2d[:num_points], opacities, img_height,
                           img_width, block_width, cholesky=True)


def project_gaussians_backward_cholesky(num_points, extents, cholesky, conics, v_xy, v_conic):
    """csrc/bindings.cu:204-237 -> (v_cholesky, v_mean2d)."""
    return ops.project_bwd_saved(extents[:num_points], cholesky, conics, v_xy, v_conic,
                                 cholesky=True)


def compute_cov2d_bounds(num_pts, covs2d, opacities=None):
    """csrc/bindings.cu:41-66 -> (conics, extents)."""
    return ops.cov2d_bounds(covs2d[:num_pts], opacities)


def map_gaussian_to_intersects(num_points, num_intersects, xys, depths, extents, cum_tiles_hit,
                               tile_bounds, block_width):
    """csrc/bindings.cu:239-281 -> (isect_ids int64, gaussian_ids int32).

    Depth bits: the reference ORs the sign-extended int32 bit pattern of the
    depth into the low word of each written key (csrc/forward.cu:133-138)."""
    tbx, tby = int(tile_bounds[0]), int(tile_bounds[1])
    b = int(block_width)
    isect, gids = ops.map_intersects(xys[:num_points], extents[:num_points],
                                     cum_tiles_hit[:num_points], num_intersects, tby * b,
                                     tbx * b, b)
    if depths is not None and depths.numel() and bool((depths != 0).any()):
        ext = extents[:num_points]
        written = ((ext[:, 0] > 0) & (ext[:, 1] > 0))[gids.long()]
        bits = depths.contiguous().view(torch.int32)[gids.long()].to(torch.int64)
        isect = torch.where(written, isect | bits, isect)
    return isect, gids


def get_tile_bin_edges(num_intersects, isect_ids_sorted, tile_bounds):
    """csrc/bindings.cu:283-301 -> tile_bins [T, 2] int32."""
    T = int(tile_bounds[0]) * int(tile_bounds[1])
    return ops.tile_bin_edges(num_intersects, isect_ids_sorted, T)


def gradient_aware_upscale_forward(render, dx, dy, dxy, dst_h, dst_w,
                                   roi: Tuple[float, float, float, float]):
    """csrc/bindings.cu:508-559."""
    return ops.upscale_fwd(render, dx, dy, dxy, dst_h, dst_w, roi, mode=0)


def gradient_aware_upscale_backward(grad_output, render, dx, dy, dxy, dst_h, dst_w,
                                    roi: Tuple[float, float, float, float]):
    """csrc/bindings.cu:561-605 -> (grad_render, grad_dx, grad_dy, grad_dxy)."""
    return ops.upscale_bwd(grad_output, render.shape[0], render.shape[1], roi, mode=0)
