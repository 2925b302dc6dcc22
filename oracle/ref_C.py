"""The reference's `_C` extension table on the reference's own kernels
(TEST INFRASTRUCTURE ONLY).

The reference's gsplat2d package reaches its CUDA code through
`gsplat2d.cuda._backend._C`, a torch extension built from csrc/ext.cpp and
csrc/bindings.cu.  This module is that table with the same eleven names,
argument order and return tuples (csrc/bindings.h:19-159), each entry
allocating zero-filled outputs as csrc/bindings.cu does and launching the
unmodified reference kernels in oracle/_ref/libgsplat2d_ref.so (built by
`make -C oracle ref`; launchers in oracle/ref_launch.cu).  Registered as
`gsplat2d.cuda._backend`, it lets the reference's own Python glue
(rasterize.py, utils.py, project_gaussians*.py, upscale.py — compiled
unchanged into oracle/_ref/py by oracle/compile_callers.py) run as the
checker beside this library.  Undefined outputs of the C++ bindings (dx/dy/dxy
without upscale gradients, v_opacity without opacities) are None, as pybind
returns them.
"""
from __future__ import annotations

from typing import Optional

import torch

from . import ref
from .ref import _chk, _f, _p, _sync, lib


def _zeros(*shape, like: torch.Tensor, dtype=torch.float32):
    return torch.zeros(*shape, dtype=dtype, device=like.device)


def compute_cov2d_bounds(num_pts, covs2d, opacities=None):
    """csrc/bindings.cu:41-66 -> (conics, extents)."""
    return ref.cov2d_bounds(covs2d[:num_pts], opacities)


def _project(num_points, in3, means2d, opacities, img_height, img_width, block_width, chol):
    xys, ext, con, cnt = ref.project_fwd(in3[:num_points], means2d[:num_points], opacities,
                                         int(img_height), int(img_width), int(block_width),
                                         chol=chol)
    return xys, ext, con, cnt


def project_gaussians_forward(num_points, cov2d, means2d, opacities, img_height, img_width,
                              block_width):
    """csrc/bindings.cu:68-117 -> (xys, extents, conics, num_tiles_hit)."""
    return _project(num_points, cov2d, means2d, opacities, img_height, img_width, block_width,
                    False)


def project_gaussians_forward_cholesky(num_points, cholesky, means2d, opacities, img_height,
                                       img_width, block_width):
    """csrc/bindings.cu:153-202."""
    return _project(num_points, cholesky, means2d, opacities, img_height, img_width,
                    block_width, True)


def project_gaussians_backward(num_points, extents, conics, v_xy, v_conic):
    """csrc/bindings.cu:119-151 -> (v_cov2d, v_mean2d)."""
    return ref.project_bwd(extents[:num_points], None, conics, v_xy, v_conic, chol=False)


def project_gaussians_backward_cholesky(num_points, extents, cholesky, conics, v_xy, v_conic):
    """csrc/bindings.cu:204-237 -> (v_cholesky, v_mean2d)."""
    return ref.project_bwd(extents[:num_points], cholesky, conics, v_xy, v_conic, chol=True)


def map_gaussian_to_intersects(num_points, num_intersects, xys, depths, extent, cum_tiles_hit,
                               tile_bounds, block_width):
    """csrc/bindings.cu:239-281 -> (isect_ids int64, gaussian_ids int32)."""
    n, m = int(num_points), int(num_intersects)
    xys, depths, extent = _f(xys), _f(depths), _f(extent)
    cum = cum_tiles_hit.to(torch.int32).contiguous()
    isect = _zeros(m, like=xys, dtype=torch.int64)
    gids = _zeros(m, like=xys, dtype=torch.int32)
    _sync()
    _chk(lib().ref_map_intersects(n, m, _p(xys), _p(depths), _p(extent), _p(cum),
                                  int(tile_bounds[0]), int(tile_bounds[1]), int(block_width),
                                  _p(isect), _p(gids)), "ref_map_intersects")
    _sync()
    return isect, gids


def get_tile_bin_edges(num_intersects, isect_ids_sorted, tile_bounds):
    """csrc/bindings.cu:283-301 -> tile_bins [T, 2] int32."""
    t = int(tile_bounds[0]) * int(tile_bounds[1])
    keys = isect_ids_sorted.contiguous()
    bins = _zeros(t, 2, like=keys, dtype=torch.int32)
    _sync()
    _chk(lib().ref_tile_bin_edges(int(num_intersects), _p(keys), t, _p(bins)),
         "ref_tile_bin_edges")
    _sync()
    return bins


def rasterize_forward(tile_bounds, block, img_size, gaussian_ids_sorted, tile_bins, xys, conics,
                      colors, opacities: Optional[torch.Tensor],
                      compute_upscale_gradients: bool = True):
    """csrc/bindings.cu:303-401 -> (out_img, out_wsum, out_dx, out_dy, out_dxy, final_idx)."""
    W, H = int(img_size[0]), int(img_size[1])
    B = int(block[0])
    # inputs held in locals: a converted copy must outlive the launch
    ids, bins = gaussian_ids_sorted.contiguous(), tile_bins.contiguous()
    xys, conics, colors, opac = _f(xys), _f(conics), _f(colors), _f(opacities)
    ch = colors.shape[1]
    img = _zeros(H, W, ch, like=xys)
    wsum = _zeros(H, W, like=xys)
    fin = _zeros(H, W, like=xys, dtype=torch.int32)
    ga = bool(compute_upscale_gradients)
    dx, dy, dxy = ((_zeros(H, W, ch, like=xys) for _ in range(3)) if ga else (None,) * 3)
    _sync()
    _chk(lib().ref_raster_fwd(H, W, B, _p(ids), _p(bins), _p(xys), _p(conics), _p(colors),
                              _p(opac), int(ga), _p(fin), _p(img), _p(wsum), _p(dx), _p(dy),
                              _p(dxy)), "ref_raster_fwd")
    _sync()
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
    n = xys.shape[0]
    ga = v_output_dx is not None
    ids, bins, fin = (gaussians_ids_sorted.contiguous(), tile_bins.contiguous(),
                      final_idx.contiguous())
    xys, conics, colors, opac = _f(xys), _f(conics), _f(colors), _f(opacities)
    v_out, v_w = _f(v_output), _f(v_render_wsum)
    v_dx, v_dy, v_dxy = ((_f(v_output_dx), _f(v_output_dy), _f(v_output_dxy)) if ga
                         else (None,) * 3)
    v_xy, v_abs = _zeros(n, 2, like=xys), _zeros(n, 2, like=xys)
    v_con, v_rgb = _zeros(n, 3, like=xys), _zeros(n, 3, like=xys)
    v_op = _zeros(n, like=xys) if opac is not None else None
    _sync()
    _chk(lib().ref_raster_bwd(int(img_height), int(img_width), int(block_width), n, _p(ids),
                              _p(bins), _p(xys), _p(conics), _p(colors), _p(opac), _p(fin),
                              _p(v_out), _p(v_w), _p(v_dx), _p(v_dy), _p(v_dxy), _p(v_xy),
                              _p(v_abs), _p(v_con), _p(v_rgb), _p(v_op)), "ref_raster_bwd")
    _sync()
    return v_xy, v_abs, v_con, v_rgb, v_op


def gradient_aware_upscale_forward(render, dx, dy, dxy, dst_h, dst_w, roi):
    """csrc/bindings.cu:508-559."""
    return ref.upscale_fwd(render, dx, dy, dxy, int(dst_h), int(dst_w), roi)


def gradient_aware_upscale_backward(grad_output, render, dx, dy, dxy, dst_h, dst_w, roi):
    """csrc/bindings.cu:561-605 -> (grad_render, grad_dx, grad_dy, grad_dxy)."""
    h, w = int(render.shape[0]), int(render.shape[1])
    return ref.upscale_bwd(grad_output, h, w, roi)


__all__ = ["compute_cov2d_bounds", "project_gaussians_forward",
           "project_gaussians_forward_cholesky", "project_gaussians_backward",
           "project_gaussians_backward_cholesky", "map_gaussian_to_intersects",
           "get_tile_bin_edges", "rasterize_forward", "rasterize_backward",
           "gradient_aware_upscale_forward", "gradient_aware_upscale_backward"]
