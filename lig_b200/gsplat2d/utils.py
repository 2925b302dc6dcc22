"""Binning helpers: drop-in for gsplat2d/gsplat2d/utils.py:12-100.

Same names, signatures and return tuples.  `compute_cumulative_intersects`
keeps the reference's contract of returning the count as a Python int (so it
synchronises, as the reference's .item() does); `bin_and_sort_gaussians` runs
emission + stable radix sort + tile ranges in one device pipeline."""
from typing import Optional, Tuple

import torch
from torch import Tensor

from .. import ops
from . import cuda as _C


def map_gaussian_to_intersects(num_points: int, num_intersects: int, xys: Tensor,
                               depths: Tensor, extents: Tensor, cum_tiles_hit: Tensor,
                               tile_bounds: Tuple[int, int, int],
                               block_size: int) -> Tuple[Tensor, Tensor]:
    isect_ids, gaussian_ids = _C.map_gaussian_to_intersects(
        num_points, num_intersects, xys.contiguous(), depths.contiguous(),
        extents.contiguous(), cum_tiles_hit.contiguous(), tile_bounds, block_size)
    return (isect_ids, gaussian_ids)


def get_tile_bin_edges(num_intersects: int, isect_ids_sorted: Tensor,
                       tile_bounds: Tuple[int, int, int]) -> Tensor:
    return _C.get_tile_bin_edges(num_intersects, isect_ids_sorted.contiguous(), tile_bounds)


def compute_cov2d_bounds(cov2d: Tensor,
                         opacities: Optional[Tensor] = None) -> Tuple[Tensor, Tensor]:
    assert cov2d.shape[-1] == 3, (
        f"Expected input cov2d to be of shape (*batch, 3) (upper triangular values), "
        f"but got {tuple(cov2d.shape)}")
    num_pts = cov2d.shape[0]
    assert num_pts > 0
    return _C.compute_cov2d_bounds(num_pts, cov2d.contiguous(),
                                   opacities.contiguous() if opacities is not None else None)


def compute_cumulative_intersects(num_tiles_hit: Tensor) -> Tuple[int, Tensor]:
    cum_tiles_hit, total = ops.cumsum_tiles(num_tiles_hit)
    num_intersects = int(total.item())
    return num_intersects, cum_tiles_hit


def bin_and_sort_gaussians(num_points: int, num_intersects: int, xys: Tensor, depths: Tensor,
                           extents: Tensor, cum_tiles_hit: Tensor,
                           tile_bounds: Tuple[int, int, int], block_size: int):
    """-> (isect_ids, gaussian_ids, isect_ids_sorted, gaussian_ids_sorted, tile_bins).

    Keys with non-zero depth bits fall back to the reference-shaped steps
    (emission with depth bits, 64-bit stable sort, edge detection)."""
    if depths is not None and depths.numel() and bool((depths != 0).any()):
        isect_ids, gaussian_ids = map_gaussian_to_intersects(
            num_points, num_intersects, xys, depths, extents, cum_tiles_hit, tile_bounds,
            block_size)
        isect_ids_sorted, order = torch.sort(isect_ids, stable=True)
        gaussian_ids_sorted = torch.gather(gaussian_ids, 0, order)
        tile_bins = get_tile_bin_edges(num_intersects, isect_ids_sorted, tile_bounds)
        return isect_ids, gaussian_ids, isect_ids_sorted, gaussian_ids_sorted, tile_bins
    tbx, tby = int(tile_bounds[0]), int(tile_bounds[1])
    b = int(block_size)
    total = torch.full((1,), int(num_intersects), dtype=torch.int32, device=xys.device)
    gid_sorted, bins, isect, gids, isect_sorted = ops._run_bin(
        xys[:num_points].contiguous(), extents[:num_points].contiguous(),
        cum_tiles_hit[:num_points].contiguous(), total, tby * b, tbx * b, b,
        int(num_intersects), True)
    m = int(num_intersects)
    return isect[:m], gids[:m], isect_sorted[:m], gid_sorted[:m], bins
