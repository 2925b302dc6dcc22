"""gsplat2d API on B200-native kernels — drop-in for gsplat2d/gsplat2d/__init__.py.

Exports the reference's names, its deprecated Function wrappers, and the
GaussianImage-style aliases project_gaussians_2d / rasterize_gaussians_sum.
Use ``lig_b200.install_gsplat2d()`` to make ``import gsplat2d`` resolve here."""
import warnings
from typing import Any

import torch

from .project_gaussians import project_gaussians
from .project_gaussians_cholesky import project_gaussians_cholesky
from .rasterize import rasterize_gaussians
from .upscale import gradient_aware_upscale
from .utils import (
    bin_and_sort_gaussians,
    compute_cov2d_bounds,
    compute_cumulative_intersects,
    get_tile_bin_edges,
    map_gaussian_to_intersects,
)
from .version import __version__

project_gaussians_2d = project_gaussians
rasterize_gaussians_sum = rasterize_gaussians

__all__ = [
    "__version__",
    "project_gaussians",
    "rasterize_gaussians",
    "project_gaussians_cholesky",
    "bin_and_sort_gaussians",
    "compute_cumulative_intersects",
    "compute_cov2d_bounds",
    "get_tile_bin_edges",
    "map_gaussian_to_intersects",
    "gradient_aware_upscale",
    "project_gaussians_2d",
    "rasterize_gaussians_sum",
    "ProjectGaussians",
    "RasterizeGaussians",
    "BinAndSortGaussians",
    "ComputeCumulativeIntersects",
    "ComputeCov2dBounds",
    "GetTileBinEdges",
    "MapGaussiansToIntersects",
]


def _deprecated(name: str, fn_name: str, fn):
    """Deprecated Function wrapper with the reference's behaviour
    (gsplat2d/gsplat2d/__init__.py:38-135): warns, forwards, no backward."""

    def forward(ctx, *args, **kwargs):
        warnings.warn(f"{name} is deprecated, use {fn_name} instead", DeprecationWarning)
        return fn(*args, **kwargs)

    def backward(ctx: Any, *grad_outputs: Any) -> Any:
        raise NotImplementedError

    return type(name, (torch.autograd.Function,),
                {"forward": staticmethod(forward), "backward": staticmethod(backward)})


MapGaussiansToIntersects = _deprecated("MapGaussiansToIntersects", "map_gaussian_to_intersects",
                                       map_gaussian_to_intersects)
ComputeCumulativeIntersects = _deprecated("ComputeCumulativeIntersects",
                                          "compute_cumulative_intersects",
                                          compute_cumulative_intersects)
ComputeCov2dBounds = _deprecated("ComputeCov2dBounds", "compute_cov2d_bounds",
                                 compute_cov2d_bounds)
GetTileBinEdges = _deprecated("GetTileBinEdges", "get_tile_bin_edges", get_tile_bin_edges)
BinAndSortGaussians = _deprecated("BinAndSortGaussians", "bin_and_sort_gaussians",
                                  bin_and_sort_gaussians)
ProjectGaussians = _deprecated("ProjectGaussians", "project_gaussians", project_gaussians)
RasterizeGaussians = _deprecated("RasterizeGaussians", "rasterize_gaussians",
                                 rasterize_gaussians)
