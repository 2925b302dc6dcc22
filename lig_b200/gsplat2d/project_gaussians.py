"""project_gaussians: drop-in for gsplat2d/gsplat2d/project_gaussians.py:13-104.

Same signature, return tuple and errors.  The backward recomputes the conic,
extent and tile bbox from the saved inputs instead of saving conics/extents
(one kernel, bit-identical to the forward's math)."""
from typing import Optional, Tuple

from torch import Tensor
from torch.autograd import Function

from .. import ops


def project_gaussians(
    cov2d: Tensor,
    means2d: Tensor,
    img_height: int,
    img_width: int,
    block_width: int,
    opacities: Optional[Tensor] = None,
) -> Tuple[Tensor, Tensor, Tensor, Tensor]:
    assert block_width > 1 and block_width <= 16, "block_width must be between 2 and 16"
    return _ProjectGaussians.apply(
        cov2d.contiguous(),
        means2d.contiguous(),
        opacities.contiguous() if opacities is not None else None,
        img_height,
        img_width,
        block_width,
    )


class _ProjectGaussians(Function):
    @staticmethod
    def forward(ctx, cov2d, means2d, opacities, img_height, img_width, block_width):
        num_points = cov2d.shape[-2]
        if num_points < 1 or cov2d.shape[-1] != 3:
            raise ValueError(f"Invalid shape for cov2d: {cov2d.shape}")
        xys, extents, conics, num_tiles_hit = ops.project_fwd(
            cov2d, means2d, opacities, img_height, img_width, block_width, cholesky=False)
        ctx.geom = (img_height, img_width, block_width)
        ctx.save_for_backward(cov2d, means2d, opacities)
        return xys, extents, conics, num_tiles_hit

    @staticmethod
    def backward(ctx, v_xys, v_extents, v_conics, v_num_tiles_hit):
        cov2d, means2d, opacities = ctx.saved_tensors
        h, w, b = ctx.geom
        v_cov2d, v_mean2d = ops.project_bwd(cov2d, means2d, opacities, h, w, b, False,
                                            v_xys, v_conics)
        return v_cov2d, v_mean2d, None, None, None, None
