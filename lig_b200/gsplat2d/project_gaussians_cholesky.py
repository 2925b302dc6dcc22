"""project_gaussians_cholesky: drop-in for
gsplat2d/gsplat2d/project_gaussians_cholesky.py:10-112 (same signature,
returns, errors).  Backward recomputes the conic from the Cholesky factor."""
from typing import Optional, Tuple

from torch import Tensor
from torch.autograd import Function

from .. import ops


def project_gaussians_cholesky(
    cholesky: Tensor,
    means2d: Tensor,
    img_height: int,
    img_width: int,
    block_width: int,
    opacities: Optional[Tensor] = None,
) -> Tuple[Tensor, Tensor, Tensor, Tensor]:
    """Project gaussians directly from the Cholesky factor [l11, l21, l22].

    Returns xys, extents, conics, num_tiles_hit."""
    assert block_width > 1 and block_width <= 16, "block_width must be between 2 and 16"
    return _ProjectGaussiansCholesky.apply(
        cholesky.contiguous(),
        means2d.contiguous(),
        opacities.contiguous() if opacities is not None else None,
        img_height,
        img_width,
        block_width,
    )


class _ProjectGaussiansCholesky(Function):
    @staticmethod
    def forward(ctx, cholesky, means2d, opacities, img_height, img_width, block_width):
        num_points = cholesky.shape[-2]
        if num_points < 1 or cholesky.shape[-1] != 3:
            raise ValueError(f"Invalid shape for cholesky: {cholesky.shape}")
        xys, extents, conics, num_tiles_hit = ops.project_fwd(
            cholesky, means2d, opacities, img_height, img_width, block_width, cholesky=True)
        ctx.geom = (img_height, img_width, block_width)
        ctx.save_for_backward(cholesky, means2d, opacities)
        return xys, extents, conics, num_tiles_hit

    @staticmethod
    def backward(ctx, v_xys, v_extents, v_conics, v_num_tiles_hit):
        cholesky, means2d, opacities = ctx.saved_tensors
        h, w, b = ctx.geom
        v_chol, v_mean2d = ops.project_bwd(cholesky, means2d, opacities, h, w, b, True,
                                           v_xys, v_conics)
        return v_chol, v_mean2d, None, None, None, None
