"""gradient_aware_upscale: drop-in for gsplat2d/gsplat2d/upscale.py:10-82
(half-pixel mapping over an optional ROI; backward as a gather)."""
from typing import Optional, Tuple

from torch import Tensor
from torch.autograd import Function

from .. import ops


class _GradientAwareSplineUpscale(Function):
    @staticmethod
    def forward(ctx, render, dx, dy, dxy, dst_h, dst_w, roi):
        ctx.src_hw = (render.shape[0], render.shape[1])
        ctx.dst_h = dst_h
        ctx.dst_w = dst_w
        ctx.roi = roi
        return ops.upscale_fwd(render, dx, dy, dxy, dst_h, dst_w, roi, mode=0)

    @staticmethod
    def backward(ctx, grad_output):
        h, w = ctx.src_hw
        g_render, g_dx, g_dy, g_dxy = ops.upscale_bwd(grad_output.contiguous(), h, w, ctx.roi,
                                                      mode=0)
        return g_render, g_dx, g_dy, g_dxy, None, None, None


def gradient_aware_upscale(
    render: Tensor,
    dx: Tensor,
    dy: Tensor,
    dxy: Tensor,
    dst_h: int,
    dst_w: int,
    roi: Optional[Tuple[float, float, float, float]] = None,
) -> Tensor:
    """Bicubic (Hermite) spline upscale using analytical gradients.

    render, dx, dy, dxy: [H, W, 3]; roi: (x1, y1, x2, y2), default full image.
    Returns [dst_h, dst_w, 3]."""
    h, w, c = render.shape
    if roi is None:
        roi = (0.0, 0.0, float(w), float(h))
    return _GradientAwareSplineUpscale.apply(
        render.contiguous(), dx.contiguous(), dy.contiguous(), dxy.contiguous(), dst_h, dst_w,
        roi)
