"""torch_gradient_aware_upscale: drop-in for upscaler_torch.py:91-183.

Same align-corners spline (torch.linspace(0, n-1, steps) coordinates, corner
clamping, Hermite basis C^-1), computed by the lig_b200 upscale kernel
(mode 1) with a gather backward, on the input's device rather than a
hard-coded cuda:0, and without materialising [H, W, 4, 4] per channel."""
import torch
from torch.autograd import Function

from . import ops


class _AlignCornersUpscale(Function):
    @staticmethod
    def forward(ctx, render, dx, dy, dxy, new_h, new_w):
        ctx.src_hw = (render.shape[0], render.shape[1])
        return ops.upscale_fwd(render, dx, dy, dxy, new_h, new_w, None, mode=1)

    @staticmethod
    def backward(ctx, g):
        h, w = ctx.src_hw
        gr, gx, gy, gxy = ops.upscale_bwd(g.contiguous(), h, w, None, mode=1)
        return gr, gx, gy, gxy, None, None


def torch_gradient_aware_upscale(render_hwc: torch.Tensor, dx: torch.Tensor, dy: torch.Tensor,
                                 dxy: torch.Tensor, new_h: int, new_w: int) -> torch.Tensor:
    """[H, W, 3] value/dx/dy/dxy planes -> [new_h, new_w, 3]."""
    return _AlignCornersUpscale.apply(render_hwc.contiguous(), dx.contiguous(), dy.contiguous(),
                                      dxy.contiguous(), int(new_h), int(new_w))


def torch_gradient_aware_upscale_single_channel(render, dx, dy, dxy, new_h: int, new_w: int):
    """Single-channel form [H, W] -> [new_h, new_w] (upscaler_torch.py:91-165),
    on the kernel's one-channel instantiation."""
    planes = [t.unsqueeze(-1).contiguous() for t in (render, dx, dy, dxy)]
    return _AlignCornersUpscale.apply(*planes, int(new_h), int(new_w))[..., 0]
