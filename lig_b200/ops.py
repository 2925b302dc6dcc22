"""Torch-level wrappers of the lig_b200 C ABI.

Outputs and workspaces are allocated with torch (caching allocator, on the
input's device) and every kernel runs on ``torch.cuda.current_stream()``.

Intersection capacity.  The reference learns the intersection count with a
blocking ``.item()`` between the prefix sum and the emission
(gsplat2d/gsplat2d/utils.py:66), which stalls the GPU while the host launches
the rest of the pipeline.  Here the count stays on the device: binning and
rasterization are enqueued against a speculative capacity (the previous
count for the same problem size plus slack), the 4-byte count is copied to
pinned host memory behind the prefix sum, and the host checks it only after
everything is enqueued.  If the guess was too small (device status flag) the
binning and rasterization are re-run with the exact count.
"""
from __future__ import annotations

import ctypes
import threading
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib
from ._lib import call as _raw_call

_VP = ctypes.c_void_p


def _p(t: Optional[torch.Tensor]):
    return None if t is None else _VP(t.data_ptr())


def _stream(dev: torch.device):
    return _VP(torch.cuda.current_stream(dev).cuda_stream)


def _dt(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return _lib.LIG_F32
    if t.dtype == torch.float64:
        return _lib.LIG_F64
    raise TypeError(f"lig_b200 kernels take float32 or float64 tensors, got {t.dtype}")


def _check_cuda(*ts):
    for t in ts:
        if t is not None and not t.is_cuda:
            raise RuntimeError("lig_b200: tensors must be CUDA tensors (no CPU fallback)")


def _c(t: Optional[torch.Tensor], dtype=None) -> Optional[torch.Tensor]:
    if t is None:
        return None
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()


def tile_bounds(img_h: int, img_w: int, block: int):
    return (img_w + block - 1) // block, (img_h + block - 1) // block


# Optional per-entry-point timing with CUDA events on the launching stream
# (used by bench.py inside its timed region).
_TIMER = None


def call(name, *args):
    t = _TIMER
    if t is None:
        return _raw_call(name, *args)
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record()
    _raw_call(name, *args)
    e.record()
    t.append((name, s, e))


class KernelTimer:
    """Context manager: records (entry point, start, end) events for every
    lig_* call made inside it; summary() -> {name: (calls, total_ms)}."""

    def __enter__(self):
        global _TIMER
        self.events = []
        _TIMER = self.events
        return self

    def __exit__(self, *exc):
        global _TIMER
        _TIMER = None
        return False

    def summary(self):
        torch.cuda.synchronize()
        out = {}
        for name, s, e in self.events:
            n, ms = out.get(name, (0, 0.0))
            out[name] = (n + 1, ms + s.elapsed_time(e))
        return out


def probe_fp32(device=None, blocks=None, iters=4096):
    """Measured FP32 FMA throughput of this device (FLOP/s)."""
    dev = torch.device(device or "cuda")
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks = blocks or sms * 8
    out = torch.empty((blocks,), dtype=torch.float32, device=dev)
    st = _stream(dev)
    for _ in range(2):
        _raw_call("lig_probe_fp32", blocks, iters, _p(out), st)
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record()
    reps = 5
    for _ in range(reps):
        _raw_call("lig_probe_fp32", blocks, iters, _p(out), st)
    e.record()
    torch.cuda.synchronize()
    secs = s.elapsed_time(e) / 1e3
    return reps * blocks * 256.0 * iters * 8 * 2 / secs


# ------------------------------------------------------------------ projection
def project_fwd(in3, means2d, opacities, img_h, img_w, block, cholesky: bool):
    _check_cuda(in3, means2d, opacities)
    in3 = _c(in3)
    means2d = _c(means2d, in3.dtype)
    opacities = _c(opacities, in3.dtype)
    n = in3.shape[0]
    xys = torch.empty((n, 2), dtype=in3.dtype, device=in3.device)
    ext = torch.empty((n, 2), dtype=in3.dtype, device=in3.device)
    con = torch.empty((n, 3), dtype=in3.dtype, device=in3.device)
    cnt = torch.empty((n,), dtype=torch.int32, device=in3.device)
    call("lig_project_fwd", _dt(in3), n, int(cholesky), _p(in3), _p(means2d), _p(opacities),
         int(img_h), int(img_w), int(block), _p(xys), _p(ext), _p(con), _p(cnt),
         _stream(in3.device))
    return xys, ext, con, cnt


def project_fwd_view(in3, means2d, opacities, img_h, img_w, block, cholesky: bool,
                     origin=(0.0, 0.0), scale=(1.0, 1.0)):
    """Projection of the view means' = (means - origin) * scale,
    L' = diag(scale) L (or cov' = S cov S) onto an img_h x img_w output."""
    _check_cuda(in3, means2d, opacities)
    in3 = _c(in3)
    means2d = _c(means2d, in3.dtype)
    opacities = _c(opacities, in3.dtype)
    n = in3.shape[0]
    xys = torch.empty((n, 2), dtype=in3.dtype, device=in3.device)
    ext = torch.empty((n, 2), dtype=in3.dtype, device=in3.device)
    con = torch.empty((n, 3), dtype=in3.dtype, device=in3.device)
    cnt = torch.empty((n,), dtype=torch.int32, device=in3.device)
    call("lig_project_fwd_view", _dt(in3), n, int(cholesky), _p(in3), _p(means2d),
         _p(opacities), int(img_h), int(img_w), int(block), float(origin[0]), float(origin[1]),
         float(scale[0]), float(scale[1]), _p(xys), _p(ext), _p(con), _p(cnt),
         _stream(in3.device))
    return xys, ext, con, cnt


def _rows(t: torch.Tensor, width: int) -> torch.Tensor:
    """Row-strided view accepted by the kernels (unit inner stride)."""
    if t.dim() != 2 or t.shape[1] != width or t.stride(1) != 1 or t.stride(0) < width:
        t = t.contiguous()
    return t


def project_bwd(in3, means2d, opacities, img_h, img_w, block, cholesky, v_xy, v_conic):
    _check_cuda(in3, means2d, v_xy, v_conic)
    in3 = _c(in3)
    means2d = _c(means2d, in3.dtype)
    opacities = _c(opacities, in3.dtype)
    v_xy = _rows(v_xy.to(in3.dtype), 2)
    v_conic = _rows(v_conic.to(in3.dtype), 3)
    n = in3.shape[0]
    v_in3 = torch.empty((n, 3), dtype=in3.dtype, device=in3.device)
    v_mean = torch.empty((n, 2), dtype=in3.dtype, device=in3.device)
    call("lig_project_bwd", _dt(in3), n, int(cholesky), _p(in3), _p(means2d), _p(opacities),
         int(img_h), int(img_w), int(block), _p(v_xy), v_xy.stride(0), _p(v_conic),
         v_conic.stride(0), _p(v_in3), _p(v_mean), _stream(in3.device))
    return v_in3, v_mean


def project_bwd_saved(extents, in3, conics, v_xy, v_conic, cholesky: bool):
    _check_cuda(extents, conics, v_xy, v_conic)
    extents = _c(extents)
    dt = extents.dtype
    conics, v_xy, v_conic = _c(conics, dt), _c(v_xy, dt), _c(v_conic, dt)
    in3 = _c(in3, dt)
    n = extents.shape[0]
    v_in3 = torch.empty((n, 3), dtype=dt, device=extents.device)
    v_mean = torch.empty((n, 2), dtype=dt, device=extents.device)
    call("lig_project_bwd_saved", _dt(extents), n, int(cholesky), _p(extents), _p(in3),
         _p(conics), _p(v_xy), _p(v_conic), _p(v_in3), _p(v_mean), _stream(extents.device))
    return v_in3, v_mean


def cov2d_bounds(cov2d, opacities=None):
    _check_cuda(cov2d, opacities)
    cov2d = _c(cov2d)
    opacities = _c(opacities, cov2d.dtype)
    n = cov2d.shape[0]
    con = torch.empty((n, 3), dtype=cov2d.dtype, device=cov2d.device)
    ext = torch.empty((n, 2), dtype=cov2d.dtype, device=cov2d.device)
    call("lig_cov2d_bounds", _dt(cov2d), n, _p(cov2d), _p(opacities), _p(con), _p(ext),
         _stream(cov2d.device))
    return con, ext


# ------------------------------------------------------------------ binning
def cumsum_tiles(num_tiles_hit: torch.Tensor):
    """Inclusive int32 prefix sum; returns (cum, total) with total a 1-element
    int32 device tensor (no host synchronisation)."""
    _check_cuda(num_tiles_hit)
    cnt = _c(num_tiles_hit.reshape(-1), torch.int32)
    n = cnt.shape[0]
    dev = cnt.device
    cum = torch.empty((n,), dtype=torch.int32, device=dev)
    total = torch.empty((1,), dtype=torch.int32, device=dev)
    wsb = _lib.lib.lig_cumsum_workspace_bytes(n)
    ws = torch.empty((wsb,), dtype=torch.uint8, device=dev)
    call("lig_cumsum_tiles", n, _p(cnt), _p(cum), _p(total), _p(ws), wsb, _stream(dev))
    return cum, total


@dataclass
class Binning:
    num_intersects: int                 # host copy (known after the check)
    total: torch.Tensor                 # device int32 [1]
    capacity: int
    cum_tiles_hit: torch.Tensor
    gaussian_ids_sorted: torch.Tensor   # [capacity] (first num_intersects valid)
    tile_bins: torch.Tensor             # [T, 2] int32
    isect_ids: Optional[torch.Tensor] = None
    gaussian_ids: Optional[torch.Tensor] = None
    isect_ids_sorted: Optional[torch.Tensor] = None


class _HostCount:
    """Per-thread pinned 4-byte landing slot for the device intersection count."""
    _tls = threading.local()

    @classmethod
    def slot(cls) -> torch.Tensor:
        s = getattr(cls._tls, "buf", None)
        if s is None:
            s = torch.empty((1,), dtype=torch.int32, pin_memory=True)
            cls._tls.buf = s
        return s


_CAP_HINT: dict = {}
_SLACK = 1.125


def _run_bin(xys, extents, cum, total, img_h, img_w, block, capacity, want_keys):
    dev = xys.device
    tbx, tby = tile_bounds(img_h, img_w, block)
    T = tbx * tby
    n = xys.shape[0]
    cap = max(int(capacity), 0)
    wsb = _lib.lib.lig_bin_workspace_bytes(n, cap, T)
    ws = torch.empty((max(wsb, 1),), dtype=torch.uint8, device=dev)
    gid_sorted = torch.empty((max(cap, 1),), dtype=torch.int32, device=dev)
    bins = torch.empty((T, 2), dtype=torch.int32, device=dev)
    status = torch.empty((1,), dtype=torch.int32, device=dev)
    isect = gids = isect_sorted = None
    if want_keys:
        isect = torch.empty((max(cap, 1),), dtype=torch.int64, device=dev)
        gids = torch.empty((max(cap, 1),), dtype=torch.int32, device=dev)
        isect_sorted = torch.empty((max(cap, 1),), dtype=torch.int64, device=dev)
    call("lig_bin", _dt(xys), n, _p(xys), _p(extents), _p(cum), _p(total), int(img_h),
         int(img_w), int(block), cap, _p(ws), wsb, _p(gid_sorted), _p(bins), _p(isect),
         _p(gids), _p(isect_sorted), _p(status), _stream(dev))
    return gid_sorted, bins, isect, gids, isect_sorted


def bin_gaussians(xys, extents, num_tiles_hit, img_h, img_w, block, want_keys=False,
                  after_enqueue=None):
    """Prefix sum + emission + stable radix sort + tile ranges.

    ``after_enqueue(binning)`` (optional) is called once the binning is
    enqueued and before the host waits for the count, so callers can enqueue
    the rasterizer behind it; it is called again if the binning is redone."""
    _check_cuda(xys, extents, num_tiles_hit)
    xys = _c(xys)
    extents = _c(extents, xys.dtype)
    n = xys.shape[0]
    cum, total = cumsum_tiles(num_tiles_hit)
    host = _HostCount.slot()
    host.copy_(total, non_blocking=True)
    ev = torch.cuda.Event()
    ev.record(torch.cuda.current_stream(xys.device))
    key = (n, img_h, img_w, block, xys.device.index)
    hint = _CAP_HINT.get(key)
    if hint is None:
        ev.synchronize()
        m = int(host.item())
        cap = m
    else:
        cap = int(hint * _SLACK) + 256
    res = _run_bin(xys, extents, cum, total, img_h, img_w, block, cap, want_keys)
    b = Binning(-1, total, cap, cum, *res)
    extra = after_enqueue(b) if after_enqueue is not None else None
    if hint is not None:
        ev.synchronize()
        m = int(host.item())
        if m > cap:  # speculation failed: redo with the exact count
            res = _run_bin(xys, extents, cum, total, img_h, img_w, block, m, want_keys)
            b = Binning(-1, total, m, cum, *res)
            extra = after_enqueue(b) if after_enqueue is not None else None
    _CAP_HINT[key] = m
    b.num_intersects = m
    return (b, extra) if after_enqueue is not None else b


def map_intersects(xys, extents, cum, num_intersects, img_h, img_w, block):
    _check_cuda(xys, extents, cum)
    xys = _c(xys)
    extents = _c(extents, xys.dtype)
    cum = _c(cum, torch.int32)
    tbx, tby = tile_bounds(img_h, img_w, block)
    m = int(num_intersects)
    isect = torch.empty((m,), dtype=torch.int64, device=xys.device)
    gids = torch.empty((m,), dtype=torch.int32, device=xys.device)
    call("lig_map_intersects", _dt(xys), xys.shape[0], m, _p(xys), _p(extents), _p(cum), tbx,
         tby, int(block), _p(isect), _p(gids), _stream(xys.device))
    return isect, gids


def tile_bin_edges(num_intersects, isect_sorted, num_tiles):
    _check_cuda(isect_sorted)
    isect_sorted = _c(isect_sorted, torch.int64)
    bins = torch.empty((num_tiles, 2), dtype=torch.int32, device=isect_sorted.device)
    call("lig_tile_bin_edges", int(num_intersects), _p(isect_sorted), int(num_tiles), _p(bins),
         _stream(isect_sorted.device))
    return bins


# ------------------------------------------------------------------ raster
def _raster_ws(dtype_code, n, dev):
    wsb = _lib.lib.lig_raster_workspace_bytes(dtype_code, n)
    return torch.empty((wsb,), dtype=torch.uint8, device=dev), wsb


def raster_fwd(img_h, img_w, block, gaussian_ids_sorted, tile_bins, total, xys, conics,
               colors, opacities, grad_aware: bool):
    _check_cuda(xys, conics, colors, opacities, tile_bins, total)
    xys = _c(xys)
    dt = xys.dtype
    conics, colors, opacities = _c(conics, dt), _c(colors, dt), _c(opacities, dt)
    n = xys.shape[0]
    dev = xys.device
    code = _dt(xys)
    ws, wsb = _raster_ws(code, n, dev)
    img = torch.empty((img_h, img_w, 3), dtype=dt, device=dev)
    wsum = torch.empty((img_h, img_w), dtype=dt, device=dev)
    fin = torch.empty((img_h, img_w), dtype=torch.int32, device=dev)
    dx = dy = dxy = None
    if grad_aware:
        dx = torch.empty_like(img)
        dy = torch.empty_like(img)
        dxy = torch.empty_like(img)
    call("lig_raster_fwd", code, int(img_h), int(img_w), int(block), n, _p(gaussian_ids_sorted),
         _p(tile_bins), _p(total), _p(xys), _p(conics), _p(colors), _p(opacities), _p(ws), wsb,
         _p(img), _p(wsum), _p(dx), _p(dy), _p(dxy), _p(fin), _stream(dev))
    return img, wsum, dx, dy, dxy, fin


def raster_bwd(img_h, img_w, block, gaussian_ids_sorted, tile_bins, total, xys, conics, colors,
               opacities, final_idx, v_img, v_wsum, v_dx=None, v_dy=None, v_dxy=None,
               alpha_clamp: float = 0.0):
    _check_cuda(xys, conics, colors, final_idx, v_img)
    xys = _c(xys)
    dt = xys.dtype
    conics, colors, opacities = _c(conics, dt), _c(colors, dt), _c(opacities, dt)
    v_img, v_wsum = _c(v_img, dt), _c(v_wsum, dt)
    v_dx, v_dy, v_dxy = _c(v_dx, dt), _c(v_dy, dt), _c(v_dxy, dt)
    n = xys.shape[0]
    dev = xys.device
    code = _dt(xys)
    ws, wsb = _raster_ws(code, n, dev)
    v_xy = torch.empty((n, 2), dtype=dt, device=dev)
    v_abs = torch.empty((n, 2), dtype=dt, device=dev)
    v_con = torch.empty((n, 3), dtype=dt, device=dev)
    v_rgb = torch.empty((n, 3), dtype=dt, device=dev)
    v_op = torch.empty((n,), dtype=dt, device=dev) if opacities is not None else None
    call("lig_raster_bwd", code, int(img_h), int(img_w), int(block), n, _p(gaussian_ids_sorted),
         _p(tile_bins), _p(total), _p(xys), _p(conics), _p(colors), _p(opacities),
         _p(_c(final_idx, torch.int32)), _p(v_img), _p(v_wsum), _p(v_dx), _p(v_dy), _p(v_dxy),
         float(alpha_clamp), _p(ws), wsb, _p(v_xy), _p(v_abs), _p(v_con), _p(v_rgb), _p(v_op),
         _stream(dev))
    return v_xy, v_abs, v_con, v_rgb, v_op


def raster_bwd_l2(img_h, img_w, block, gaussian_ids_sorted, tile_bins, total, xys, conics,
                  colors, opacities, final_idx, img, target, grad_loss, alpha_clamp: float = 0.0):
    """Sum backward with the clamped-L2 loss gradient computed in-kernel."""
    _check_cuda(xys, conics, colors, final_idx, img, target, grad_loss)
    xys = _c(xys)
    dt = xys.dtype
    conics, colors, opacities = _c(conics, dt), _c(colors, dt), _c(opacities, dt)
    img, target, grad_loss = _c(img, dt), _c(target, dt), _c(grad_loss.reshape(1), dt)
    n = xys.shape[0]
    dev = xys.device
    code = _dt(xys)
    ws, wsb = _raster_ws(code, n, dev)
    v_xy = torch.empty((n, 2), dtype=dt, device=dev)
    v_abs = torch.empty((n, 2), dtype=dt, device=dev)
    v_con = torch.empty((n, 3), dtype=dt, device=dev)
    v_rgb = torch.empty((n, 3), dtype=dt, device=dev)
    v_op = torch.empty((n,), dtype=dt, device=dev) if opacities is not None else None
    call("lig_raster_bwd_l2", code, int(img_h), int(img_w), int(block), n,
         _p(gaussian_ids_sorted), _p(tile_bins), _p(total), _p(xys), _p(conics), _p(colors),
         _p(opacities), _p(_c(final_idx, torch.int32)), _p(img), _p(target), _p(grad_loss),
         float(alpha_clamp), _p(ws), wsb, _p(v_xy), _p(v_abs), _p(v_con), _p(v_rgb), _p(v_op),
         _stream(dev))
    return v_xy, v_abs, v_con, v_rgb, v_op


def raster_fwd_l2(img_h, img_w, block, gaussian_ids_sorted, tile_bins, total, xys, conics,
                  colors, opacities, target, want_final_idx: bool = True):
    """Fit-loop forward with the clamped-L2 loss fused in.  Returns
    (diff [H,W,3], final_idx [H,W], loss 0-d): diff = (0 <= x <= 1) ?
    clamp(x) - target : 0 for the render x, loss = mean((clamp(x) - target)^2).
    A uint8 target (an RGB image as stored) is read as byte / 255, the value
    torchvision's ToTensor gives.  want_final_idx=False (the backward without
    opacities never reads it): final_idx is None and the kernel neither
    tracks nor writes it."""
    _check_cuda(xys, conics, colors, opacities, tile_bins, total, target)
    xys = _c(xys)
    dt = xys.dtype
    conics, colors, opacities = _c(conics, dt), _c(colors, dt), _c(opacities, dt)
    u8 = target.dtype == torch.uint8
    target = target.contiguous() if u8 else _c(target, dt)
    n = xys.shape[0]
    dev = xys.device
    code = _dt(xys)
    ws, wsb = _raster_ws(code, n, dev)
    tbx, tby = tile_bounds(img_h, img_w, block)
    part = torch.empty((_lib.lib.lig_l2_tile_partials_bytes(tbx * tby) // 8,), dtype=torch.float64,
                       device=dev)
    diff = torch.empty((img_h, img_w, 3), dtype=dt, device=dev)
    fin = torch.empty((img_h, img_w), dtype=torch.int32, device=dev) if want_final_idx else None
    loss = torch.empty((), dtype=dt, device=dev)
    call("lig_raster_fwd_l2_u8" if u8 else "lig_raster_fwd_l2", code, int(img_h), int(img_w),
         int(block), n,
         _p(gaussian_ids_sorted), _p(tile_bins), _p(total), _p(xys), _p(conics), _p(colors),
         _p(opacities), _p(target), _p(ws), wsb, _p(part), _p(diff), _p(fin), _p(loss),
         _stream(dev))
    return diff, fin, loss


def raster_bwd_diff(img_h, img_w, block, gaussian_ids_sorted, tile_bins, total, xys, conics,
                    colors, opacities, final_idx, diff, grad_loss, alpha_clamp: float = 0.0):
    """Sum backward of the fused-L2 forward's loss, from its diff."""
    _check_cuda(xys, conics, colors, final_idx, diff, grad_loss)
    xys = _c(xys)
    dt = xys.dtype
    conics, colors, opacities = _c(conics, dt), _c(colors, dt), _c(opacities, dt)
    diff, grad_loss = _c(diff, dt), _c(grad_loss.reshape(1), dt)
    n = xys.shape[0]
    dev = xys.device
    code = _dt(xys)
    ws, wsb = _raster_ws(code, n, dev)
    v_xy = torch.empty((n, 2), dtype=dt, device=dev)
    v_abs = torch.empty((n, 2), dtype=dt, device=dev)
    v_con = torch.empty((n, 3), dtype=dt, device=dev)
    v_rgb = torch.empty((n, 3), dtype=dt, device=dev)
    v_op = torch.empty((n,), dtype=dt, device=dev) if opacities is not None else None
    call("lig_raster_bwd_diff", code, int(img_h), int(img_w), int(block), n,
         _p(gaussian_ids_sorted), _p(tile_bins), _p(total), _p(xys), _p(conics), _p(colors),
         _p(opacities), _p(_c(final_idx, torch.int32)), _p(diff), _p(grad_loss),
         float(alpha_clamp), _p(ws), wsb, _p(v_xy), _p(v_abs), _p(v_con), _p(v_rgb), _p(v_op),
         _stream(dev))
    return v_xy, v_abs, v_con, v_rgb, v_op


def l2_clamped_loss(img, target):
    """mean((clamp(img, 0, 1) - target)^2) as a 0-d device tensor."""
    _check_cuda(img, target)
    img = _c(img)
    target = _c(target, img.dtype)
    if img.numel() != target.numel():
        raise ValueError("img and target must have the same number of elements")
    out = torch.empty((), dtype=img.dtype, device=img.device)
    wsb = _lib.lib.lig_l2_workspace_bytes()
    ws = torch.empty((wsb,), dtype=torch.uint8, device=img.device)
    call("lig_l2_clamped_loss", _dt(img), img.numel(), _p(img), _p(target), _p(out), _p(ws), wsb,
         _stream(img.device))
    return out


# ------------------------------------------------------------------ upscale
def upscale_fwd(render, dx, dy, dxy, dst_h, dst_w, roi=None, mode: int = 0):
    """[H, W, C] value / dx / dy / dxy planes (C = 3, or 1 for the
    single-channel form) -> [dst_h, dst_w, C]."""
    _check_cuda(render, dx, dy, dxy)
    render = _c(render)
    dt = render.dtype
    dx, dy, dxy = _c(dx, dt), _c(dy, dt), _c(dxy, dt)
    h, w, c = render.shape
    if c not in (1, 3):
        raise ValueError("gradient-aware upscale expects [H, W, 3] (or [H, W, 1]) planes")
    if roi is None:
        roi = (0.0, 0.0, float(w), float(h))
    out = torch.empty((int(dst_h), int(dst_w), c), dtype=dt, device=render.device)
    call("lig_upscale_fwd_nc", _dt(render), int(mode), c, h, w, int(dst_h), int(dst_w),
         float(roi[0]), float(roi[1]), float(roi[2]), float(roi[3]), _p(render), _p(dx), _p(dy),
         _p(dxy), _p(out), _stream(render.device))
    return out


def upscale_bwd(grad_out, src_h, src_w, roi=None, mode: int = 0):
    _check_cuda(grad_out)
    grad_out = _c(grad_out)
    dt = grad_out.dtype
    dh, dw, c = grad_out.shape
    if c not in (1, 3):
        raise ValueError("gradient-aware upscale expects [H, W, 3] (or [H, W, 1]) planes")
    if roi is None:
        roi = (0.0, 0.0, float(src_w), float(src_h))
    outs = [torch.empty((int(src_h), int(src_w), c), dtype=dt, device=grad_out.device)
            for _ in range(4)]
    call("lig_upscale_bwd_nc", _dt(grad_out), int(mode), c, int(src_h), int(src_w), dh, dw,
         float(roi[0]), float(roi[1]), float(roi[2]), float(roi[3]), _p(grad_out),
         *[_p(o) for o in outs], _stream(grad_out.device))
    return tuple(outs)
