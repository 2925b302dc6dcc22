"""The reference's own CUDA kernels, as a GPU oracle (TEST INFRASTRUCTURE ONLY).

oracle/_ref/libgsplat2d_ref.so is compiled by `make -C oracle ref` from the
reference sources (csrc/forward.cu, backward.cu, gradient_aware_rasterizer.cu,
gradient_aware_upscaler.cu) with the reference's setup.py flags, plus our
torch-free launchers (oracle/ref_launch.cu).  This module restates the
reference's torch glue around them:

  render()  = gaussianlig.Gaussian2D.forward / rasterize.py:54-138 with
              utils.py:61-100 (cumsum, .item(), map, torch.sort, gather, edges)
  backward() = rasterize.py:141-197

The reference sort is `torch.sort(isect_ids)`; its within-tile order is only
defined for a stable sort, so the oracle uses `stable=True` (the order the
reference gets from cub's radix sort on inputs larger than 4096 keys).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Optional

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
# Tests synchronise around every reference launch (clear error attribution);
# timing runs set this False so the reference runs with only its own
# host synchronisations (the .item() of utils.py:66).
STRICT_SYNC = True
LIB_PATH = os.path.join(_HERE, "_ref", "libgsplat2d_ref.so")
_lib = None


def _sync():
    if STRICT_SYNC:
        torch.cuda.synchronize()


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"reference kernels not built ({LIB_PATH}); run `make -C oracle ref`")
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _p(t: Optional[torch.Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


# Converted input copies made by _f stay referenced until the launch that
# reads them has been enqueued (_chk runs after it): freed earlier, the
# caching allocator could hand the block to a later copy in the same call.
_keep = []


def _chk(rc, name):
    _keep.clear()
    if rc != 0:
        raise RuntimeError(f"{name}: CUDA error {rc}")


def _f(t):
    if t is None:
        return None
    t = t.detach().to(torch.float32).contiguous()
    _keep.append(t)
    return t


def project_fwd(in3, means, opac, H, W, B, chol=True):
    n = in3.shape[0]
    dev = in3.device
    xys = torch.empty(n, 2, device=dev)
    ext = torch.empty(n, 2, device=dev)
    con = torch.empty(n, 3, device=dev)
    cnt = torch.empty(n, dtype=torch.int32, device=dev)
    _sync()
    _chk(lib().ref_project_fwd(n, int(chol), _p(_f(in3)), _p(_f(means)), _p(_f(opac)), H, W, B,
                               _p(xys), _p(ext), _p(con), _p(cnt)), "ref_project_fwd")
    _sync()
    return xys, ext, con, cnt


def project_bwd(extents, in3, conics, v_xy, v_conic, chol=True):
    n = extents.shape[0]
    dev = extents.device
    v_in3 = torch.empty(n, 3, device=dev)
    v_mean = torch.empty(n, 2, device=dev)
    _sync()
    _chk(lib().ref_project_bwd(n, int(chol), _p(_f(extents)), _p(_f(in3)), _p(_f(conics)),
                               _p(_f(v_xy)), _p(_f(v_conic)), _p(v_in3), _p(v_mean)),
         "ref_project_bwd")
    _sync()
    return v_in3, v_mean


def cov2d_bounds(cov, opac=None):
    n = cov.shape[0]
    con = torch.empty(n, 3, device=cov.device)
    ext = torch.empty(n, 2, device=cov.device)
    _sync()
    _chk(lib().ref_cov2d_bounds(n, _p(_f(cov)), _p(_f(opac)), _p(con), _p(ext)), "ref_cov2d_bounds")
    _sync()
    return con, ext


@dataclass
class RefBinning:
    num_intersects: int
    cum_tiles_hit: torch.Tensor
    isect_ids: torch.Tensor
    gaussian_ids: torch.Tensor
    isect_ids_sorted: torch.Tensor
    gaussian_ids_sorted: torch.Tensor
    tile_bins: torch.Tensor


def bin_and_sort(xys, extents, counts, H, W, B) -> RefBinning:
    """gsplat2d/gsplat2d/utils.py:61-100 with the reference's map/edge kernels."""
    tbx, tby = (W + B - 1) // B, (H + B - 1) // B
    n = xys.shape[0]
    cum = torch.cumsum(counts, dim=0, dtype=torch.int32)
    m = int(cum[-1].item()) if n else 0
    dev = xys.device
    depths = torch.zeros(n, device=dev)
    isect = torch.empty(m, dtype=torch.int64, device=dev)
    gids = torch.empty(m, dtype=torch.int32, device=dev)
    _sync()
    _chk(lib().ref_map_intersects(n, m, _p(_f(xys)), _p(depths), _p(_f(extents)), _p(cum), tbx,
                                  tby, B, _p(isect), _p(gids)), "ref_map_intersects")
    _sync()
    isect_sorted, order = torch.sort(isect, stable=True)
    gid_sorted = torch.gather(gids, 0, order)
    bins = torch.empty(tbx * tby, 2, dtype=torch.int32, device=dev)
    _sync()
    _chk(lib().ref_tile_bin_edges(m, _p(isect_sorted), tbx * tby, _p(bins)), "ref_tile_bin_edges")
    _sync()
    return RefBinning(m, cum, isect, gids, isect_sorted, gid_sorted, bins)


def raster_fwd(H, W, B, bn: RefBinning, xys, conics, colors, opac, grad_aware=False):
    dev = xys.device
    if bn.num_intersects < 1:  # rasterize.py:80-90
        z3 = torch.zeros(H, W, 3, device=dev)
        return dict(img=torch.ones(H, W, 3, device=dev), wsum=torch.zeros(H, W, device=dev),
                    dx=z3, dy=z3.clone(), dxy=z3.clone(),
                    final_idx=torch.zeros(H, W, dtype=torch.int32, device=dev))
    img = torch.empty(H, W, 3, device=dev)
    wsum = torch.empty(H, W, device=dev)
    fin = torch.empty(H, W, dtype=torch.int32, device=dev)
    dx = torch.empty(H, W, 3, device=dev) if grad_aware else None
    dy = torch.empty(H, W, 3, device=dev) if grad_aware else None
    dxy = torch.empty(H, W, 3, device=dev) if grad_aware else None
    _sync()
    _chk(lib().ref_raster_fwd(H, W, B, _p(bn.gaussian_ids_sorted), _p(bn.tile_bins), _p(_f(xys)),
                              _p(_f(conics)), _p(_f(colors)), _p(_f(opac)), int(grad_aware),
                              _p(fin), _p(img), _p(wsum), _p(dx), _p(dy), _p(dxy)),
         "ref_raster_fwd")
    _sync()
    return dict(img=img, wsum=wsum, dx=dx, dy=dy, dxy=dxy, final_idx=fin)


def raster_bwd(H, W, B, bn: RefBinning, xys, conics, colors, opac, final_idx, v_img, v_wsum,
               v_dx=None, v_dy=None, v_dxy=None):
    n = xys.shape[0]
    dev = xys.device
    v_xy = torch.zeros(n, 2, device=dev)
    v_abs = torch.zeros(n, 2, device=dev)
    v_con = torch.zeros(n, 3, device=dev)
    v_rgb = torch.zeros(n, 3, device=dev)
    v_op = torch.zeros(n, device=dev) if opac is not None else None
    if bn.num_intersects >= 1:
        _sync()
        _chk(lib().ref_raster_bwd(H, W, B, n, _p(bn.gaussian_ids_sorted), _p(bn.tile_bins),
                                  _p(_f(xys)), _p(_f(conics)), _p(_f(colors)), _p(_f(opac)),
                                  _p(final_idx.contiguous()), _p(_f(v_img)), _p(_f(v_wsum)),
                                  _p(_f(v_dx)), _p(_f(v_dy)), _p(_f(v_dxy)), _p(v_xy), _p(v_abs),
                                  _p(v_con), _p(v_rgb), _p(v_op)), "ref_raster_bwd")
        _sync()
    return dict(v_xy=v_xy, v_xy_abs=v_abs, v_conic=v_con, v_rgb=v_rgb, v_opacity=v_op)


def upscale_fwd(f, fx, fy, fxy, dst_h, dst_w, roi=None):
    h, w, _ = f.shape
    if roi is None:
        roi = (0.0, 0.0, float(w), float(h))
    out = torch.empty(dst_h, dst_w, 3, device=f.device)
    _sync()
    cf = ctypes.c_float
    _chk(lib().ref_upscale_fwd(h, w, dst_h, dst_w, cf(roi[0]), cf(roi[1]), cf(roi[2]), cf(roi[3]),
                               _p(_f(f)), _p(_f(fx)), _p(_f(fy)), _p(_f(fxy)), _p(out)),
         "ref_upscale_fwd")
    _sync()
    return out


def upscale_bwd(g, src_h, src_w, roi=None):
    dh, dw, _ = g.shape
    if roi is None:
        roi = (0.0, 0.0, float(src_w), float(src_h))
    outs = [torch.empty(src_h, src_w, 3, device=g.device) for _ in range(4)]
    _sync()
    cf = ctypes.c_float
    _chk(lib().ref_upscale_bwd(src_h, src_w, dh, dw, cf(roi[0]), cf(roi[1]), cf(roi[2]),
                               cf(roi[3]), _p(_f(g)), *[_p(o) for o in outs]), "ref_upscale_bwd")
    _sync()
    return tuple(outs)


def render(in3, means, colors, opac, H, W, B, chol=True, grad_aware=False):
    xys, ext, con, cnt = project_fwd(in3, means, opac, H, W, B, chol)
    bn = bin_and_sort(xys, ext, cnt, H, W, B)
    out = raster_fwd(H, W, B, bn, xys, con, colors, opac, grad_aware)
    out.update(xys=xys, extents=ext, conics=con, counts=cnt, binning=bn)
    return out
