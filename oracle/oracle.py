"""numpy front-end of the C restatement in oracle/lig_oracle.c.

TEST INFRASTRUCTURE ONLY.  Used by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of bench.py as the checker / CPU timing of the gsplat2d hot
path; the product package (lig_b200) never imports it.

Every function mirrors one reference entry point (paths relative to the
reference project root, "csrc/" = gsplat2d/gsplat2d/cuda/csrc/):

  project_fwd      csrc/bindings.cu:73-117, :158-202   (forward.cu:13-105)
  project_bwd      csrc/bindings.cu:122-151, :207-237  (backward.cu:185-246)
  cov2d_bounds     csrc/bindings.cu:19-66
  cumsum           gsplat2d/gsplat2d/utils.py:61-67
  map_intersects   gsplat2d/gsplat2d/utils.py:12-33    (forward.cu:109-143)
  sort_by_tile     gsplat2d/gsplat2d/utils.py:97-98    (stable torch.sort)
  tile_bins        gsplat2d/gsplat2d/utils.py:36-44    (forward.cu:148-170)
  bin_and_sort     gsplat2d/gsplat2d/utils.py:70-100
  raster_fwd       csrc/bindings.cu:304-401 + rasterize.py:78-121
  raster_bwd       csrc/bindings.cu:411-506 + rasterize.py:141-197
  upscale_fwd/bwd  csrc/bindings.cu:508-605 (mode 0), upscaler_torch.py:91-183 (mode 1)
  dense_fwd_f64    FP64 dense evaluation with the reference's culling
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblig_oracle.so")
_lib = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile liblig_oracle.so with oracle/Makefile if it is missing."""
    if not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE, "liblig_oracle.so"], check=True)
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
    return _lib


def _sfx(dtype) -> str:
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _arr(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


def _real(dtype):
    return ctypes.c_double if np.dtype(dtype) == np.float64 else ctypes.c_float


def tile_bounds(H: int, W: int, B: int):
    return (W + B - 1) // B, (H + B - 1) // B


# ----------------------------------------------------------------- projection
def project_fwd(in3, means, opac, H, W, B, chol=False, dtype=np.float32):
    in3, means, opac = _arr(in3, dtype), _arr(means, dtype), _arr(opac, dtype)
    n = in3.shape[0]
    xys = np.zeros((n, 2), dtype)
    ext = np.zeros((n, 2), dtype)
    con = np.zeros((n, 3), dtype)
    cnt = np.zeros((n,), np.int32)
    getattr(lib(), "orc_project_fwd_" + _sfx(dtype))(
        ctypes.c_int(n), ctypes.c_int(int(chol)), _ptr(in3), _ptr(means), _ptr(opac),
        ctypes.c_int(H), ctypes.c_int(W), ctypes.c_int(B),
        _ptr(xys), _ptr(ext), _ptr(con), _ptr(cnt))
    return xys, ext, con, cnt


def project_bwd(extents, in3, conics, v_xy, v_conic, chol=False, dtype=np.float32):
    extents, conics = _arr(extents, dtype), _arr(conics, dtype)
    in3 = _arr(in3, dtype)
    v_xy, v_conic = _arr(v_xy, dtype), _arr(v_conic, dtype)
    n = extents.shape[0]
    v_in3 = np.zeros((n, 3), dtype)
    v_mean = np.zeros((n, 2), dtype)
    getattr(lib(), "orc_project_bwd_" + _sfx(dtype))(
        ctypes.c_int(n), ctypes.c_int(int(chol)), _ptr(extents), _ptr(in3), _ptr(conics),
        _ptr(v_xy), _ptr(v_conic), _ptr(v_in3), _ptr(v_mean))
    return v_in3, v_mean


def cov2d_bounds(cov, opac=None, dtype=np.float32):
    cov, opac = _arr(cov, dtype), _arr(opac, dtype)
    n = cov.shape[0]
    con = np.zeros((n, 3), dtype)
    ext = np.zeros((n, 2), dtype)
    getattr(lib(), "orc_cov2d_bounds_" + _sfx(dtype))(
        ctypes.c_int(n), _ptr(cov), _ptr(opac), _ptr(con), _ptr(ext))
    return con, ext


# ----------------------------------------------------------------- binning
def cumsum(counts):
    counts = _arr(counts, np.int32)
    out = np.zeros_like(counts)
    lib().orc_cumsum_i32(ctypes.c_int(counts.shape[0]), _ptr(counts), _ptr(out))
    return out


def map_intersects(xys, extents, cum, H, W, B, dtype=np.float32):
    xys, extents, cum = _arr(xys, dtype), _arr(extents, dtype), _arr(cum, np.int32)
    n = xys.shape[0]
    M = int(cum[-1]) if n else 0
    tbx, tby = tile_bounds(H, W, B)
    isect = np.zeros((M,), np.int64)
    gids = np.zeros((M,), np.int32)
    getattr(lib(), "orc_map_intersects_" + _sfx(dtype))(
        ctypes.c_int(n), _ptr(xys), _ptr(extents), _ptr(cum), ctypes.c_int(tbx),
        ctypes.c_int(tby), ctypes.c_int(B), _ptr(isect), _ptr(gids))
    return isect, gids


def sort_by_tile(isect, gids, T):
    isect, gids = _arr(isect, np.int64), _arr(gids, np.int32)
    M = isect.shape[0]
    isect_s = np.zeros_like(isect)
    gid_s = np.zeros_like(gids)
    rc = lib().orc_sort_by_tile(ctypes.c_int(M), _ptr(isect), _ptr(gids), ctypes.c_int(T),
                                _ptr(isect_s), _ptr(gid_s))
    if rc != 0:
        raise ValueError(f"orc_sort_by_tile failed ({rc})")
    return isect_s, gid_s


def tile_bins(isect_sorted, T):
    isect_sorted = _arr(isect_sorted, np.int64)
    bins = np.zeros((T, 2), np.int32)
    lib().orc_tile_bins(ctypes.c_int(isect_sorted.shape[0]), _ptr(isect_sorted),
                        ctypes.c_int(T), _ptr(bins))
    return bins


@dataclass
class Binning:
    num_intersects: int
    cum_tiles_hit: np.ndarray
    isect_ids: np.ndarray
    gaussian_ids: np.ndarray
    isect_ids_sorted: np.ndarray
    gaussian_ids_sorted: np.ndarray
    tile_bins: np.ndarray


def bin_and_sort(xys, extents, counts, H, W, B, dtype=np.float32) -> Binning:
    cum = cumsum(counts)
    M = int(cum[-1]) if cum.size else 0
    tbx, tby = tile_bounds(H, W, B)
    isect, gids = map_intersects(xys, extents, cum, H, W, B, dtype)
    isect_s, gid_s = sort_by_tile(isect, gids, tbx * tby)
    bins = tile_bins(isect_s, tbx * tby)
    return Binning(M, cum, isect, gids, isect_s, gid_s, bins)


# ----------------------------------------------------------------- raster
def raster_fwd(H, W, B, binning: Binning, xys, conics, colors, opac=None, grad_aware=False,
               dtype=np.float32):
    """rasterize_gaussians forward incl. the M < 1 branch (rasterize.py:80-90)."""
    P = H * W
    if binning.num_intersects < 1:
        img = np.ones((H, W, 3), dtype)
        z3 = np.zeros((H, W, 3), dtype)
        return dict(img=img, wsum=np.zeros((H, W), dtype), dx=z3, dy=z3.copy(), dxy=z3.copy(),
                    final_idx=np.zeros((H, W), np.int32))
    xys, conics, colors, opac = (_arr(xys, dtype), _arr(conics, dtype), _arr(colors, dtype),
                                 _arr(opac, dtype))
    img = np.zeros((P, 3), dtype)
    wsum = np.zeros((P,), dtype)
    dx = np.zeros((P, 3), dtype) if grad_aware else None
    dy = np.zeros((P, 3), dtype) if grad_aware else None
    dxy = np.zeros((P, 3), dtype) if grad_aware else None
    fin = np.zeros((P,), np.int32)
    getattr(lib(), "orc_raster_fwd_" + _sfx(dtype))(
        ctypes.c_int(H), ctypes.c_int(W), ctypes.c_int(B),
        _ptr(np.ascontiguousarray(binning.gaussian_ids_sorted, np.int32)),
        _ptr(np.ascontiguousarray(binning.tile_bins, np.int32)),
        _ptr(xys), _ptr(conics), _ptr(colors), _ptr(opac), ctypes.c_int(int(grad_aware)),
        _ptr(img), _ptr(wsum), _ptr(dx), _ptr(dy), _ptr(dxy), _ptr(fin))
    out = dict(img=img.reshape(H, W, 3), wsum=wsum.reshape(H, W), final_idx=fin.reshape(H, W),
               dx=None, dy=None, dxy=None)
    if grad_aware:
        out.update(dx=dx.reshape(H, W, 3), dy=dy.reshape(H, W, 3), dxy=dxy.reshape(H, W, 3))
    return out


def raster_bwd(H, W, B, binning: Binning, xys, conics, colors, opac, final_idx, v_img, v_wsum,
               v_dx=None, v_dy=None, v_dxy=None, clamp=None, dtype=np.float32):
    """rasterize backward incl. the M < 1 branch (rasterize.py:156-161).
    clamp defaults to the reference's: 0.99 (sum kernel), 0.999 (gradient-aware)."""
    grad_aware = v_dx is not None
    if clamp is None:
        clamp = 0.999 if grad_aware else 0.99
    xys = _arr(xys, dtype)
    N = xys.shape[0]
    v_xy = np.zeros((N, 2), dtype)
    v_abs = np.zeros((N, 2), dtype)
    v_con = np.zeros((N, 3), dtype)
    v_rgb = np.zeros((N, 3), dtype)
    v_op = np.zeros((N,), dtype) if opac is not None else None
    M = binning.num_intersects
    if M >= 1:
        part = np.zeros((M * 11,), dtype)
        getattr(lib(), "orc_raster_bwd_" + _sfx(dtype))(
            ctypes.c_int(H), ctypes.c_int(W), ctypes.c_int(B), ctypes.c_int(M),
            _ptr(np.ascontiguousarray(binning.gaussian_ids_sorted, np.int32)),
            _ptr(np.ascontiguousarray(binning.tile_bins, np.int32)),
            _ptr(xys), _ptr(_arr(conics, dtype)), _ptr(_arr(colors, dtype)), _ptr(_arr(opac, dtype)),
            _ptr(_arr(final_idx, np.int32)), _ptr(_arr(v_img, dtype)), _ptr(_arr(v_wsum, dtype)),
            _ptr(_arr(v_dx, dtype)), _ptr(_arr(v_dy, dtype)), _ptr(_arr(v_dxy, dtype)),
            _real(dtype)(clamp), _ptr(part), ctypes.c_int(N),
            _ptr(v_xy), _ptr(v_abs), _ptr(v_con), _ptr(v_rgb), _ptr(v_op))
    return dict(v_xy=v_xy, v_xy_abs=v_abs, v_conic=v_con, v_rgb=v_rgb, v_opacity=v_op)


def dense_fwd_f64(H, W, B, xys, extents, counts, conics, colors, opac=None, grad_aware=False):
    f = np.float64
    xys, extents, conics, colors = _arr(xys, f), _arr(extents, f), _arr(conics, f), _arr(colors, f)
    counts, opac = _arr(counts, np.int32), _arr(opac, f)
    P = H * W
    img = np.zeros((P, 3), f)
    wsum = np.zeros((P,), f)
    dx = np.zeros((P, 3), f) if grad_aware else None
    dy = np.zeros((P, 3), f) if grad_aware else None
    dxy = np.zeros((P, 3), f) if grad_aware else None
    lib().orc_dense_fwd_f64(ctypes.c_int(H), ctypes.c_int(W), ctypes.c_int(B),
                            ctypes.c_int(xys.shape[0]), _ptr(xys), _ptr(extents), _ptr(counts),
                            _ptr(conics), _ptr(colors), _ptr(opac), ctypes.c_int(int(grad_aware)),
                            _ptr(img), _ptr(wsum), _ptr(dx), _ptr(dy), _ptr(dxy))
    out = dict(img=img.reshape(H, W, 3), wsum=wsum.reshape(H, W))
    if grad_aware:
        out.update(dx=dx.reshape(H, W, 3), dy=dy.reshape(H, W, 3), dxy=dxy.reshape(H, W, 3))
    return out


# ----------------------------------------------------------------- upscale
def upscale_fwd(f, fx, fy, fxy, dst_h, dst_w, roi=None, mode=0, dtype=np.float32):
    f, fx, fy, fxy = (_arr(a, dtype) for a in (f, fx, fy, fxy))
    h, w, _ = f.shape
    if roi is None:
        roi = (0.0, 0.0, float(w), float(h))
    out = np.zeros((dst_h, dst_w, 3), dtype)
    R = _real(dtype)
    getattr(lib(), "orc_upscale_fwd_" + _sfx(dtype))(
        ctypes.c_int(mode), ctypes.c_int(h), ctypes.c_int(w), ctypes.c_int(dst_h),
        ctypes.c_int(dst_w), R(roi[0]), R(roi[1]), R(roi[2]), R(roi[3]),
        _ptr(f), _ptr(fx), _ptr(fy), _ptr(fxy), _ptr(out))
    return out


def upscale_bwd(g, src_h, src_w, roi=None, mode=0, dtype=np.float32):
    g = _arr(g, dtype)
    dst_h, dst_w, _ = g.shape
    if roi is None:
        roi = (0.0, 0.0, float(src_w), float(src_h))
    outs = [np.zeros((src_h, src_w, 3), dtype) for _ in range(4)]
    R = _real(dtype)
    getattr(lib(), "orc_upscale_bwd_" + _sfx(dtype))(
        ctypes.c_int(mode), ctypes.c_int(src_h), ctypes.c_int(src_w), ctypes.c_int(dst_h),
        ctypes.c_int(dst_w), R(roi[0]), R(roi[1]), R(roi[2]), R(roi[3]),
        _ptr(g), *[_ptr(o) for o in outs])
    return tuple(outs)


# ----------------------------------------------------------------- pipeline
def render(in3, means, colors, opac, H, W, B, chol=True, grad_aware=False, dtype=np.float32):
    """project -> bin -> raster, the forward of gaussianlig.Gaussian2D.forward
    (gaussianlig.py:70-93) / minimal_trainer_upscale.py:124-136."""
    xys, ext, con, cnt = project_fwd(in3, means, opac, H, W, B, chol=chol, dtype=dtype)
    bn = bin_and_sort(xys, ext, cnt, H, W, B, dtype=dtype)
    out = raster_fwd(H, W, B, bn, xys, con, colors, opac, grad_aware=grad_aware, dtype=dtype)
    out.update(xys=xys, extents=ext, conics=con, counts=cnt, binning=bn)
    return out
