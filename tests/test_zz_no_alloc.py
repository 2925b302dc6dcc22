"""The allocation-free rasterizer entry point, lig_raster_fwd_noalloc.

It exists for callers that cannot allocate device memory when they render
(e.g. a plugin inside a framework that has reserved nearly all GPU memory for
its own pool): its scratch is a fixed array inside the library.  This test
calls it through the C ABI and checks it against the regular workspace entry
point, lig_raster_fwd, on two calls in a row (different scenes, so the
second call runs on scratch the first one left behind), at exactly
LIG_STATIC_MAX_POINTS Gaussians (the array full), that repeated calls leave
the device's free memory unchanged, and that an oversized request is refused
before any GPU work.  Collected last on purpose.
"""
import ctypes

import pytest
import torch

from lig_b200 import _lib, ops
from tests._scene import scene

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5
P = ctypes.c_void_p


def _p(t):
    return None if t is None else P(t.data_ptr())


def _binned_scene(n, H, W, B, seed, opac):
    means, L, colors, op = scene(n, H, W, diag=(0.5, 4.0), seed=seed, opac=opac)
    xys, ext, con, cnt = ops.project_fwd(L, means, op, H, W, B, True)
    b = ops.bin_gaussians(xys, ext, cnt, H, W, B)
    return xys, con, colors, op, b


def _noalloc(H, W, B, xys, con, colors, op, b):
    img = torch.empty(H, W, 3, device="cuda")
    wsum = torch.empty(H, W, device="cuda")
    fin = torch.empty(H, W, dtype=torch.int32, device="cuda")
    rc = _lib.lib.lig_raster_fwd_noalloc(
        H, W, B, xys.shape[0], _p(b.gaussian_ids_sorted), _p(b.tile_bins), _p(b.total),
        _p(xys), _p(con), _p(colors), _p(op), _p(img), _p(wsum), _p(fin),
        P(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.LIG_OK
    return img, wsum, fin


def test_noalloc_matches_workspace_entry_point_on_consecutive_calls():
    cases = [(4000, 200, 240, 16, 0, (0.05, 1.0)), (1500, 97, 131, 8, 1, None)]
    for n, H, W, B, seed, opac in cases:
        xys, con, colors, op, b = _binned_scene(n, H, W, B, seed, opac)
        img, wsum, fin = _noalloc(H, W, B, xys, con, colors, op, b)
        r_img, r_wsum, _, _, _, r_fin = ops.raster_fwd(H, W, B, b.gaussian_ids_sorted,
                                                       b.tile_bins, b.total, xys, con, colors,
                                                       op, False)
        torch.cuda.synchronize()
        assert torch.equal(fin, r_fin)
        assert (img - r_img).abs().max().item() <= IMG_TOL
        assert (wsum - r_wsum).abs().max().item() <= IMG_TOL


def test_noalloc_rejects_more_points_than_its_scratch():
    n = _lib.LIG_STATIC_MAX_POINTS + 1
    rc = _lib.lib.lig_raster_fwd_noalloc(16, 16, 16, n, None, None, None, None, None, None,
                                         None, None, None, None, None)
    assert rc == _lib.LIG_ERR_TOO_LARGE


def _check_against_workspace_entry(n, H, W, B, seed, opac):
    xys, con, colors, op, b = _binned_scene(n, H, W, B, seed, opac)
    img, wsum, fin = _noalloc(H, W, B, xys, con, colors, op, b)
    r_img, r_wsum, _, _, _, r_fin = ops.raster_fwd(H, W, B, b.gaussian_ids_sorted, b.tile_bins,
                                                   b.total, xys, con, colors, op, False)
    torch.cuda.synchronize()
    assert torch.equal(fin, r_fin)
    assert (img - r_img).abs().max().item() <= IMG_TOL
    assert (wsum - r_wsum).abs().max().item() <= IMG_TOL


def test_noalloc_at_its_maximum_size():
    # every record slot of the array in use
    _check_against_workspace_entry(_lib.LIG_STATIC_MAX_POINTS, 384, 512, 16, 2, (0.05, 1.0))


def test_noalloc_calls_allocate_no_device_memory():
    H, W, B = 160, 192, 16
    xys, con, colors, op, b = _binned_scene(3000, H, W, B, 3, None)
    img = torch.empty(H, W, 3, device="cuda")
    wsum = torch.empty(H, W, device="cuda")
    fin = torch.empty(H, W, dtype=torch.int32, device="cuda")
    stream = P(torch.cuda.current_stream().cuda_stream)
    args = (H, W, B, xys.shape[0], _p(b.gaussian_ids_sorted), _p(b.tile_bins), _p(b.total),
            _p(xys), _p(con), _p(colors), _p(op), _p(img), _p(wsum), _p(fin), stream)
    assert _lib.lib.lig_raster_fwd_noalloc(*args) == _lib.LIG_OK   # warm-up (address lookup)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert _lib.lib.lig_raster_fwd_noalloc(*args) == _lib.LIG_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
