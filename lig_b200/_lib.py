"""ctypes binding of liblig_b200.so (the C ABI declared in include/lig_b200.h).

The library is the only compute path of this package: if it is missing or
fails to load, importing lig_b200 raises — there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "liblig_b200.so")

LIG_OK = 0
LIG_ERR_INVALID = 1
LIG_ERR_CAPACITY = 2
LIG_ERR_LAUNCH = 3
LIG_ERR_WORKSPACE = 4
LIG_ERR_TOO_LARGE = 5
LIG_STATIC_MAX_POINTS = 131072
LIG_F32 = 0
LIG_F64 = 1
LIG_STATUS_OVERFLOW = 1
LIG_STATUS_BADBOX = 2

_ERRORS = {
    LIG_ERR_INVALID: "invalid argument",
    LIG_ERR_CAPACITY: "intersection capacity exceeded",
    LIG_ERR_LAUNCH: "CUDA kernel launch failed",
    LIG_ERR_WORKSPACE: "workspace too small",
    LIG_ERR_TOO_LARGE: f"more Gaussians than the allocation-free entry point's fixed scratch "
                       f"holds ({LIG_STATIC_MAX_POINTS})",
}

P = ctypes.c_void_p
I = ctypes.c_int
I64 = ctypes.c_int64
D = ctypes.c_double
SZ = ctypes.c_size_t

# name -> (restype, argtypes), mirroring include/lig_b200.h
SIGNATURES = {
    "lig_abi_version": (I, []),
    "lig_kernel_launches": (I64, []),
    "lig_project_fwd": (I, [I, I, I, P, P, P, I, I, I, P, P, P, P, P]),
    "lig_project_bwd": (I, [I, I, I, P, P, P, I, I, I, P, I64, P, I64, P, P, P]),
    "lig_project_bwd_saved": (I, [I, I, I, P, P, P, P, P, P, P, P]),
    "lig_cov2d_bounds": (I, [I, I, P, P, P, P, P]),
    "lig_cumsum_workspace_bytes": (SZ, [I]),
    "lig_cumsum_tiles": (I, [I, P, P, P, P, SZ, P]),
    "lig_bin_workspace_bytes": (SZ, [I, I, I]),
    "lig_bin": (I, [I, I, P, P, P, P, I, I, I, I, P, SZ, P, P, P, P, P, P, P]),
    "lig_map_intersects": (I, [I, I, I, P, P, P, I, I, I, P, P, P]),
    "lig_tile_bin_edges": (I, [I, P, I, P, P]),
    "lig_raster_workspace_bytes": (SZ, [I, I]),
    "lig_raster_fwd": (I, [I, I, I, I, I, P, P, P, P, P, P, P, P, SZ, P, P, P, P, P, P, P]),
    "lig_raster_bwd": (I, [I, I, I, I, I, P, P, P, P, P, P, P, P, P, P, P, P, P, D, P, SZ,
                           P, P, P, P, P, P]),
    "lig_upscale_fwd": (I, [I, I, I, I, I, I, D, D, D, D, P, P, P, P, P, P]),
    "lig_upscale_bwd": (I, [I, I, I, I, I, I, D, D, D, D, P, P, P, P, P, P]),
    "lig_upscale_fwd_nc": (I, [I, I, I, I, I, I, I, D, D, D, D, P, P, P, P, P, P]),
    "lig_upscale_bwd_nc": (I, [I, I, I, I, I, I, I, D, D, D, D, P, P, P, P, P, P]),
    "lig_probe_fp32": (I, [I, I, P, P]),
    "lig_wait_timeouts": (I, []),
    "lig_alpha_cut": (I, [P, P]),
    "lig_raster_fwd_noalloc": (I, [I, I, I, I, P, P, P, P, P, P, P, P, P, P, P]),
    "lig_raster_bwd_l2": (I, [I, I, I, I, I, P, P, P, P, P, P, P, P, P, P, P, D, P, SZ, P, P, P,
                              P, P, P]),
    "lig_l2_workspace_bytes": (SZ, []),
    "lig_l2_clamped_loss": (I, [I, I64, P, P, P, P, SZ, P]),
    "lig_project_fwd_batch": (I, [I, I, P, P, P, I, P, P, P, I, P, P, P, P, P]),
    "lig_project_bwd_batch": (I, [I, I, P, P, P, I, P, P, P, I, P, I64, P, I64, P, P, P]),
    "lig_bin_batch": (I, [I, I, P, P, P, I, P, P, P, P, I, P, SZ, P, P, P, P]),
    "lig_raster_fwd_batch": (I, [I, I, P, P, P, I, P, P, P, P, P, P, P, P, I, P, P, SZ, P, P, P,
                                 P, P, P, P]),
    "lig_raster_bwd_l2_batch": (I, [I, I, P, P, P, I, P, P, P, P, P, P, P, P, P, P, P, P, D, I,
                                    P, P, SZ, P, P, P, P, P, P]),
    "lig_l2_batch_workspace_bytes": (SZ, [I]),
    "lig_l2_clamped_loss_batch": (I, [I, I, P, P, P, P, P, P, P, SZ, P]),
    "lig_l2_tile_partials_bytes": (SZ, [I]),
    "lig_raster_fwd_l2": (I, [I, I, I, I, I, P, P, P, P, P, P, P, P, P, SZ, P, P, P, P, P]),
    "lig_raster_fwd_l2_u8": (I, [I, I, I, I, I, P, P, P, P, P, P, P, P, P, SZ, P, P, P, P, P]),
    "lig_raster_bwd_diff": (I, [I, I, I, I, I, P, P, P, P, P, P, P, P, P, P, D, P, SZ, P, P, P,
                                P, P, P]),
    "lig_raster_fwd_l2_batch": (I, [I, I, P, P, P, I, P, P, P, P, P, P, P, P, P, I, P, P, SZ,
                                    P, P, P, P, P, P]),
    "lig_raster_fwd_l2_u8_batch": (I, [I, I, P, P, P, I, P, P, P, P, P, P, P, P, P, I, P, P, SZ,
                                    P, P, P, P, P, P]),
    "lig_raster_bwd_diff_batch": (I, [I, I, P, P, P, I, P, P, P, P, P, P, P, P, P, P, P, D, I,
                                      P, P, SZ, P, P, P, P, P, P]),
    "lig_adam_scratch_bytes": (SZ, []),
    "lig_adam_step": (I, [I64, P, P, P, P, D, D, D, D, P, P, P, P, P]),
    "lig_adam_batch_scratch_bytes": (SZ, [I]),
    "lig_level_residual": (I, [I64, P, P, P, P, P]),
    "lig_level_compose": (I, [I, I, P, I, I, P, P, D, D, I, I, P, P]),
    "lig_project_fwd_view": (I, [I, I, I, P, P, P, I, I, I, D, D, D, D, P, P, P, P, P]),
    "lig_adam_step_batch": (I, [I, P, P, P, P, P, D, D, D, D, P, P, P, P, SZ, P]),
}
LIG_MAX_BATCH = 64


class LigError(RuntimeError):
    """A lig_* entry point returned a non-zero status."""

    def __init__(self, name: str, code: int):
        self.code = code
        super().__init__(f"{name} failed: {_ERRORS.get(code, 'error')} (status {code})")


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"lig_b200 CUDA library not built ({LIB_PATH}); run `python -m lig_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def call(name: str, *args) -> None:
    rc = getattr(lib, name)(*args)
    if rc != LIG_OK:
        if rc == LIG_ERR_INVALID:
            raise ValueError(f"{name}: invalid argument")
        raise LigError(name, rc)
