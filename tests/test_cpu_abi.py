"""The C-ABI library (no GPU needed): it loads, exports every entry point that
include/lig_b200.h declares with the argument count the ctypes layer binds,
answers workspace queries, and rejects invalid arguments before touching the
GPU."""
import ctypes
import os
import re

import pytest

from lig_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lig_b200.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(?:int|size_t|int64_t)\s+(lig_\w+)\s*\(([^)]*)\)\s*;", src):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = len(args)
    return out


def test_header_declares_entry_points():
    d = _declared()
    assert len(d) >= 17
    for name in ("lig_project_fwd", "lig_bin", "lig_raster_fwd", "lig_raster_bwd",
                 "lig_upscale_fwd", "lig_upscale_bwd"):
        assert name in d


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for name, nargs in _declared().items():
        assert hasattr(lib, name), f"{name} not exported"
        assert name in _lib.SIGNATURES, f"{name} has no ctypes binding"
        assert len(_lib.SIGNATURES[name][1]) == nargs, f"{name}: arity mismatch"


def test_abi_version_and_workspace_queries():
    L = _lib.lib
    assert L.lig_abi_version() == 1
    assert L.lig_cumsum_workspace_bytes(1) >= 8
    assert L.lig_cumsum_workspace_bytes(2_000_000) >= 4 * (2_000_000 // 4096)
    small = L.lig_bin_workspace_bytes(100, 1000, 16)
    big = L.lig_bin_workspace_bytes(2_000_000, 13_000_000, 262144)
    assert 0 < small < big
    assert big >= 2 * 4 * 262144  # per-tile counts and cursors
    # packed 48/96-byte records + packed [N][12] gradients
    assert L.lig_raster_workspace_bytes(_lib.LIG_F32, 10) >= 10 * 48 + 10 * 48
    assert L.lig_raster_workspace_bytes(_lib.LIG_F64, 10) >= 10 * 96 + 10 * 96
    assert L.lig_l2_workspace_bytes() > 0


def test_invalid_arguments_rejected_without_gpu():
    L = _lib.lib
    # negative point count, bad dtype, bad block width: rejected on the host
    assert L.lig_project_fwd(0, -1, 1, None, None, None, 8, 8, 16, None, None, None, None,
                             None) == _lib.LIG_ERR_INVALID
    assert L.lig_project_fwd(7, 0, 1, None, None, None, 8, 8, 16, None, None, None, None,
                             None) == _lib.LIG_ERR_INVALID
    assert L.lig_raster_fwd(0, 8, 8, 64, 0, None, None, None, None, None, None, None, None, 0,
                            None, None, None, None, None, None, None) == _lib.LIG_ERR_INVALID
    assert L.lig_upscale_fwd(0, 2, 4, 4, 8, 8, 0.0, 0.0, 4.0, 4.0, None, None, None, None, None,
                             None) == _lib.LIG_ERR_INVALID
    assert L.lig_cumsum_tiles(-1, None, None, None, None, 0, None) == _lib.LIG_ERR_INVALID


def test_call_maps_status_to_exceptions():
    with pytest.raises(ValueError):
        _lib.call("lig_cumsum_tiles", -1, None, None, None, None, 0, None)
    e = _lib.LigError("lig_bin", _lib.LIG_ERR_WORKSPACE)
    assert "workspace" in str(e) and e.code == _lib.LIG_ERR_WORKSPACE
