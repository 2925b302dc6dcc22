"""LIG's caller modules resolve on this library (no GPU needed).

The reference's gaussianlig.py, train.py and minimal_trainer_upscale.py are
imported (bytecode of the unmodified files, tests/_callers.py) after
lig_b200.install_gsplat2d(): every `from gsplat2d... import ...` they make
must bind to this library.  Where the reference tree is present, the bytecode
is checked to be of the unmodified sources (PEP 552 source hashes).
"""
import importlib.util
import os

import pytest

import _callers

pytestmark = pytest.mark.skipif(not _callers.available(),
                                reason="reference caller bytecode not built (make -C oracle ref)")

REF = os.environ.get("LIG_REFERENCE", "/root/reference")


def test_callers_bind_to_this_library():
    with _callers.bound("lig"):
        import gaussianlig
        import minimal_trainer_upscale as mtu
        import train  # noqa: F401
        assert gaussianlig.project_gaussians.__module__ == "lig_b200.gsplat2d.project_gaussians"
        assert gaussianlig.rasterize_gaussians.__module__ == "lig_b200.gsplat2d.rasterize"
        assert mtu.project_gaussians_cholesky.__module__ == \
            "lig_b200.gsplat2d.project_gaussians_cholesky"
        assert mtu.gradient_aware_upscale.__module__ == "lig_b200.gsplat2d.upscale"
        assert mtu.torch_gradient_aware_upscale.__module__ == "lig_b200.upscaler_torch"


def test_checker_binds_to_the_reference_package():
    with _callers.bound("ref"):
        import gaussianlig
        import gsplat2d
        assert "_ref" in _callers.module_origin("gsplat2d")
        assert gaussianlig.rasterize_gaussians is gsplat2d.rasterize_gaussians
    import sys
    assert "gsplat2d" not in sys.modules and "gaussianlig" not in sys.modules


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
def test_bytecode_is_of_the_unmodified_reference_files():
    import sys
    sys.path.insert(0, os.path.join(_callers.ROOT, "oracle"))
    try:
        import compile_callers
    finally:
        sys.path.pop(0)
    import zipfile
    n = 0
    for src, archive, member in compile_callers.sources(REF):
        with zipfile.ZipFile(os.path.join(_callers.PYDIR, archive)) as z:
            header = z.read(member)[:16]
        flags = int.from_bytes(header[4:8], "little")
        assert flags & 1, member                    # hash-based pyc
        with open(src, "rb") as f:
            assert header[8:16] == importlib.util.source_hash(f.read()), member
        n += 1
    assert n == 14
