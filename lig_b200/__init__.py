"""lig_b200 — B200-native (sm_100a) gsplat2d hot path for LIG.

The compute path is the CUDA library liblig_b200.so (C ABI in
include/lig_b200.h), loaded at import; there is no CPU fallback.

    import lig_b200
    lig_b200.install_gsplat2d()      # `import gsplat2d` / `upscaler_torch` now resolve here
"""
import importlib
import sys

from . import _lib  # noqa: F401  (loads liblig_b200.so; raises if missing)
from . import ops  # noqa: F401
from . import gsplat2d  # noqa: F401
from . import upscaler_torch  # noqa: F401

__all__ = ["ops", "gsplat2d", "upscaler_torch", "install_gsplat2d"]


def install_gsplat2d() -> None:
    """Register this package under the reference's module names so that LIG's
    own code (gaussianlig.py, train.py, minimal_trainer_upscale.py) imports it
    unchanged: gsplat2d, gsplat2d.<submodule>, gsplat2d.cuda, upscaler_torch."""
    # submodules by module path: the package attributes `project_gaussians` etc.
    # are the functions (as in the reference's __init__), not the modules
    mods = {"gsplat2d": gsplat2d, "upscaler_torch": upscaler_torch}
    for sub in ("cuda", "project_gaussians", "project_gaussians_cholesky", "rasterize",
                "upscale", "utils", "version"):
        mods["gsplat2d." + sub] = importlib.import_module(f"{__name__}.gsplat2d.{sub}")
    sys.modules.update(mods)
