"""LIG's own caller modules, unmodified, bound to one gsplat2d implementation.

oracle/compile_callers.py compiles the reference's gaussianlig.py, train.py,
minimal_trainer_upscale.py (and utils.py, optimizer.py, upscaler_torch.py
they import) and its gsplat2d package to bytecode in two zip archives under
oracle/_ref/py (imported through zipimport).
`bound(arm)` imports those modules with `gsplat2d` / `upscaler_torch`
resolving to

  "lig": this library, through lig_b200.install_gsplat2d() — the drop-in
         under test;
  "ref": the reference's own gsplat2d package (its rasterize.py, utils.py,
         project_gaussians*.py, upscale.py) on the reference's kernels
         (oracle/ref_C.py as its `_C`), and the reference's upscaler_torch —
         the checker.

Each arm gets a fresh set of these modules and the previous sys.modules /
sys.path state is restored on exit, so both arms run in one process.
`pytorch_msssim` (an evaluation-only metric the reference imports, absent
here) is replaced by a stub whose ms_ssim/ssim return 1.0; no code path
under test uses it for a loss.  TorchScript is off inside the context:
`@torch.jit.script` needs the source text, which bytecode does not carry, so
the reference's upscaler_torch functions run as the eager Python functions
they script (the same torch operations).
"""
from __future__ import annotations

import contextlib
import os
import sys
import types

import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PYDIR = os.path.join(ROOT, "oracle", "_ref", "py")
CALLERS = os.path.join(PYDIR, "callers.zip")
REF_PKG = os.path.join(PYDIR, "pkg.zip")

_OWNED = ("gaussianlig", "utils", "optimizer", "train", "minimal_trainer_upscale",
          "upscaler_torch", "pytorch_msssim", "gsplat2d")


def _has(archive: str, member: str) -> bool:
    import zipfile
    try:
        with zipfile.ZipFile(archive) as z:
            return member in z.namelist()
    except (OSError, zipfile.BadZipFile):
        return False


def available() -> bool:
    from oracle import ref
    return (_has(CALLERS, "gaussianlig.pyc") and _has(REF_PKG, "gsplat2d/__init__.pyc")
            and ref.available())


def _owned(name: str) -> bool:
    return any(name == o or name.startswith(o + ".") for o in _OWNED)


def _msssim_stub() -> types.ModuleType:
    m = types.ModuleType("pytorch_msssim")

    def _one(x, *a, **k):
        return torch.ones((), device=x.device)

    m.ms_ssim = m.ssim = _one
    return m


@contextlib.contextmanager
def bound(arm: str):
    """Context in which `import gaussianlig` etc. load LIG's unmodified
    modules on the chosen gsplat2d ("lig" or "ref")."""
    if arm not in ("lig", "ref"):
        raise ValueError(arm)
    saved = {k: v for k, v in sys.modules.items() if _owned(k)}
    for k in saved:
        del sys.modules[k]
    path = list(sys.path)
    import torch.jit._state as jit_state
    jit_enabled = jit_state._enabled.enabled
    jit_state._enabled.enabled = False
    try:
        sys.modules["pytorch_msssim"] = _msssim_stub()
        if arm == "lig":
            import lig_b200
            lig_b200.install_gsplat2d()
        else:
            from oracle import ref_C
            sys.path.insert(0, REF_PKG)
            backend = types.ModuleType("gsplat2d.cuda._backend")
            backend._C = ref_C
            sys.modules["gsplat2d.cuda._backend"] = backend
        sys.path.insert(0, CALLERS)
        yield
    finally:
        for k in [k for k in sys.modules if _owned(k)]:
            del sys.modules[k]
        sys.modules.update(saved)
        sys.path[:] = path
        jit_state._enabled.enabled = jit_enabled


def module_origin(name: str) -> str:
    """File a loaded module came from (to show which implementation ran)."""
    return getattr(sys.modules[name], "__file__", "") or ""
