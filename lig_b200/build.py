"""Build recipe for the lig_b200 CUDA library (sm_100a only).

Compiles every ``lig_b200/csrc/*.cu`` with nvcc for ``sm_100a`` into
``lig_b200/_build/*.o`` (in parallel, skipping up-to-date objects) and links
``lig_b200/liblig_b200.so``, which ``lig_b200._lib`` loads through ctypes.
Run it as a script (``python lig_b200/build.py``): importing the package
loads the library, which must exist first.

Flags: ``-O3 --use_fast_math`` matches the reference's setup.py
(gsplat2d/setup.py:65-77), which the bit-exact tile counts and alpha-threshold
decisions depend on; ``-lineinfo`` keeps source correlation for ncu.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "liblig_b200.so")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "--use_fast_math", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-I", INCLUDE]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the lig_b200 CUDA library cannot be built")
    return path


def _deps(src: str):
    return [src] + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(INCLUDE, "lig_b200.h")]


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, extra) -> str:
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if _stale(obj, _deps(src)):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if r.stderr.strip():
            sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, extra=()) -> str:
    """Compile (incrementally) and link liblig_b200.so; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, list(extra)), srcs))
    if _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
