"""Compile the reference's Python callers and its gsplat2d package to bytecode
(TEST INFRASTRUCTURE ONLY).

    python oracle/compile_callers.py <reference root> <output dir>

The reference's own driver files — gaussianlig.py, train.py,
minimal_trainer_upscale.py and the modules they import (utils.py,
optimizer.py, upscaler_torch.py) — and its gsplat2d Python package
(gsplat2d/gsplat2d/*.py, cuda/__init__.py) are compiled unchanged, where they
lie, into sourceless .pyc files stored in two zip archives (Python imports
sourceless bytecode from a zip on sys.path through zipimport; an archive
travels where loose .pyc files, treated as caches, may not):

    <out>/callers.zip: <module>.pyc     the LIG driver modules
    <out>/pkg.zip: gsplat2d/...         the reference gsplat2d package

The GPU tests import these to run LIG's unmodified training code against
this library (through lig_b200.install_gsplat2d) and, as the checker, against
the reference's own Python glue on the reference's kernels
(oracle/_ref/libgsplat2d_ref.so through oracle/ref_C.py).  The reference tree
is not present where the GPU tests run; the bytecode travels with the other
oracle/_ref build outputs and is never committed.

Each .pyc uses the unchecked-hash form (PEP 552): it records the SipHash of
the source it was compiled from, which tests/test_cpu_callers.py compares
with the reference files to show the bytecode is of the unmodified sources.
cuda/_backend.py (the reference's JIT build of its extension) is left out:
the checker supplies `_C` itself.
"""
from __future__ import annotations

import os
import py_compile
import sys
import tempfile
import zipfile

CALLERS = ("gaussianlig", "utils", "optimizer", "train", "minimal_trainer_upscale",
           "upscaler_torch")
PACKAGE = ("__init__", "project_gaussians", "project_gaussians_cholesky", "rasterize", "upscale",
           "utils", "version", "cuda/__init__")


def sources(ref: str):
    """(source path, archive name, member name) triples."""
    for m in CALLERS:
        yield os.path.join(ref, m + ".py"), "callers.zip", m + ".pyc"
    for m in PACKAGE:
        yield (os.path.join(ref, "gsplat2d", "gsplat2d", m + ".py"), "pkg.zip",
               "gsplat2d/" + m + ".pyc")


def main(ref: str, out: str) -> None:
    os.makedirs(out, exist_ok=True)
    members = {}
    with tempfile.TemporaryDirectory() as tmp:
        for src, archive, member in sources(ref):
            dst = os.path.join(tmp, archive, member)
            os.makedirs(os.path.dirname(dst), exist_ok=True)
            py_compile.compile(src, cfile=dst, dfile=os.path.relpath(src, ref), doraise=True,
                               invalidation_mode=py_compile.PycInvalidationMode.UNCHECKED_HASH)
            members.setdefault(archive, []).append((dst, member))
        for archive, files in members.items():
            path = os.path.join(out, archive)
            with zipfile.ZipFile(path + ".tmp", "w", zipfile.ZIP_STORED) as z:
                for dst, member in files:
                    z.write(dst, member)
            os.replace(path + ".tmp", path)


if __name__ == "__main__":
    if len(sys.argv) != 3:
        sys.exit(__doc__)
    main(sys.argv[1], sys.argv[2])
