"""Fit speed and PSNR: this library vs the reference's own CUDA kernels.

Both sides run the same LIG level fit (same seeded init, target and Adam
settings): render -> clamp -> L2 -> backward -> Adam.  The reference side is
its kernels (oracle/_ref, compiled from the reference sources) with its torch
glue restated in oracle/ref.py — cumsum + .item(), torch.sort + gather — and
the L2/clamp gradient computed as autograd would; only the reference's own
host synchronisation remains.  Prints one JSON line per configuration.

    python tests/perf_vs_reference.py [--configs c0,c1l2] [--iters N]
"""
import argparse
import json
import os
import sys

import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from lig_b200 import synthetic  # noqa: E402
from lig_b200.fit import LevelFit, downsample, fit_two_level, make_target, psnr  # noqa: E402
from oracle import ref  # noqa: E402
from _reffit import RefFit, ref_two_level  # noqa: E402

CONFIGS = {
    # name: (H=W, fit N, teacher N, diag, noise, noise std, timed iters, psnr iters)
    "c0": (512, 50_000, 20_000, (0.5, 4.0), "white", 0.02, 200, 1000),
    "c1l2": (8192, 2_000_000, 2_000_000, (0.5, 6.0), "spectral", 0.03, 20, 100),
    "c3": (4096, 1_000_000, 1_000_000, (0.5, 8.0), "white", 0.02, 20, 0),
}


def timed(fit, target, iters):
    for _ in range(3):
        fit.step(target)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(iters):
        fit.step(target)
    e.record()
    torch.cuda.synchronize()
    return iters / (s.elapsed_time(e) / 1e3)


def run_two_level(iters, rgb_init="uniform", lr=1e-3):
    """Config 1 end to end: 8192^2 target (2M teacher, diag U[0.5,6], 1/f^2
    noise std 0.03), level 1 = 1M Gaussians on the 4x bicubic-downsampled
    image, gradient-aware upscale, level 2 = 2M Gaussians on the residual.
    rgb_init "uniform" is the configuration's colour draw, "zeros" the
    reference's own initialisation (gaussianlig.py:57)."""
    gt = make_target(8192, 8192, 2_000_000, (0.5, 6.0), noise="spectral", noise_std=0.03)
    ref.STRICT_SYNC = False
    mine = fit_two_level(gt, 1_000_000, 2_000_000, iters, lr=lr, rgb_init=rgb_init)
    torch.cuda.empty_cache()
    theirs = ref_two_level(gt, 1_000_000, 2_000_000, iters, lr=lr, rgb_init=rgb_init)
    out = {"config": "c1_two_level", "iters_per_level": iters, "rgb_init": rgb_init, "lr": lr,
           "lig": {"psnr": mine.psnr, "level_psnr": mine.level_psnr, "up_psnr": mine.up_psnr,
                   "iters_per_s": mine.iters_per_s},
           "ref": theirs, "psnr_delta_db": mine.psnr - theirs["psnr"],
           "speedup_per_level": [a / b for a, b in zip(mine.iters_per_s,
                                                       theirs["iters_per_s"])]}
    print(json.dumps(out), flush=True)


def run(name):
    size, n, nt, diag, noise, std, iters, piters = CONFIGS[name]
    target = make_target(size, size, nt, diag, noise=noise, noise_std=std)
    ref.STRICT_SYNC = False
    out = {"config": name, "size": size, "points": n}
    mine = LevelFit(n, size, size, lr=1e-3, diag=diag)
    out["lig_iters_per_s"] = timed(mine, target, iters)
    del mine
    theirs = RefFit(n, size, size, diag)
    out["ref_iters_per_s"] = timed(theirs, target, iters)
    del theirs
    out["speedup"] = out["lig_iters_per_s"] / out["ref_iters_per_s"]
    if name == "c0":  # the C restatement (oracle/, OpenMP) on this host's cores
        import bench
        v, cores, _, _, _ = bench.cpu_band_sample(size, n, 5.0, 3, diag=diag)
        out.update(cpu_iters_per_s=v, cpu_cores=cores)
    if piters:
        mine, theirs = LevelFit(n, size, size, lr=1e-3, diag=diag), RefFit(n, size, size, diag)
        for _ in range(piters):
            mine.step(target)
            theirs.step(target)
        with torch.no_grad():
            pm = psnr(torch.clamp(mine.render()[0], 0, 1), target)
            pr = psnr(torch.clamp(theirs.render()["img"], 0, 1), target)
        out.update(psnr_iters=piters, lig_psnr=pm, ref_psnr=pr, psnr_delta_db=pm - pr)
    print(json.dumps(out), flush=True)
    torch.cuda.empty_cache()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", default="c0,c1l2")
    ap.add_argument("--two-level-iters", type=int, default=0,
                    help="also run config 1 end to end with this many iterations per level")
    ap.add_argument("--rgb-init", default="uniform,zeros",
                    help="colour initialisations of the two-level runs")
    ap.add_argument("--two-level-lr", default="0.001,0.01",
                    help="Adam learning rate per colour initialisation")
    a = ap.parse_args()
    for c in [c for c in a.configs.split(",") if c]:
        run(c)
    if a.two_level_iters:
        lrs = [float(x) for x in a.two_level_lr.split(",")]
        for init, lr in zip(a.rgb_init.split(","), lrs):
            run_two_level(a.two_level_iters, init, lr)


if __name__ == "__main__":
    main()
