"""Batched uneven fit: one batched iteration over 64 images vs the per-image
loop of the same kernels (and of the reference kernels).

Workload: lig_b200.batch.uneven_batch — 64 seeded images, heights
log-uniform in [256, 4096], aspect U[0.5, 2], targets rendered from seeded
teacher Gaussians (20000 per 512^2) plus N(0, 0.02) noise; each image fitted
with min(0.2 H W, 1M) Gaussians (fp32, L2 on the clamped render, Adam).

Prints one JSON line: the autotuner's table (tile size x tile walk), the
batched throughput (images x iterations per second, CUDA graph replays),
three per-image loops — the plain drop-in API (gsplat2d project + rasterize,
clamp + F.mse_loss under autograd, torch Adam: what LIG's own training code
does per image), this library's CUDA-graph engine (LevelFit, fused loss,
one image after another) and the reference kernels — and the kernel time
per stage of the batched iteration next to the same kernels summed over the
per-image graph loop (eager runs, CUDA events): where that sum is close to
the batched time, batching can only remove launch gaps and tails.

    python tests/perf_batched.py [--images 64] [--iters 20] [--quality-iters 0]
"""
import argparse
import json
import os
import sys
import time

import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from lig_b200 import ops, synthetic  # noqa: E402
from lig_b200.batch import BatchedFit, autotune, uneven_batch  # noqa: E402
from lig_b200.fit import LevelFit  # noqa: E402

DIAG = (0.5, 4.0)


def _events_s(fn, iters):
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(iters):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / 1e3 / iters


def _kernel_ms(items, reps=3):
    """Per entry point: milliseconds per iteration of eager runs of the
    iteration's kernels, summed over (BatchedFit, target) items."""
    tot = {}
    for fit, target in items:
        fit._enqueue_step(target)
        torch.cuda.synchronize()
        with ops.KernelTimer() as kt:
            for _ in range(reps):
                fit._enqueue_step(target)
        for name, (_, ms) in kt.summary().items():
            tot[name] = tot.get(name, 0.0) + ms / reps
    tot["total"] = sum(tot.values())
    return {k: round(v, 3) for k, v in sorted(tot.items(), key=lambda kv: -kv[1])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--images", type=int, default=64)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--tune-iters", type=int, default=3)
    ap.add_argument("--loop-iters", type=int, default=20)
    ap.add_argument("--api-loop-iters", type=int, default=5)
    ap.add_argument("--ref-loop-iters", type=int, default=5)
    ap.add_argument("--size-scale", type=float, default=1.0)
    ap.add_argument("--blocks", default="8,16,32")
    ap.add_argument("--quality-iters", type=int, default=0,
                    help="also fit this many iterations and report per-image PSNR")
    a = ap.parse_args()
    t0 = time.time()
    targets, counts = uneven_batch(n_img=a.images, size_scale=a.size_scale)
    shapes = [tuple(t.shape[:2]) for t in targets]
    init = []
    for i, ((h, w), c) in enumerate(zip(shapes, counts)):
        init.append(tuple(x.cuda() for x in synthetic.gaussians(c, h, w, diag=DIAG,
                                                                seed=3000 + i)))
    out = {"workload": "batched uneven fit", "images": a.images,
           "pixels": sum(h * w for h, w in shapes), "gaussians": sum(counts),
           "setup_s": round(time.time() - t0, 1)}
    blocks = tuple(int(b) for b in a.blocks.split(","))
    tune = autotune(targets, counts, blocks=blocks, walks=(False, True), iters=a.tune_iters,
                    init=init)
    out["autotune"] = tune["table"]
    out["chosen"] = {"block": tune["block"], "persistent": tune["persistent"]}
    torch.cuda.empty_cache()

    fit = BatchedFit(targets, counts, block=tune["block"], persistent=tune["persistent"],
                     init=init)
    for _ in range(3):
        fit.step()
    s_batch = fit.time_iters(a.iters)
    out["batched"] = {"s_per_iter": s_batch, "image_iters_per_s": a.images / s_batch,
                      "capacity": fit.capacity, "skipped": fit.stats.skipped}
    if a.quality_iters:
        fit.fit(a.quality_iters)
        p = fit.psnr()
        out["batched"]["psnr_mean"] = sum(p) / len(p)
    out["batched"]["kernel_ms"] = _kernel_ms([(fit, None)])
    del fit
    torch.cuda.empty_cache()

    # per-image loop, this library's kernels (16x16 tiles, as the drop-in API)
    fits = []
    for i, ((h, w), c) in enumerate(zip(shapes, counts)):
        f = LevelFit(c, h, w, lr=1e-3, block=16, diag=DIAG, seed=3000 + i)
        fits.append(f)

    def loop_round():
        for f, t in zip(fits, targets):
            f.step(t)

    loop_round()
    s_loop = _events_s(loop_round, a.loop_iters)
    out["loop_lig"] = {"s_per_iter": s_loop, "image_iters_per_s": a.images / s_loop,
                       "kernel_ms": _kernel_ms([(f._batch, t.reshape(-1, 3))
                                                for f, t in zip(fits, targets)])}
    out["speedup_vs_loop"] = s_loop / s_batch
    del fits
    torch.cuda.empty_cache()

    # per-image loop, the plain drop-in API under autograd (LIG's own loop)
    if a.api_loop_iters:
        afits = [LevelFit(c, h, w, lr=1e-3, block=16, diag=DIAG, seed=3000 + i,
                          engine="autograd", fused_loss=False)
                 for i, ((h, w), c) in enumerate(zip(shapes, counts))]

        def api_round():
            for f, t in zip(afits, targets):
                f.step(t)

        api_round()
        s_api = _events_s(api_round, a.api_loop_iters)
        out["loop_api"] = {"s_per_iter": s_api, "image_iters_per_s": a.images / s_api}
        out["speedup_vs_api_loop"] = s_api / s_batch
        del afits
        torch.cuda.empty_cache()

    # per-image loop, the reference kernels (when built)
    if a.ref_loop_iters:
        try:
            from _reffit import RefFit
            from oracle import ref
            ref.STRICT_SYNC = False
            rfits = [RefFit(c, h, w, DIAG, seed=3000 + i)
                     for i, ((h, w), c) in enumerate(zip(shapes, counts))]

            def ref_round():
                for f, t in zip(rfits, targets):
                    f.step(t)

            ref_round()
            s_ref = _events_s(ref_round, a.ref_loop_iters)
            out["loop_ref"] = {"s_per_iter": s_ref, "image_iters_per_s": a.images / s_ref}
            out["speedup_vs_ref_loop"] = s_ref / s_batch
        except (ImportError, OSError, RuntimeError) as e:  # reference kernels not built
            out["loop_ref"] = {"unavailable": str(e)}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
