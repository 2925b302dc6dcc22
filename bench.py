"""Benchmark: LIG fit iterations/s at 8192^2 (level 2 of the two-level fit).

Workload (one "step"): one fit iteration of LIG's full-resolution level —
2M Cholesky Gaussians (means U[0,8192)^2, diagonals U[0.5,6], off-diagonal
N(0,0.5), colours U(0,1)) on an 8192x8192 RGB target (a render of 2M
seeded teacher Gaussians plus 1/f^2 noise of std 0.03, clipped and stored as
8-bit RGB, the form of the PNG images LIG's train.py reads and converts with
ToTensor; the loss kernel reads each byte as byte / 255): project ->
bin -> raster forward with the clamped L2 loss fused in -> raster backward
-> projection backward -> Adam, as lig_b200.fit.LevelFit.step runs it (its
CUDA-graph engine: one graph replay per iteration).  Synthetic data stands
in for the DIV2K/STimage images (not available offline).

  value  device-timed iterations/s, target resident in HBM (inputs > L2).
  e2e    same loop through LevelFit.step with the step's input (the 8-bit
         target image) copied host->device from pinned memory every step (double
         buffered on a copy stream, overlapping the previous step) and the
         loss copied back to pinned host memory every step.
  roofline  the dominant kernel's algorithmic rate (reference-defined
         Gaussian-pixel evaluations x FLOP per evaluation) / measured FP32
         FMA peak of this device; per-kernel times come from three eager
         runs of the graph's kernels just before the timed loop.
  cpu_baseline  the C restatement of the reference algorithm (oracle/) on
         this host's cores, on a horizontal band of the same workload.

`--impl reference` times that CPU implementation (the reference has no CPU
path of its own; its GPU kernels are compared in tests/) and prints the
same metric.  Multi-GPU: independent replicas (no data-path collective),
value = total iterations of all ranks / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch
import torch.distributed as dist

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LIG fit iters/s (fwd+bwd) at 8192^2, PSNR-matched; render p50/p99 ms"
H = W = 8192
N_FIT = 2_000_000
N_TEACHER = 2_000_000
DIAG = (0.5, 6.0)
BLOCK = 16
FLOP_PER_EVAL = {"lig_raster_fwd": 20.0, "lig_raster_bwd": 40.0, "lig_raster_bwd_l2": 40.0,
                 "lig_raster_fwd_l2": 20.0, "lig_raster_bwd_diff": 40.0,
                 "lig_raster_fwd_l2_batch": 20.0, "lig_raster_fwd_l2_u8_batch": 20.0,
                 "lig_raster_bwd_diff_batch": 40.0}
# DRAM bytes (read + write) per launch measured by an ncu capture of the same
# kernels on the 2048^2 / 125k-Gaussian step (same density); traffic grows
# with pixels and Gaussians, so a size-S launch is scaled by (S / 2048)^2.
DRAM_BYTES_2048 = {"lig_raster_fwd_l2_u8_batch": 21.7e6 + 15.3e6,
                   "lig_raster_bwd_diff_batch": 63.4e6 + 1.0e6}
CLOCK_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["lig", "reference"], default="lig")
    ap.add_argument("--size", type=int, default=H, help="image side (default 8192)")
    ap.add_argument("--points", type=int, default=None,
                    help="fitted Gaussians (default 2M scaled by (size/8192)^2)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="approximate CPU work per baseline sample")
    return ap.parse_args()


def points_for(args) -> int:
    if args.points is not None:
        return args.points
    return max(1, int(N_FIT * (args.size / H) ** 2))


# ----------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={CLOCK_FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        # wait for the sampler's first line, so that sampling is live when the
        # timed region starts; lines written before it are not counted
        self.n_pre = 0
        t_end = time.time() + 5.0
        while self.proc is not None and time.time() < t_end:
            n = self._count()
            if n > 0:
                self.n_pre = n
                break
            time.sleep(0.02)
        return self

    def _count(self) -> int:
        try:
            with open(self.path) as f:
                return sum(1 for line in f if line.count(",") >= 8)
        except OSError:
            return 0

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        finally:
            os.unlink(self.path)
        if len(rows) > self.n_pre:
            rows = rows[self.n_pre:]  # samples taken during the timed region
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


# ------------------------------------------------------------------ setup
def make_workload(size: int, n: int, device):
    from lig_b200 import synthetic
    from lig_b200.fit import LevelFit, make_target
    n_teacher = max(1, int(N_TEACHER * (size / H) ** 2))
    target = make_target(size, size, n_teacher, DIAG, noise="spectral", noise_std=0.03,
                         device=device, block=BLOCK)
    target = torch.round(target * 255).clamp_(0, 255).to(torch.uint8)  # 8-bit RGB image
    fit = LevelFit(n, size, size, device=device, lr=1e-3, block=BLOCK, diag=DIAG,
                   seed=synthetic.SEED_INIT)
    return target, fit


def workload_name(size: int, n: int) -> str:
    return (f"LIG level-2 fit step, {size}x{size} RGB (8-bit target), {n} Gaussians "
            f"(diag U[0.5,6]), 16x16 tiles, L2 + Adam")


def evaluations(fit) -> tuple[int, int]:
    """(M, E): intersections and reference-defined Gaussian-pixel evaluations
    (sum over tiles of list length x pixels of the tile inside the image)."""
    from lig_b200 import ops
    with torch.no_grad():
        xys, ext, con, cnt = ops.project_fwd(fit.chol, fit.means, None, fit.H, fit.W, fit.block,
                                             True)
        b = ops.bin_gaussians(xys, ext, cnt, fit.H, fit.W, fit.block)
        tbx, tby = ops.tile_bounds(fit.H, fit.W, fit.block)
        lens = (b.tile_bins[:, 1] - b.tile_bins[:, 0]).to(torch.int64)
        tx = torch.arange(tbx * tby, device=lens.device) % tbx
        ty = torch.arange(tbx * tby, device=lens.device) // tbx
        pw = torch.clamp(fit.W - tx * fit.block, max=fit.block)
        ph = torch.clamp(fit.H - ty * fit.block, max=fit.block)
        e = int((lens * pw * ph).sum().item())
    return b.num_intersects, e


# -------------------------------------------------------------- CPU side
def _synthetic_module():
    """lig_b200/synthetic.py (the seeded draws; torch only) loaded by path:
    importing it through the package would load the CUDA library, which the
    CPU reference arm must not touch."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "lig_synthetic_draws", os.path.join(ROOT, "lig_b200", "synthetic.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _adam_np(params, grads, state, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """torch.optim.Adam's update (the GPU step's optimiser) on float32 arrays."""
    state["t"] = state.get("t", 0) + 1
    t = state["t"]
    for i, (p, g) in enumerate(zip(params, grads)):
        m = state.setdefault(("m", i), np.zeros_like(p))
        v = state.setdefault(("v", i), np.zeros_like(p))
        m *= b1
        m += (1 - b1) * g
        v *= b2
        v += (1 - b2) * g * g
        mhat = m / (1 - b1 ** t)
        vhat = v / (1 - b2 ** t)
        p -= (lr * mhat / (np.sqrt(vhat) + eps)).astype(np.float32)


def cpu_band_sample(size, n, target_secs, steps, diag=DIAG):
    """Time the oracle (C restatement, OpenMP) on horizontal bands of the
    workload; returns (iters/s for the full image, cores, description)."""
    from oracle import oracle as O
    synthetic = _synthetic_module()
    cores = os.cpu_count() or 1
    means, chol, colors = synthetic.gaussians(n, size, size, diag=diag, seed=synthetic.SEED_INIT)
    means, chol, colors = means.numpy(), chol.numpy(), colors.numpy()
    rng = np.random.default_rng(0)

    def band_step(rows):
        sel = (means[:, 1] >= -32) & (means[:, 1] < rows + 32)
        m, L, c = means[sel], chol[sel], colors[sel]
        tgt = (rng.integers(0, 256, (rows, size, 3)) / 255).astype(np.float32)
        state = {}
        t0 = time.perf_counter()
        xys, ext, con, cnt = O.project_fwd(L, m, None, rows, size, BLOCK, chol=True)
        bn = O.bin_and_sort(xys, ext, cnt, rows, size, BLOCK)
        out = O.raster_fwd(rows, size, BLOCK, bn, xys, con, c, None)
        img = out["img"]
        v_img = (2.0 / img.size) * (np.clip(img, 0, 1) - tgt) * ((img >= 0) & (img <= 1))
        g = O.raster_bwd(rows, size, BLOCK, bn, xys, con, c, None, out["final_idx"],
                         v_img.astype(np.float32), np.zeros((rows, size), np.float32))
        v_L, v_m = O.project_bwd(ext, L, con, g["v_xy"], g["v_conic"], chol=True)
        _adam_np([c, m, L], [g["v_rgb"], v_m, v_L], state)
        return time.perf_counter() - t0

    probe_rows = max(BLOCK, (size // 64) // BLOCK * BLOCK)
    t_probe = band_step(probe_rows)
    rows = int(min(size, max(BLOCK, probe_rows * target_secs / max(t_probe, 1e-3))))
    rows = max(BLOCK, rows // BLOCK * BLOCK)
    times = [band_step(rows) for _ in range(steps)]
    t = statistics.median(times)
    full_secs = t * size / rows
    desc = (f"{rows}x{size} band of the {size}^2 level-2 fit step (Gaussians with centres in "
            f"the band +-32 px), project+bin+raster fwd+L2 grad+raster bwd+proj bwd+Adam, "
            f"fp32, scaled by {size / rows:.2f} to the full image; median of {steps}")
    return 1.0 / full_secs, cores, desc, times, rows


def run_reference(args, rank, world):
    if rank != 0:
        return
    size = args.size
    n = points_for(args)
    per_step = max(1.0, 120.0 / max(args.steps + args.warmup, 1))
    _, cores, desc, times, rows = cpu_band_sample(size, n, per_step, args.warmup + args.steps)
    timed = times[args.warmup:] or times
    secs = statistics.median(timed) * size / rows
    val = 1.0 / secs
    line = {"metric": METRIC, "value": val, "unit": "iters/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_name(size, n),
                       "global_batch": 1, "parallelism": "replicas"},
            "cpu_baseline": {"value": val, "unit": "iters/s", "cores": cores, "kind": "port",
                             "sample": desc},
            "e2e": {"value": val, "unit": "iters/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def job_rate(ms_local: float, steps: int, world: int, device) -> tuple:
    """Whole-job throughput: the slowest rank's time (max over ranks of the
    device-timed milliseconds) and world * steps units over it."""
    t = torch.tensor([ms_local], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    return world * steps / (ms_max / 1e3), ms_max


# -------------------------------------------------------------- GPU side
def run_lig(args, rank, world, local_rank):
    from lig_b200 import _lib, ops
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    size = args.size
    n = points_for(args)
    target, fit = make_workload(size, n, dev)
    for _ in range(args.warmup):
        fit.step(target)
    torch.cuda.synchronize()
    m_isect, evals = evaluations(fit)

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- per-kernel times and launch count: the iteration replays as a CUDA
    # graph, so the same kernels are run eagerly a few times (outside the
    # timed region) to time each entry point and count its launches
    batch = fit._batch
    torch.cuda.synchronize()
    l0 = _lib.lib.lig_kernel_launches()
    with ops.KernelTimer() as kt:
        for _ in range(3):
            batch._enqueue_step(target.reshape(-1, 3))
        torch.cuda.synchronize()
    launches_per_step = (_lib.lib.lig_kernel_launches() - l0) / 3
    per = kt.summary()
    per_steps = 3
    fit.step(target)  # back onto the captured graph
    torch.cuda.synchronize()

    # ---- device-timed loop (value)
    barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clocks:
        start.record()
        for _ in range(args.steps):
            fit.step(target)
        end.record()
        torch.cuda.synchronize()
    barrier()
    launches = launches_per_step * args.steps
    value, ms_max = job_rate(start.elapsed_time(end), args.steps, world, dev)
    clk = clocks.summary()

    # ---- end-to-end loop through the public API with host buffers: every
    # step uploads its target from pinned host memory (double-buffered on a
    # copy stream, so step k+1's upload overlaps step k's kernels) and copies
    # its loss back to pinned host memory; the losses are read at the end.
    host_target = target.cpu().pin_memory()
    bufs = [torch.empty_like(target), torch.empty_like(target)]
    host_loss = torch.empty(args.steps, dtype=torch.float32, pin_memory=True)
    copy_stream = torch.cuda.Stream(dev)
    ready = [torch.cuda.Event(), torch.cuda.Event()]
    consumed = [torch.cuda.Event(), torch.cuda.Event()]
    cur = torch.cuda.current_stream(dev)
    for b in bufs:  # capture the iteration once per upload buffer, untimed
        b.copy_(host_target)
        fit.step(b)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    copy_stream.wait_stream(cur)
    with torch.cuda.stream(copy_stream):
        bufs[0].copy_(host_target, non_blocking=True)
        ready[0].record(copy_stream)
    for k in range(args.steps):
        b = k % 2
        if k + 1 < args.steps:
            nb = (k + 1) % 2
            with torch.cuda.stream(copy_stream):
                if k >= 1:
                    copy_stream.wait_event(consumed[nb])  # step k-1 is done with it
                bufs[nb].copy_(host_target, non_blocking=True)
                ready[nb].record(copy_stream)
        cur.wait_event(ready[b])
        loss = fit.step(bufs[b])
        consumed[b].record(cur)
        host_loss[k].copy_(loss, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    assert bool(torch.isfinite(host_loss).all())
    barrier()
    e2e, _ = job_rate(e0.elapsed_time(e1), args.steps, world, dev)

    if rank != 0:
        return
    # ---- roofline of the dominant kernel
    fp32_peak = ops.probe_fp32(dev)
    kernels = {}
    for name, (calls, tot) in per.items():
        k = {"calls_per_step": calls / per_steps, "ms_per_step": tot / per_steps,
             "ms_per_call": tot / calls}
        if name in FLOP_PER_EVAL:
            rate = FLOP_PER_EVAL[name] * evals / (k["ms_per_call"] / 1e3)
            k.update(algorithmic_tflops=rate / 1e12, frac_of_fp32=rate / fp32_peak)
        kernels[name] = k
    dom = max(kernels, key=lambda k: kernels[k]["ms_per_step"])
    dk = kernels[dom]
    if dom in FLOP_PER_EVAL:
        achieved = FLOP_PER_EVAL[dom] * evals / (dk["ms_per_call"] / 1e3) / 1e12
        traffic = None
        if dom in DRAM_BYTES_2048:
            traffic = DRAM_BYTES_2048[dom] * (size / 2048) ** 2
        roof = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak / 1e12,
                "unit": "TFLOP/s", "frac": achieved * 1e12 / fp32_peak, "traffic": traffic,
                "traffic_note": "ncu dram bytes of the 2048^2 capture x (size/2048)^2",
                "kernel": dom, "per_launch_units": evals,
                "note": "algorithmic = reference Gaussian-pixel evaluations x FLOP/eval "
                        f"({FLOP_PER_EVAL[dom]:.0f}); peak = FP32 FMA probe measured on this "
                        "device (a SIMT-bound kernel: neither HBM nor tensor cores bound it)"}
    else:
        roof = {"bound": "hbm", "achieved": None, "peak": None, "unit": "GB/s", "frac": None,
                "traffic": None, "kernel": dom}
    tbytes = int(target.numel() * target.element_size())
    diff_bytes = int(target.numel() * 4)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        v, cores, desc, _, _ = cpu_band_sample(size, n, args.cpu_seconds, 1)
        cpu = {"value": v, "unit": "iters/s", "cores": cores, "kind": "port", "sample": desc}
    line = {"metric": METRIC, "value": value, "unit": "iters/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": workload_name(size, n),
                       "global_batch": world, "seq_len": None,
                       "parallelism": f"replicas{world}",
                       "l2": f"inputs > L2 ({tbytes / 1e6:.0f} MB target read and "
                             f"{diff_bytes / 1e6:.0f} MB masked difference written and read "
                             f"per step)",
                       "intersections": m_isect, "evaluations": evals},
            "e2e": {"value": e2e, "unit": "iters/s",
                    "h2d_bytes_per_step": tbytes, "d2h_bytes_per_step": 4},
            "gpu_launches": launches, "gpu_launches_per_step": launches_per_step,
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
            "kernels": kernels}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    try:
        run_lig(args, rank, world, local_rank)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
