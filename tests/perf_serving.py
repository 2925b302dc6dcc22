"""Serving loop under a Poisson mix of renders and fits (one GPU).

Workload (seeded, synthetic): 64 resident sets of 100k-3M Gaussians, 0.2
Gaussians per pixel of the set's image, fitted to synthetic images and
stored / loaded in LIG's checkpoint format (lig_b200.serve.fitted_sets;
--random-sets uses unfitted seeded draws instead);
Poisson arrivals at --rate per second for --duration seconds, a --fit-frac
share of fits (square target side U[512, 4096], min(0.2 side^2, 1M)
Gaussians, --fit-iters iterations, targets cropped from one 4096^2 teacher
render with N(0, 0.02) noise) and the rest renders (a set, output side
U[256, 4096], scale U[0.25, 2], crop origin uniform over the set's image).
Admission against an HBM budget (--budget-gb).  After the last arrival the
server gets --drain seconds; what is still queued or running then is
counted as unfinished.

Prints one JSON line: counts, render p50/p99 (all, and 2048^2 +-12.5%),
fit latency p50/p99 of finished fits, throughput, unfinished, memory peak.

    python tests/perf_serving.py [--duration 60] [--rate 200] [--drain 30]
"""
import argparse
import json
import os
import sys
import time

# a server loads every kernel up front rather than on first use mid-request
os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")

import torch  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from lig_b200.fit import make_target  # noqa: E402
from lig_b200.serve import (Server, fitted_sets, percentile, poisson_requests,  # noqa: E402
                            resident_sets, run_workload)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--duration", type=float, default=60.0)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--fit-frac", type=float, default=0.3)
    ap.add_argument("--fit-iters", type=int, default=300)
    ap.add_argument("--drain", type=float, default=30.0)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--sets", type=int, default=64)
    ap.add_argument("--set-fit-iters", type=int, default=100,
                    help="iterations of the resident sets' fits")
    ap.add_argument("--random-sets", action="store_true",
                    help="unfitted seeded draws as resident sets")
    ap.add_argument("--fit-chunk", type=int, default=20)
    ap.add_argument("--fit-ahead", type=int, default=2,
                    help="fit iterations queued on the device at most (0: a whole chunk)")
    ap.add_argument("--no-fit-graph", action="store_true")
    ap.add_argument("--reserve-fit-gb", type=float, default=60.0)
    ap.add_argument("--reserve-render-gb", type=float, default=8.0)
    ap.add_argument("--dump", default="", help="write per-request timings (CSV) here")
    a = ap.parse_args()
    t0 = time.time()
    sets = (resident_sets(a.sets) if a.random_sets
            else fitted_sets(a.sets, iters=a.set_fit_iters))
    torch.cuda.empty_cache()
    master = make_target(4096, 4096, int(round(20000 / 512**2 * 4096**2)), (0.5, 4.0),
                         noise="white", noise_std=0.02)
    schedule = poisson_requests(a.duration, a.rate, a.fit_frac, sets, fit_iters=a.fit_iters,
                                seed=5000)
    srv = Server(budget_bytes=int(a.budget_gb * 1e9), fit_chunk=a.fit_chunk,
                 fit_graph=not a.no_fit_graph, reserve_fit_bytes=int(a.reserve_fit_gb * 1e9),
                 reserve_render_bytes=int(a.reserve_render_gb * 1e9), fit_ahead=a.fit_ahead)
    for k, gs in sets.items():
        srv.add_set(k, gs)
    # start the workers and warm the render path before the clock starts
    from lig_b200.serve import warm_up
    srv.start()
    warm_up(srv)
    setup = time.time() - t0
    st = run_workload(srv, schedule, master, drain_s=a.drain)
    r, r2, f = st.render_latency_ms, st.render_2048_latency_ms, st.fit_latency_s
    out = {
        "workload": "serving loop", "duration_s": a.duration, "rate": a.rate,
        "fit_frac": a.fit_frac, "fit_iters": a.fit_iters, "drain_s": a.drain,
        "setup_s": round(setup, 1), "wall_s": round(st.wall_s, 1),
        "requests": {"render": st.n_render, "fit": st.n_fit},
        "finished": {"render": len(r), "fit": len(f)}, "unfinished": st.unfinished,
        "render_ms": {"p50": percentile(r, 50), "p99": percentile(r, 99), "n": len(r)},
        "render_2048_ms": {"p50": percentile(r2, 50), "p99": percentile(r2, 99), "n": len(r2)},
        "render_parts_ms": {k: {"p50": percentile(v, 50), "p99": percentile(v, 99)}
                            for k, v in (("wait", st.render_wait_ms),
                                         ("enqueue", st.render_enqueue_ms),
                                         ("device", st.render_device_ms))},
        "fit_s": {"p50": percentile(f, 50), "p99": percentile(f, 99), "n": len(f)},
        "throughput_per_s": {"render": len(r) / st.wall_s, "fit": len(f) / st.wall_s},
        "slow_render_fit_phases": st.slow_render_phases, "fit_ahead": a.fit_ahead,
        "fit_phase_s": {ph: round(sum(b - a for a, b, p in srv.fit_phases if p == ph), 2)
                        for ph in ("build", "iterate", "finish")},
        "fit_batches": srv.fit_batches, "budget_peak_gb": srv.budget.peak / 1e9,
        "sets": "random draws" if a.random_sets else f"fitted ({a.set_fit_iters} iters), "
                                                      "saved and loaded with save_lig/load_lig",
        "render_batches": {"count": len(srv.render_batches),
                           "mean_size": (sum(srv.render_batches) / len(srv.render_batches)
                                         if srv.render_batches else 0.0),
                           "max_size": max(srv.render_batches, default=0)},
        "errors": srv.errors[:5],
    }
    if a.dump:
        with open(a.dump, "w") as f:
            f.write("id,kind,t_submit,t_start,t_enqueued,t_done,error\n")
            for rid, r in sorted(srv.results.items()):
                f.write(f"{rid},{r.kind},{r.t_submit:.6f},{r.t_start:.6f},{r.t_enqueued:.6f},"
                        f"{r.t_done:.6f},{1 if r.error else 0}\n")
            for a0, b0, ph in srv.fit_phases:
                f.write(f"-1,phase:{ph},{a0:.6f},{b0:.6f},0,0,0\n")
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
