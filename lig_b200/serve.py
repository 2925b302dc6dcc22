"""Serving loop: region decodes of resident Gaussian sets and fit requests on
one GPU, with HBM-budget admission and continuous batching.

The reference has no server: it fits one image per process and renders a
level with ``Gaussian2D.forward`` (train.py:181-207, gaussianlig.py:70-93).
This module serves both kinds of work at once:

* **Render requests** decode a crop of a resident set at a scale: the view
  transform means' = (means - origin) * s, L' = s L is folded into the
  projection (lig_project_fwd_view), then binning and the forward rasterizer
  produce the [h, w, 3] image in HBM.  The renders queued when the render
  worker is free are decoded together (continuous batching): one batched
  binning and one batched forward launch for all of them (render_views),
  each image identical to its own single render.  They run on a
  high-priority CUDA stream, so their thread blocks are scheduled ahead of
  queued fit blocks.
* **Fit requests** (target image, Gaussian count, iterations) run on a
  low-priority stream as one BatchedFit over every admitted fit: jobs join
  and leave the batch between chunks of iterations (continuous batching);
  each job keeps its own parameters, Adam moments and step, so its result
  does not depend on what it was batched with.
* **Admission**: every request reserves an estimate of its device bytes
  against the HBM budget before it starts and releases it when done; a
  request that does not fit waits in its queue (FIFO per kind).

Latency is measured on the host from submission to the completion of the
request's device work (a CUDA event on its stream).
"""
from __future__ import annotations

import collections
import math
import sys
import threading
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import torch

from . import _lib, ops, synthetic
from .batch import BatchedFit, BatchLayout, FitState


@dataclass
class GaussianSet:
    """A resident fitted level: means [N,2], cholesky [N,3] (or cov2d with
    cholesky=False), rgb [N,3] on the device; H, W its native image size."""
    means: torch.Tensor
    chol: torch.Tensor
    rgbs: torch.Tensor
    H: int
    W: int
    opacities: Optional[torch.Tensor] = None
    cholesky: bool = True

    @property
    def n(self) -> int:
        return self.means.shape[0]

    @property
    def nbytes(self) -> int:
        t = [self.means, self.chol, self.rgbs] + ([self.opacities] if self.opacities is not None
                                                   else [])
        return sum(x.numel() * x.element_size() for x in t)


def render_view(gs: GaussianSet, out_h: int, out_w: int, origin=(0.0, 0.0), scale=(1.0, 1.0),
                block: int = 16, grad_aware: bool = False):
    """Decode the view ((x - ox) sx, (y - oy) sy) of a set as an
    [out_h, out_w, 3] image (plus wsum and, with grad_aware, dx/dy/dxy) on
    the current stream."""
    with torch.no_grad():
        xys, ext, con, cnt = ops.project_fwd_view(gs.chol, gs.means, gs.opacities, out_h, out_w,
                                                  block, gs.cholesky, origin, scale)

        def enqueue(b):
            return ops.raster_fwd(out_h, out_w, block, b.gaussian_ids_sorted, b.tile_bins,
                                  b.total, xys, con, gs.rgbs, gs.opacities, grad_aware)

        _, outs = ops.bin_gaussians(xys, ext, cnt, out_h, out_w, block, after_enqueue=enqueue)
    img, wsum, dx, dy, dxy, _ = outs
    return (img, wsum, dx, dy, dxy) if grad_aware else (img, wsum)


def render_views(views, block: int = 16) -> List[torch.Tensor]:
    """Decode several views in one launch chain per stage.

    views: [(GaussianSet, out_h, out_w, origin, scale), ...] (at most
    LIG_MAX_BATCH).  Each view is projected (lig_project_fwd_view) into its
    slice of concatenated per-Gaussian arrays; one batched prefix sum,
    binning (lig_bin_batch: a single stable sort, tile keys offset per view)
    and forward (lig_raster_fwd_batch) then render every view.  A view's tile
    lists are exactly its single-view lists, so each [out_h, out_w, 3] image
    equals render_view's bit for bit.  Runs on the current stream; one host
    synchronisation (the intersection count sizes the sort)."""
    if not views:
        return []
    L = BatchLayout([v[1] for v in views], [v[2] for v in views], [v[0].n for v in views],
                    block)
    dev = views[0][0].means.device
    N = L.points
    f32 = dict(dtype=torch.float32, device=dev)
    xys, ext = torch.empty(max(N, 1), 2, **f32), torch.empty(max(N, 1), 2, **f32)
    con, rgbs = torch.empty(max(N, 1), 3, **f32), torch.empty(max(N, 1), 3, **f32)
    cnt = torch.empty(max(N, 1), dtype=torch.int32, device=dev)
    any_op = any(v[0].opacities is not None for v in views)
    opac = torch.ones(max(N, 1), **f32) if any_op else None
    st = ops._stream(dev)
    p = ops._p
    for k, (gs, h, w, origin, scale) in enumerate(views):
        a, b = L.g_off[k], L.g_off[k + 1]
        if b == a:
            continue
        # inputs held in locals: a converted copy must outlive the launch
        o = None if gs.opacities is None else ops._c(gs.opacities, torch.float32)
        in3, mu = ops._c(gs.chol, torch.float32), ops._c(gs.means, torch.float32)
        ops.call("lig_project_fwd_view", _lib.LIG_F32, b - a, int(gs.cholesky), p(in3), p(mu),
                 p(o), int(h), int(w), int(block), float(origin[0]), float(origin[1]),
                 float(scale[0]), float(scale[1]), p(xys[a:b]), p(ext[a:b]), p(con[a:b]),
                 p(cnt[a:b]), st)
        rgbs[a:b].copy_(gs.rgbs)
        if o is not None:
            opac[a:b].copy_(o)
    cum = torch.empty(max(N, 1), dtype=torch.int32, device=dev)
    total = torch.zeros(1, dtype=torch.int32, device=dev)
    if N > 0:
        cws = torch.empty(_lib.lib.lig_cumsum_workspace_bytes(N), dtype=torch.uint8, device=dev)
        ops.call("lig_cumsum_tiles", N, p(cnt), p(cum), p(total), p(cws), cws.numel(), st)
    m = int(total.item())
    cap = max(m, 1)
    bws = torch.empty(max(_lib.lib.lig_bin_workspace_bytes(N, cap, L.tiles), 1),
                      dtype=torch.uint8, device=dev)
    gids = torch.empty(cap, dtype=torch.int32, device=dev)
    bins = torch.empty(L.tiles, 2, dtype=torch.int32, device=dev)
    status = torch.empty(1, dtype=torch.int32, device=dev)
    ops.call("lig_bin_batch", _lib.LIG_F32, *L.args(), L.block, p(xys), p(ext), p(cum),
             p(total), cap, p(bws), bws.numel(), p(gids), p(bins), p(status), st)
    rws = torch.empty(_lib.lib.lig_raster_workspace_bytes(_lib.LIG_F32, N), dtype=torch.uint8,
                      device=dev)
    img = torch.empty(max(L.pixels, 1), 3, **f32)
    wsum = torch.empty(max(L.pixels, 1), **f32)
    fin = torch.empty(max(L.pixels, 1), dtype=torch.int32, device=dev)
    ops.call("lig_raster_fwd_batch", _lib.LIG_F32, *L.args(), L.block, p(gids), p(bins),
             p(total), p(cum), p(xys), p(con), p(rgbs), p(opac), 0, None, p(rws), rws.numel(),
             p(img), p(wsum), None, None, None, p(fin), st)
    return [L.image(img, k).clone() for k in range(L.n)]


# ---------------------------------------------------------------- requests
@dataclass
class RenderRequest:
    set_id: str
    out_h: int
    out_w: int
    origin: tuple = (0.0, 0.0)
    scale: float = 1.0
    keep: bool = True   # keep the decoded image in the result


@dataclass
class FitRequest:
    """target: [H, W, 3] device tensor, or a callable returning one (made
    when the fit is admitted, so queued requests hold no device memory;
    shape (H, W) is then required)."""
    target: object
    n_points: int
    iters: int
    lr: float = 1e-3
    seed: int = 0
    keep: bool = True        # keep the fitted parameters in the result
    shape: Optional[tuple] = None

    def hw(self):
        return tuple(self.shape) if self.shape is not None else tuple(self.target.shape[:2])


@dataclass
class Result:
    req_id: int
    kind: str
    t_submit: float
    t_start: float = 0.0      # dequeued / admitted
    t_enqueued: float = 0.0   # device work enqueued (renders)
    t_done: float = 0.0
    output: object = None
    error: Optional[str] = None

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class MemoryBudget:
    """Device bytes reserved by admitted requests and resident sets."""

    def __init__(self, budget_bytes: int):
        self.budget = int(budget_bytes)
        self.used = 0
        self.peak = 0
        self._lock = threading.Lock()

    def try_reserve(self, n: int) -> bool:
        with self._lock:
            if self.used + n > self.budget:
                return False
            self.used += n
            self.peak = max(self.peak, self.used)
            return True

    def release(self, n: int):
        with self._lock:
            self.used -= n


def render_bytes(gs: GaussianSet, out_h: int, out_w: int, block: int = 16) -> int:
    """Upper estimate of a decode's device bytes: per-Gaussian projection,
    colour / opacity copies of a batched decode and record buffers,
    intersections (keys, ids, sort buffers) from the worst tile coverage of a
    Gaussian of this set at this output size, outputs (and the batch
    buffer's copy of them)."""
    n, p = gs.n, out_h * out_w
    tiles = ((out_w + block - 1) // block) * ((out_h + block - 1) // block)
    m = min(n * 16, n + 4 * tiles * 64)
    return n * (36 + 16 + 48 + 8) + m * 20 + p * 32 + tiles * 8 + (1 << 20)


def fit_bytes(h: int, w: int, n: int, block: int = 16) -> int:
    """Estimate of a fit job's device bytes inside a batched fit: parameters,
    gradients and moments (8 floats each), per-Gaussian buffers, per-pixel
    target / render / wsum / final index, intersections (about 8 per Gaussian
    at the configs' scales) with sort buffers."""
    p = h * w
    return n * (8 * 4 * 4 + 60 + 96 + 28) + p * 32 + n * 8 * 20 + (1 << 20)


@dataclass(eq=False)
class _FitJob:
    req_id: int
    req: FitRequest
    target: Optional[torch.Tensor] = None
    state: Optional[FitState] = None
    done: int = 0
    reserved: int = 0


class Server:
    """Render + fit server on one GPU (see module docstring).

    budget_bytes: HBM budget for admission; max_fit_batch: images per batched
    fit (<= 64); fit_chunk: iterations between batch changes; fit_ahead: fit
    iterations the fit worker may have queued on the device at once (a
    deeper queue makes a render's launches wait behind it);
    max_render_batch / render_batch_pixels: most renders, and most output
    pixels, decoded together in one batch."""

    def __init__(self, budget_bytes: int = 150 * 10**9, device="cuda", block: int = 16,
                 max_fit_batch: int = 64, fit_chunk: int = 20, fit_graph: bool = True,
                 reserve_fit_bytes: int = 0, reserve_render_bytes: int = 0,
                 fit_ahead: int = 2, max_render_batch: int = 16,
                 render_batch_pixels: int = 64 << 20):
        dev = torch.device(device)
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.dev = dev
        self.block = block
        self.max_fit_batch = max_fit_batch
        self.fit_chunk = fit_chunk
        self.fit_graph = fit_graph
        self.fit_ahead = fit_ahead
        self.budget = MemoryBudget(budget_bytes)
        # lower is higher priority; out-of-range values map to the extremes
        self.render_stream = torch.cuda.Stream(self.dev, priority=-16)
        self.fit_stream = torch.cuda.Stream(self.dev, priority=0)
        self.sets: Dict[str, GaussianSet] = {}
        self.results: Dict[int, Result] = {}
        self._render_q: collections.deque = collections.deque()
        self._fit_q: collections.deque = collections.deque()
        self._cv = threading.Condition()
        self._next_id = 0
        self._running = False
        self._abort = False
        self._threads: List[threading.Thread] = []
        self.fit_batches = 0
        self.max_render_batch = max(1, min(int(max_render_batch), _lib.LIG_MAX_BATCH))
        self.render_batch_pixels = int(render_batch_pixels)
        self.render_batches: List[int] = []  # renders per decoded batch
        self.errors: List[str] = []
        # device memory taken into the allocator's cache per stream at start,
        # so the workers' allocations come from the cache: a large cudaMalloc
        # in the fit thread holds up the render thread's launches meanwhile
        self.reserve = {"fit": int(reserve_fit_bytes), "render": int(reserve_render_bytes)}
        self.fit_phases: List[tuple] = []  # (t0, t1, phase) of the fit thread

    # ----------------------------------------------------------- resources
    def add_set(self, set_id: str, gs: GaussianSet):
        if not self.budget.try_reserve(gs.nbytes):
            raise MemoryError(f"set {set_id}: {gs.nbytes} bytes exceed the HBM budget")
        self.sets[set_id] = gs

    def submit(self, req) -> int:
        with self._cv:
            rid = self._next_id
            self._next_id += 1
            kind = "render" if isinstance(req, RenderRequest) else "fit"
            self.results[rid] = Result(rid, kind, time.perf_counter())
            (self._render_q if kind == "render" else self._fit_q).append((rid, req))
            self._cv.notify_all()
        return rid

    def start(self):
        for kind, stream in (("fit", self.fit_stream), ("render", self.render_stream)):
            if self.reserve[kind] > 0:
                with torch.cuda.stream(stream):
                    block = torch.empty(self.reserve[kind], dtype=torch.uint8, device=self.dev)
                    del block  # stays cached for this stream
        torch.cuda.synchronize(self.dev)
        # the render thread needs the GIL back within a fraction of a
        # millisecond while the fit thread runs Python between launches
        self._switch = sys.getswitchinterval()
        sys.setswitchinterval(2e-4)
        self._running = True
        self._threads = [threading.Thread(target=self._render_loop, name="lig-render",
                                          daemon=True),
                         threading.Thread(target=self._fit_loop, name="lig-fit", daemon=True)]
        for t in self._threads:
            t.start()

    def drain(self, timeout: Optional[float] = None) -> bool:
        """Wait until every submitted request has finished."""
        t_end = None if timeout is None else time.perf_counter() + timeout
        while True:
            with self._cv:
                pending = [r for r in self.results.values() if r.t_done == 0.0]
                if not pending:
                    return True
                left = None if t_end is None else t_end - time.perf_counter()
                if left is not None and left <= 0:
                    return False
                self._cv.wait(0.05 if left is None else min(0.05, left))

    def stop(self, abort: bool = False):
        """Stop the workers after the queues drain (abort: drop what is
        queued or running; those requests stay unfinished)."""
        with self._cv:
            self._running = False
            self._abort = abort
            if abort:
                self._render_q.clear()
                self._fit_q.clear()
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        if getattr(self, "_switch", None) is not None:
            sys.setswitchinterval(self._switch)
            self._switch = None

    def _finish(self, rid: int, output=None, error: Optional[str] = None):
        with self._cv:
            r = self.results[rid]
            r.output = output
            r.error = error
            r.t_done = time.perf_counter()
            if error:
                self.errors.append(f"{r.kind} {rid}: {error}")
            self._cv.notify_all()

    # -------------------------------------------------------------- renders
    def _take_renders(self):
        """Under the lock: the queued renders to decode next, FIFO, as many as
        memory, max_render_batch and render_batch_pixels allow (the head of
        the queue waits for memory); unknown sets are returned as errors."""
        batch, errors, pixels = [], [], 0
        while self._render_q and len(batch) < self.max_render_batch:
            rid, req = self._render_q[0]
            gs = self.sets.get(req.set_id)
            if gs is None:
                self._render_q.popleft()
                errors.append((rid, req))
                continue
            px = req.out_h * req.out_w
            if batch and pixels + px > self.render_batch_pixels:
                break
            need = render_bytes(gs, req.out_h, req.out_w, self.block)
            if not self.budget.try_reserve(need):
                break
            self._render_q.popleft()
            batch.append((rid, req, gs, need))
            pixels += px
        return batch, errors

    def _render_loop(self):
        torch.cuda.set_device(self.dev)
        while True:
            with self._cv:
                if self._abort:
                    return
                while self._running and not self._render_q:
                    self._cv.wait(0.05)
                if not self._render_q:
                    if not self._running:
                        return
                    continue
                batch, errors = self._take_renders()
                if not batch and not errors:
                    self._cv.wait(0.01)  # head of line waits for memory
                    continue
            for rid, req in errors:
                self._finish(rid, error=f"unknown set {req.set_id}")
            if not batch:
                continue
            t0 = time.perf_counter()
            for rid, *_ in batch:
                self.results[rid].t_start = t0
            try:
                with torch.cuda.stream(self.render_stream):
                    imgs = render_views([(gs, req.out_h, req.out_w, req.origin,
                                          (req.scale, req.scale)) for _, req, gs, _ in batch],
                                        self.block)
                    ev = torch.cuda.Event()
                    ev.record(self.render_stream)
                t1 = time.perf_counter()
                for rid, *_ in batch:
                    self.results[rid].t_enqueued = t1
                self.render_batches.append(len(batch))
                ev.synchronize()
                for (rid, req, _, _), img in zip(batch, imgs):
                    self._finish(rid, img if req.keep else None)
            except Exception as e:  # reported per request; the loop keeps serving
                for rid, *_ in batch:
                    self._finish(rid, error=repr(e))
            finally:
                for *_, need in batch:
                    self.budget.release(need)

    # ----------------------------------------------------------------- fits
    def _admit_fits(self, active: List[_FitJob]) -> bool:
        """Move queued fits into the running batch while memory and batch
        slots allow (FIFO; fits with another learning rate wait until the
        batch drains)."""
        changed = False
        with self._cv:
            while self._fit_q and len(active) < self.max_fit_batch:
                rid, req = self._fit_q[0]
                if active and req.lr != active[0].req.lr:
                    break
                h, w = req.hw()
                need = fit_bytes(h, w, req.n_points, self.block)
                if not self.budget.try_reserve(need):
                    break
                self._fit_q.popleft()
                self.results[rid].t_start = time.perf_counter()
                active.append(_FitJob(rid, req, reserved=need))
                changed = True
        return changed

    def _build_batch(self, jobs: List[_FitJob]) -> BatchedFit:
        init = []
        for j in jobs:
            if j.target is None:
                t = j.req.target() if callable(j.req.target) else j.req.target
                j.target = t.to(self.dev, torch.float32).contiguous()
            if j.state is None:  # initial Gaussians drawn on the device
                h, w = j.target.shape[:2]
                j.state = FitState(synthetic.gaussians_on_device(j.req.n_points, h, w, self.dev,
                                                                 seed=j.req.seed))
            init.append(j.state)
        fit = BatchedFit([j.target for j in jobs], [j.req.n_points for j in jobs],
                         block=self.block, lr=jobs[0].req.lr, init=init, graph=self.fit_graph)
        self.fit_batches += 1
        return fit

    def _fit_loop(self):
        torch.cuda.set_device(self.dev)
        active: List[_FitJob] = []
        batch: Optional[BatchedFit] = None
        batch_jobs: List[_FitJob] = []
        with torch.cuda.stream(self.fit_stream):
            while True:
                if self._abort:
                    for j in active:
                        self.budget.release(j.reserved)
                    return
                changed = self._admit_fits(active)
                if not active:
                    with self._cv:
                        if not self._running and not self._fit_q:
                            return
                        self._cv.wait(0.05)
                    continue
                try:
                    if changed or batch is None:
                        t0 = time.perf_counter()
                        if batch is not None:  # carry running jobs over
                            for j, st in zip(batch_jobs, batch.export_states()):
                                j.state = st
                            batch = None
                        batch_jobs = list(active)
                        batch = self._build_batch(batch_jobs)
                        self.fit_phases.append((t0, time.perf_counter(), "build"))
                    k = min(self.fit_chunk, min(j.req.iters - j.done for j in batch_jobs))
                    t0 = time.perf_counter()
                    batch.fit(k, max_ahead=self.fit_ahead)
                    self.fit_phases.append((t0, time.perf_counter(), "iterate"))
                except Exception as e:  # fail this batch's jobs, keep serving
                    for j in active:
                        self.budget.release(j.reserved)
                        self._finish(j.req_id, error=repr(e))
                    active, batch, batch_jobs = [], None, []
                    continue
                for j in batch_jobs:
                    j.done += k
                finished = [j for j in batch_jobs if j.done >= j.req.iters]
                if finished:
                    t0 = time.perf_counter()
                    for j, st in zip(batch_jobs, batch.export_states()):
                        if j.done >= j.req.iters:
                            self.budget.release(j.reserved)
                            out = tuple(t.clone() for t in st.params) if j.req.keep else None
                            self._finish(j.req_id, out)
                        else:
                            j.state = st
                    active = [j for j in active if j.done < j.req.iters]
                    batch, batch_jobs = None, []
                    self.fit_phases.append((t0, time.perf_counter(), "finish"))


# ------------------------------------------------------------------ workload
@dataclass
class WorkloadStats:
    n_render: int = 0
    n_fit: int = 0
    render_latency_ms: List[float] = field(default_factory=list)
    render_2048_latency_ms: List[float] = field(default_factory=list)
    render_wait_ms: List[float] = field(default_factory=list)      # submit -> dequeue
    render_enqueue_ms: List[float] = field(default_factory=list)   # dequeue -> enqueued
    render_device_ms: List[float] = field(default_factory=list)    # enqueued -> done
    fit_latency_s: List[float] = field(default_factory=list)
    unfinished: int = 0
    wall_s: float = 0.0
    slow_render_phases: dict = field(default_factory=dict)  # fit phase overlapping a slow wait


def percentile(xs: List[float], q: float) -> float:
    if not xs:
        return float("nan")
    s = sorted(xs)
    k = min(len(s) - 1, max(0, int(math.ceil(q / 100.0 * len(s))) - 1))
    return s[k]


def resident_sets(n_sets: int = 64, n_min: int = 100_000, n_max: int = 3_000_000,
                  seed: int = 5000, device="cuda") -> Dict[str, GaussianSet]:
    """Seeded stand-ins for pre-fitted sets: set k has N_k ~ U[n_min, n_max]
    Gaussians drawn as the fit configurations draw them, on an image whose
    side gives 0.2 Gaussians per pixel."""
    g = torch.Generator().manual_seed(seed)
    out = {}
    for k in range(n_sets):
        n = int(n_min + (n_max - n_min) * torch.rand(1, generator=g).item())
        side = int(round(math.sqrt(n / 0.2)))
        mu, ch, co = synthetic.gaussians(n, side, side, diag=(0.5, 4.0), seed=seed + 1 + k)
        out[f"set{k}"] = GaussianSet(mu.to(device), ch.to(device), co.to(device), side, side)
    return out


def fitted_sets(n_sets: int = 64, n_min: int = 100_000, n_max: int = 3_000_000,
                seed: int = 5000, iters: int = 100, lr: float = 1e-2, directory=None,
                device="cuda", block: int = 16,
                max_batch_pixels: int = 120_000_000) -> Dict[str, GaussianSet]:
    """Resident sets that are fits, stored and loaded as LIG stores them.

    Set k has the Gaussian count and image side of resident_sets (N_k ~
    U[n_min, n_max], side sqrt(N_k / 0.2)).  Its target is a seeded
    synthetic image of that side (teacher render at the fit configurations'
    density plus N(0, 0.02) noise); N_k Gaussians (means / Cholesky factors
    drawn as resident_sets draws them, colours starting at zero as
    gaussianlig.py:57) are fitted for `iters` Adam iterations, in
    BatchedFits of at most max_batch_pixels target pixels.  Each fitted set
    is written with save_lig (the reference's checkpoint layout,
    train.py:172-176) into `directory` (a temporary directory by default)
    and read back with load_lig (train.py:49-67); the loaded sets are
    returned."""
    import os
    import tempfile

    from .fit import make_target
    from .levels import load_lig, save_lig

    g = torch.Generator().manual_seed(seed)
    counts, sides = [], []
    for k in range(n_sets):
        n = int(n_min + (n_max - n_min) * torch.rand(1, generator=g).item())
        counts.append(n)
        sides.append(int(round(math.sqrt(n / 0.2))))
    # batches of sets under a pixel budget (32-bit pixel-channel indexing and
    # memory), fitted one after another
    groups, cur, px = [], [], 0
    for k, side in enumerate(sides):
        if cur and px + side * side > max_batch_pixels:
            groups.append(cur)
            cur, px = [], 0
        cur.append(k)
        px += side * side
    groups.append(cur)
    own = directory is None
    d = tempfile.mkdtemp(prefix="lig_sets_") if own else directory
    out = {}
    try:
        for grp in groups:
            targets, init = [], []
            for k in grp:
                n, side = counts[k], sides[k]
                n_teacher = int(round(20000 / 512**2 * side * side))
                targets.append(make_target(side, side, n_teacher, (0.5, 4.0), noise="white",
                                           noise_std=0.02, device=device, block=block))
                mu, ch, _ = synthetic.gaussians(n, side, side, diag=(0.5, 4.0),
                                                seed=seed + 1 + k)
                init.append((mu.to(device), ch.to(device), torch.zeros(n, 3, device=device)))
            fit = BatchedFit(targets, [counts[k] for k in grp], block=block, lr=lr, init=init)
            fit.fit(iters)
            for i, k in enumerate(grp):
                mu, ch, co = (t.detach() for t in fit.params_of(i))
                path = os.path.join(d, f"set{k}.pth")
                save_lig(path, [GaussianSet(mu, ch, co, sides[k], sides[k])], [], [])
                out[f"set{k}"] = load_lig(path, device=device).levels[0]
                if own:
                    os.remove(path)
            del fit, targets, init
            torch.cuda.empty_cache()
    finally:
        if own:
            os.rmdir(d)
    return out


def poisson_requests(duration_s: float, rate: float, fit_frac: float, sets: Dict[str, GaussianSet],
                     fit_iters: int = 300, fit_side=(512, 4096), render_side=(256, 4096),
                     render_scale=(0.25, 2.0), seed: int = 5000):
    """Arrival schedule [(t, kind, params)]: Poisson arrivals; fits draw a
    square side U[fit_side] (0.2 Gaussians per pixel, capped at 1M); renders
    draw a set, an output side U[render_side], a scale U[render_scale] and a
    crop origin uniform over the set's image."""
    g = torch.Generator().manual_seed(seed)
    u = lambda: torch.rand(1, generator=g).item()  # noqa: E731
    names = sorted(sets)
    t, out = 0.0, []
    while True:
        t += -math.log(max(1e-12, 1.0 - u())) / rate
        if t >= duration_s:
            return out
        if u() < fit_frac:
            side = int(fit_side[0] + (fit_side[1] - fit_side[0]) * u())
            out.append((t, "fit", {"side": side, "n": min(int(round(0.2 * side * side)),
                                                          1_000_000), "iters": fit_iters,
                                   "seed": 6000 + len(out)}))
        else:
            name = names[int(u() * len(names)) % len(names)]
            gs = sets[name]
            side = int(render_side[0] + (render_side[1] - render_side[0]) * u())
            s = render_scale[0] + (render_scale[1] - render_scale[0]) * u()
            span = side / s
            ox = u() * max(0.0, gs.W - span)
            oy = u() * max(0.0, gs.H - span)
            out.append((t, "render", {"set": name, "side": side, "scale": s,
                                      "origin": (ox, oy)}))


def warm_up(server: Server, sides=(256, 1024, 2048, 4096), scales=(0.25, 1.0, 2.0),
            fit_side: int = 1024, fit_points: int = 50_000):
    """Render a few views of each resident set's kind at several output sizes
    and scales on the render stream, and run a small batched fit (through its
    CUDA-graph capture) on the fit stream, so the first requests do not pay
    for first-use costs (kernel loading, tile-count-dependent sort set-up,
    the first graph capture, pinned staging words, allocator growth) while
    other requests are in flight."""
    gs = next(iter(server.sets.values()), None)
    if gs is not None:
        with torch.cuda.stream(server.render_stream):
            for side in sides:
                for s in scales:
                    render_view(gs, side, side, (0.0, 0.0), (s, s), server.block)
    if fit_side > 0:
        with torch.cuda.stream(server.fit_stream):
            g = torch.Generator(device=server.dev).manual_seed(1)
            target = torch.rand(fit_side, fit_side, 3, generator=g, device=server.dev)
            init = FitState(synthetic.gaussians_on_device(fit_points, fit_side, fit_side,
                                                          server.dev, seed=2))
            fit = BatchedFit([target], [fit_points], block=server.block, lr=1e-3, init=[init],
                             graph=server.fit_graph)
            fit.fit(4, max_ahead=server.fit_ahead)
            del fit, target, init
    torch.cuda.synchronize(server.dev)


def run_workload(server: Server, schedule, master_target: torch.Tensor, drain_s: float = 60.0,
                 fit_lr: float = 1e-3) -> WorkloadStats:
    """Submit `schedule` (from poisson_requests) at its arrival times, wait up
    to drain_s after the last arrival, abort what is left and collect
    latencies.  Fit targets are top-left crops of master_target, copied
    when the fit is admitted."""
    st = WorkloadStats()
    kinds = {}
    if not server._threads:
        server.start()  # before the clock: start-up reserves device memory
    t0 = time.perf_counter()
    for t, kind, p in schedule:
        delay = t0 + t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        if kind == "render":
            rid = server.submit(RenderRequest(p["set"], p["side"], p["side"], p["origin"],
                                              p["scale"], keep=False))
            st.n_render += 1
        else:
            side = p["side"]
            rid = server.submit(FitRequest(
                lambda side=side: master_target[:side, :side], p["n"], p["iters"], lr=fit_lr,
                seed=p["seed"], keep=False, shape=(side, side)))
            st.n_fit += 1
        kinds[rid] = p
    server.drain(timeout=drain_s)
    server.stop(abort=True)
    st.wall_s = time.perf_counter() - t0
    for rid, r in server.results.items():
        if r.t_done == 0.0 or r.error:
            st.unfinished += 1
            continue
        if r.kind == "render":
            ms = 1e3 * r.latency
            st.render_latency_ms.append(ms)
            st.render_wait_ms.append(1e3 * (r.t_start - r.t_submit))
            st.render_enqueue_ms.append(1e3 * (r.t_enqueued - r.t_start))
            st.render_device_ms.append(1e3 * (r.t_done - r.t_enqueued))
            if 1792 <= kinds[rid]["side"] <= 2304:
                st.render_2048_latency_ms.append(ms)
        else:
            st.fit_latency_s.append(r.latency)
    # which fit-thread phase overlapped the renders that waited > 20 ms
    for rid, r in server.results.items():
        if r.kind != "render" or r.t_done == 0.0 or r.t_start - r.t_submit <= 0.02:
            continue
        hit = [ph for (a, b, ph) in server.fit_phases if a < r.t_start and b > r.t_submit]
        key = "+".join(sorted(set(hit))) or "none"
        st.slow_render_phases[key] = st.slow_render_phases.get(key, 0) + 1
    return st
