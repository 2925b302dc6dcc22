"""Batched uneven fit: many LIG levels — one Gaussian set per image, images of
different sizes — fitted together, one launch per pipeline stage per
iteration, the whole iteration captured as one CUDA graph.

The reference fits one image per process (train.py:112-158 around
gaussianlig.Gaussian2D.train_iter, gaussianlig.py:99-111): per iteration a
projection, a cumsum + ``.item()`` host sync, a sort, a forward and a
backward launch per image.  Here every image of a batch shares each launch:

* parameters of all images live in one flat fp32 buffer
  (means [N,2] | cholesky [N,3] | rgb [N,3], N = total Gaussians) with the
  gradients and Adam moments laid out the same way;
* projection, prefix sum, emission + one stable radix sort over the batch's
  flattened tile keys, the forward rasterizer over the flattened
  (image, tile) work list (optionally persistent: CTAs pull work items from a
  counter) with the per-image clamped-L2 loss fused in, the backward from the
  forward's masked difference and one guarded Adam step — no host
  synchronisation anywhere;
* the intersection capacity is fixed when the iteration is captured; a step
  whose binning overflows it is skipped on the device (lig_adam_step's
  guard) and counted, and the host grows the capacity, re-captures and redoes
  exactly the skipped steps.

The loss is the sum of the per-image mean squared errors, so each image's
Gaussians receive exactly the gradient of their own single-image fit, and
every image renders bit-identically to a single-image render of the same
Gaussians (same per-tile lists in the same order).

``autotune`` picks the tile size and the persistent/one-CTA-per-tile walk by
timing captured iterations of the actual batch.
"""
from __future__ import annotations

import ctypes
import json
import collections
import math
import os
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import torch

from . import _lib, synthetic
from .ops import call

_VP = ctypes.c_void_p


def _p(t: Optional[torch.Tensor]):
    return None if t is None else _VP(t.data_ptr())


class BatchLayout:
    """Sizes of a batch: image i is heights[i] x widths[i] with counts[i]
    Gaussians; offsets of each image in the concatenated arrays."""

    def __init__(self, heights: Sequence[int], widths: Sequence[int], counts: Sequence[int],
                 block: int):
        n = len(heights)
        if not (1 <= n <= _lib.LIG_MAX_BATCH) or len(widths) != n or len(counts) != n:
            raise ValueError(f"a batch holds 1..{_lib.LIG_MAX_BATCH} images with one height, "
                             f"width and Gaussian count each")
        if not (2 <= block <= 32):
            raise ValueError("block must be in [2, 32]")
        if min(heights) <= 0 or min(widths) <= 0 or min(counts) < 0:
            raise ValueError("heights and widths must be positive, counts non-negative")
        self.n = n
        self.block = int(block)
        self.heights = [int(h) for h in heights]
        self.widths = [int(w) for w in widths]
        self.counts = [int(c) for c in counts]
        self._h = (ctypes.c_int32 * n)(*self.heights)
        self._w = (ctypes.c_int32 * n)(*self.widths)
        self._c = (ctypes.c_int32 * n)(*self.counts)
        self.g_off, self.pix_off, self.tile_off = [0], [0], [0]
        for h, w, c in zip(self.heights, self.widths, self.counts):
            self.g_off.append(self.g_off[-1] + c)
            self.pix_off.append(self.pix_off[-1] + h * w)
            tb = ((w + block - 1) // block) * ((h + block - 1) // block)
            self.tile_off.append(self.tile_off[-1] + tb)
        if self.g_off[-1] >= 2**31 or 3 * self.pix_off[-1] >= 2**31 or self.tile_off[-1] >= 2**31:
            raise ValueError("batch too large for 32-bit indexing")

    @property
    def points(self) -> int:
        return self.g_off[-1]

    @property
    def pixels(self) -> int:
        return self.pix_off[-1]

    @property
    def tiles(self) -> int:
        return self.tile_off[-1]

    def args(self):
        """(n_img, heights*, widths*, counts*) for the lig_*_batch entries."""
        return (self.n, ctypes.cast(self._h, _VP), ctypes.cast(self._w, _VP),
                ctypes.cast(self._c, _VP))

    def hw_args(self):
        return (self.n, ctypes.cast(self._h, _VP), ctypes.cast(self._w, _VP))

    def image(self, flat_hwc: torch.Tensor, i: int) -> torch.Tensor:
        """View of image i in a concatenated [pixels, C] buffer, as [H, W, C]."""
        a, b = self.pix_off[i], self.pix_off[i + 1]
        return flat_hwc[a:b].view(self.heights[i], self.widths[i], -1)

    def points_of(self, flat: torch.Tensor, i: int) -> torch.Tensor:
        return flat[self.g_off[i]:self.g_off[i + 1]]


@dataclass
class FitState:
    """One image's fit state: (means, cholesky, rgb) parameters, the matching
    Adam first / second moments (None: zeros) and the Adam step count."""
    params: tuple
    exp_avg: Optional[tuple] = None
    exp_avg_sq: Optional[tuple] = None
    step: int = 0


@dataclass
class BatchStats:
    iters: int = 0
    skipped: int = 0
    recaptures: int = 0
    capacity: int = 0


class BatchedFit:
    """Fits one Gaussian set per target image, all images per launch.

    targets: list of [H_i, W_i, 3] CUDA tensors, all fp32 or all uint8 (RGB
    images as stored, read as byte / 255 like torchvision's ToTensor, for a
    quarter of the bytes to upload and read); counts: Gaussians per
    image; init: optional list per image of (means, cholesky, colors) or of
    a FitState (parameters plus Adam moments and step, to resume a fit); else
    seeded synthetic Gaussians, seed seed_base + i; block: tile size;
    persistent: persistent tile walk in the rasterizer; graph: capture the
    iteration as a CUDA graph (after two eager iterations)."""

    def __init__(self, targets: List[torch.Tensor], counts: Sequence[int], block: int = 16,
                 lr: float = 1e-3, betas=(0.9, 0.999), eps: float = 1e-8, diag=(0.5, 4.0),
                 init: Optional[list] = None, persistent: bool = False, graph: bool = True,
                 slack: float = 1.25, seed_base: int = 3000):
        if not targets:
            raise ValueError("no targets")
        dev = targets[0].device
        if dev.type != "cuda":
            raise RuntimeError("lig_b200: BatchedFit runs on CUDA tensors only (no CPU fallback)")
        self.dev = dev
        self.L = BatchLayout([t.shape[0] for t in targets], [t.shape[1] for t in targets],
                             counts, block)
        self.lr, self.b1, self.b2, self.eps = float(lr), float(betas[0]), float(betas[1]), eps
        self.persistent = bool(persistent)
        self.use_graph = bool(graph)
        self.slack = float(slack)
        L = self.L
        N, P = L.points, L.pixels
        f32, i32 = torch.float32, torch.int32
        kw = dict(device=dev)
        # parameters / gradients / moments: one flat buffer each
        self.flat = torch.empty(8 * N, dtype=f32, **kw)
        self.grad = torch.zeros(8 * N, dtype=f32, **kw)
        self.m = torch.zeros(8 * N, dtype=f32, **kw)
        self.v = torch.zeros(8 * N, dtype=f32, **kw)
        self.means, self.chol, self.rgbs = self._views(self.flat)
        self.g_means, self.g_chol, self.g_rgbs = self._views(self.grad)
        self.steps = torch.zeros(L.n, dtype=i32, **kw)  # Adam steps per image
        with torch.no_grad():
            for i in range(L.n):
                src = init[i] if init is not None else None
                if isinstance(src, FitState):
                    self._load_state(i, src)
                    continue
                if src is not None:
                    mu, ch, co = src
                else:
                    mu, ch, co = synthetic.gaussians(L.counts[i], L.heights[i], L.widths[i],
                                                     diag=diag, seed=seed_base + i)
                L.points_of(self.means, i).copy_(mu)
                L.points_of(self.chol, i).copy_(ch)
                L.points_of(self.rgbs, i).copy_(co)
            u8 = all(t.dtype == torch.uint8 for t in targets)
            tdt = torch.uint8 if u8 else f32
            self.target = torch.cat([t.reshape(-1, 3).to(tdt) for t in targets]).contiguous()
        # per-step buffers
        self.xys = torch.empty(N, 2, dtype=f32, **kw)
        self.ext = torch.empty(N, 2, dtype=f32, **kw)
        self.con = torch.empty(N, 3, dtype=f32, **kw)
        self.cnt = torch.empty(N, dtype=i32, **kw)
        self.cum = torch.empty(max(N, 1), dtype=i32, **kw)
        self.total = torch.zeros(1, dtype=i32, **kw)
        self.status = torch.zeros(1, dtype=i32, **kw)
        self.cs_ws = torch.empty(_lib.lib.lig_cumsum_workspace_bytes(N), dtype=torch.uint8, **kw)
        self.bins = torch.zeros(L.tiles, 2, dtype=i32, **kw)
        self.img = torch.empty(P, 3, dtype=f32, **kw)
        self.wsum = torch.empty(P, dtype=f32, **kw)
        self.fin = torch.empty(P, dtype=i32, **kw)
        self.loss = torch.zeros((), dtype=f32, **kw)
        self.per_image = torch.zeros(L.n, dtype=f32, **kw)
        self.partials = torch.empty(_lib.lib.lig_l2_tile_partials_bytes(L.tiles) // 8,
                                    dtype=torch.float64, **kw)
        self.r_ws = torch.empty(_lib.lib.lig_raster_workspace_bytes(_lib.LIG_F32, N),
                                dtype=torch.uint8, **kw)
        self.v_xy = torch.empty(N, 2, dtype=f32, **kw)
        self.v_abs = torch.empty(N, 2, dtype=f32, **kw)
        self.v_con = torch.empty(N, 3, dtype=f32, **kw)
        self.one = torch.ones((), dtype=f32, **kw)
        self.work = torch.zeros(1, dtype=i32, **kw)
        self.skipped = torch.zeros(1, dtype=i32, **kw)
        self.adam_scratch = torch.empty(_lib.lib.lig_adam_batch_scratch_bytes(L.n),
                                        dtype=torch.uint8, **kw)
        self.host_skipped = torch.zeros(1, dtype=i32, pin_memory=True)
        self.capacity = 0
        self.gids = None
        self.bin_ws = None
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self._graphs: dict = {}
        self.stats = BatchStats()
        self._size_capacity(self._count_intersections())

    # ------------------------------------------------------------ helpers
    def _segments(self, flat, i):
        """Image i's (means, cholesky, rgb) views in a flat [8N] buffer."""
        return tuple(self.L.points_of(v, i) for v in self._views(flat))

    def _load_state(self, i, st: "FitState"):
        for buf, parts in ((self.flat, st.params), (self.m, st.exp_avg), (self.v, st.exp_avg_sq)):
            if parts is None:
                continue
            for dst, src in zip(self._segments(buf, i), parts):
                dst.copy_(src)
        self.steps[i] = int(st.step)

    def export_states(self) -> List["FitState"]:
        """Every image's state at once: three buffer copies and one read of
        the step counts (the per-image states are views into the copies)."""
        flat, m, v = self.flat.clone(), self.m.clone(), self.v.clone()
        steps = self.steps.tolist()
        return [FitState(self._segments(flat, i), self._segments(m, i), self._segments(v, i),
                         steps[i]) for i in range(self.L.n)]

    def state_of(self, i: int) -> "FitState":
        """Copy of image i's parameters, Adam moments and step (device)."""
        seg = lambda buf: tuple(t.clone() for t in self._segments(buf, i))  # noqa: E731
        return FitState(seg(self.flat), seg(self.m), seg(self.v), int(self.steps[i].item()))

    def _views(self, flat):
        N = self.L.points
        return (flat[:2 * N].view(N, 2), flat[2 * N:5 * N].view(N, 3),
                flat[5 * N:].view(N, 3))

    def _stream(self):
        return _VP(torch.cuda.current_stream(self.dev).cuda_stream)

    def _project(self, st):
        L = self.L
        call("lig_project_fwd_batch", _lib.LIG_F32, *L.args(), 1, _p(self.chol), _p(self.means),
             None, L.block, _p(self.xys), _p(self.ext), _p(self.con), _p(self.cnt), st)
        call("lig_cumsum_tiles", L.points, _p(self.cnt), _p(self.cum), _p(self.total),
             _p(self.cs_ws), self.cs_ws.numel(), st)

    def _count_intersections(self) -> int:
        self._project(self._stream())
        return int(self.total.item())

    def _size_capacity(self, m: int):
        cap = int(math.ceil(m * self.slack)) + 4096
        cap = min(cap, 2**31 - 1)
        self.capacity = cap
        self.gids = torch.empty(cap, dtype=torch.int32, device=self.dev)
        nb = _lib.lib.lig_bin_workspace_bytes(self.L.points, cap, self.L.tiles)
        self.bin_ws = torch.empty(nb, dtype=torch.uint8, device=self.dev)
        self.stats.capacity = cap
        self.graph = None
        self._graphs = {}

    # -------------------------------------------------------- the iteration
    def _bin(self, st):
        L = self.L
        self._project(st)
        call("lig_bin_batch", _lib.LIG_F32, *L.args(), L.block, _p(self.xys), _p(self.ext),
             _p(self.cum), _p(self.total), self.capacity, _p(self.bin_ws), self.bin_ws.numel(),
             _p(self.gids), _p(self.bins), _p(self.status), st)

    def _render(self, st):
        """Projection, binning and the forward rasterizer (render into self.img)."""
        L = self.L
        self._bin(st)
        call("lig_raster_fwd_batch", _lib.LIG_F32, *L.args(), L.block, _p(self.gids),
             _p(self.bins), _p(self.total), _p(self.cum), _p(self.xys), _p(self.con),
             _p(self.rgbs), None, int(self.persistent), _p(self.work), _p(self.r_ws),
             self.r_ws.numel(), _p(self.img), _p(self.wsum), None, None, None, _p(self.fin), st)

    def _enqueue_step(self, target: Optional[torch.Tensor] = None):
        """Forward with the loss fused in (self.img receives the masked
        difference clamp(x) - target, self.loss / self.per_image the losses),
        the backward from that difference, the projection backward and Adam.
        target: the concatenated [pixels, 3] target (default self.target)."""
        L = self.L
        st = self._stream()
        tgt = self.target if target is None else target
        self._bin(st)
        fwd = "lig_raster_fwd_l2_u8_batch" if tgt.dtype == torch.uint8 else "lig_raster_fwd_l2_batch"
        call(fwd, _lib.LIG_F32, *L.args(), L.block, _p(self.gids),
             _p(self.bins), _p(self.total), _p(self.cum), _p(self.xys), _p(self.con),
             _p(self.rgbs), None, _p(tgt), int(self.persistent), _p(self.work),
             _p(self.r_ws), self.r_ws.numel(), _p(self.partials), _p(self.img), None,
             _p(self.loss), _p(self.per_image), st)
        # no opacities: the backward reads no final indices, so the forward
        # neither tracks nor writes them
        call("lig_raster_bwd_diff_batch", _lib.LIG_F32, *L.args(), L.block, _p(self.gids),
             _p(self.bins), _p(self.total), _p(self.cum), _p(self.xys), _p(self.con),
             _p(self.rgbs), None, None, _p(self.img), _p(self.one), 0.0,
             int(self.persistent), _p(self.work), _p(self.r_ws), self.r_ws.numel(),
             _p(self.v_xy), _p(self.v_abs), _p(self.v_con), _p(self.g_rgbs), None, st)
        call("lig_project_bwd_batch", _lib.LIG_F32, *L.args(), 1, _p(self.chol), _p(self.means),
             None, L.block, _p(self.v_xy), 2, _p(self.v_con), 3, _p(self.g_chol),
             _p(self.g_means), st)
        call("lig_adam_step_batch", L.n, L.args()[3], _p(self.flat), _p(self.grad), _p(self.m),
             _p(self.v), self.lr, self.b1, self.b2, self.eps, _p(self.status), _p(self.steps),
             _p(self.skipped), _p(self.adam_scratch), self.adam_scratch.numel(), st)
        self.host_skipped.copy_(self.skipped, non_blocking=True)

    def _capture(self, target: Optional[torch.Tensor] = None):
        """Capture one iteration on a side stream.  capture_begin/end rather
        than the torch.cuda.graph context manager, which also runs the
        Python garbage collector (holding the GIL) and empties the allocator
        cache (a device-wide synchronisation) — both stall other threads of
        a server.  Thread-local capture mode lets those threads keep
        launching meanwhile."""
        cur = torch.cuda.current_stream(self.dev)
        side = torch.cuda.Stream(self.dev)
        side.wait_stream(cur)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            g.capture_begin(capture_error_mode="thread_local")
            try:
                self._enqueue_step(target)
            finally:
                g.capture_end()
        cur.wait_stream(side)
        self.stats.recaptures += 1
        return g

    def _recover(self):
        """A step overflowed the capacity (and was skipped): grow, recapture."""
        torch.cuda.current_stream(self.dev).synchronize()
        k = int(self.skipped.item())
        self.skipped.zero_()
        self.host_skipped.zero_()
        self.stats.skipped += k
        self._size_capacity(self._count_intersections())
        return k

    def _target_arg(self, target: Optional[torch.Tensor]) -> Optional[torch.Tensor]:
        if target is None:
            return None
        t = target.reshape(-1, 3)
        if (t.dtype not in (torch.float32, torch.uint8) or t.device != self.dev
                or not t.is_contiguous() or t.shape[0] != self.L.pixels):
            raise ValueError("target must be a contiguous float32 or uint8 CUDA tensor with the "
                             "batch's [pixels, 3] values")
        return t

    def step(self, target: Optional[torch.Tensor] = None):
        """One iteration (render, loss, backward, Adam) for every image; no
        host synchronisation unless a capacity overflow is being recovered.
        target (optional): fit against this [pixels, 3] buffer instead of the
        constructor's targets, read in place; one captured graph is kept per
        target buffer (a caller alternating two upload buffers replays two
        graphs, no copies)."""
        t = self._target_arg(target)
        key = 0 if t is None else t.data_ptr()
        g = self._graphs.get(key)
        if g is None and self.use_graph and self.stats.iters >= 2:
            if len(self._graphs) >= 4:
                self._graphs.clear()
            g = self._graphs[key] = self._capture(t)
            self.graph = g
        if g is not None:
            g.replay()
        else:
            self._enqueue_step(t)
        self.stats.iters += 1

    def step_checked(self, target: Optional[torch.Tensor] = None):
        """step(), then — if an earlier step was skipped for a capacity
        overflow (noticed without a sync through the pinned counter) — grow
        the capacity and redo the skipped steps."""
        self.step(target)
        while int(self.host_skipped[0]) > 0:
            for _ in range(self._recover()):
                self.step(target)

    def fit(self, iters: int, max_ahead: Optional[int] = None) -> BatchStats:
        """Run until `iters` Adam steps have been applied (skipped steps are
        redone after the capacity grows).  max_ahead: enqueue at most this
        many iterations ahead of the device (the host waits on an event,
        without the GIL), so that other threads' launches on the device —
        a server's renders — never queue behind a long chunk of fit work."""
        applied = 0
        pending = collections.deque()
        while True:
            while applied < iters:
                self.step()
                applied += 1
                if max_ahead:
                    ev = torch.cuda.Event()
                    ev.record(torch.cuda.current_stream(self.dev))
                    pending.append(ev)
                    if len(pending) > max_ahead:
                        pending.popleft().synchronize()
                if int(self.host_skipped[0]) > 0:  # pinned copy, no sync
                    applied -= self._recover()
            torch.cuda.current_stream(self.dev).synchronize()
            if int(self.skipped.item()) == 0:
                return self.stats
            applied -= self._recover()

    @torch.no_grad()
    def render(self) -> torch.Tensor:
        """Forward render of every image into the concatenated [pixels, 3] buffer."""
        self._render(self._stream())
        return self.img

    def images(self, buf: Optional[torch.Tensor] = None) -> List[torch.Tensor]:
        buf = self.img if buf is None else buf
        return [self.L.image(buf, i) for i in range(self.L.n)]

    def psnr(self) -> List[float]:
        """Per-image PSNR of the clamped render against the targets."""
        self.render()
        out = []
        for i in range(self.L.n):
            a = torch.clamp(self.L.image(self.img, i), 0, 1)
            b = self.L.image(self.target, i)
            if b.dtype == torch.uint8:
                b = b.float() / 255
            mse = torch.mean((a - b) ** 2).item()
            out.append(10 * math.log10(1.0 / max(mse, 1e-20)))
        return out

    def params_of(self, i: int):
        L = self.L
        return (L.points_of(self.means, i), L.points_of(self.chol, i), L.points_of(self.rgbs, i))

    def time_iters(self, iters: int) -> float:
        """Seconds per iteration over `iters` iterations (CUDA events)."""
        torch.cuda.synchronize(self.dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(iters):
            self.step()
        e.record()
        torch.cuda.synchronize(self.dev)
        return s.elapsed_time(e) / 1e3 / iters


# ------------------------------------------------------------------ tuning
_TUNED: Dict[str, dict] = {}


def _signature(targets, counts) -> str:
    return ";".join(f"{t.shape[0]}x{t.shape[1]}:{c}" for t, c in zip(targets, counts))


def autotune(targets: List[torch.Tensor], counts: Sequence[int], blocks=(8, 16, 32),
             walks=(False, True), iters: int = 5, cache_path: Optional[str] = None,
             **fit_kw) -> dict:
    """Time captured iterations of the batch for every tile size x tile walk
    and return the fastest {"block", "persistent", "s_per_iter", "table"}.
    Results are cached in-process and, with cache_path, in a JSON file keyed
    by the batch's sizes."""
    key = _signature(targets, counts)
    if key in _TUNED:
        return _TUNED[key]
    disk = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            disk = json.load(f)
        if key in disk:
            _TUNED[key] = disk[key]
            return disk[key]
    table = []
    for b in blocks:
        for pers in walks:
            fit = BatchedFit(targets, counts, block=b, persistent=pers, graph=True, **fit_kw)
            for _ in range(3):
                fit.step()
            t = fit.time_iters(iters)
            table.append({"block": b, "persistent": pers, "s_per_iter": t,
                          "capacity": fit.capacity})
            del fit
            torch.cuda.empty_cache()
    best = min(table, key=lambda r: r["s_per_iter"])
    res = {"block": best["block"], "persistent": best["persistent"],
           "s_per_iter": best["s_per_iter"], "table": table}
    _TUNED[key] = res
    if cache_path:
        disk[key] = res
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        with open(cache_path, "w") as f:
            json.dump(disk, f)
    return res


# --------------------------------------------------------------- workload
def uneven_batch(n_img: int = 64, density: float = 0.2, cap: int = 1_000_000,
                 teacher_density: float = 20000 / 512**2, noise_std: float = 0.02,
                 diag=(0.5, 4.0), block: int = 16, device="cuda", size_scale: float = 1.0):
    """The batched uneven-fit workload: image i has the shape
    synthetic.fit_shapes(i) (height log-uniform in [256, 4096], aspect
    U[0.5, 2]), a target rendered from round(teacher_density * H * W) seeded
    teacher Gaussians (seed 1000 + i) plus white noise (std noise_std,
    seed 2000 + i), clipped to [0, 1]; it is fitted (BatchedFit's default
    init, seed 3000 + i) with
    min(round(density * H * W), cap) Gaussians.  size_scale < 1 shrinks every
    side (tests).  Returns (targets, counts)."""
    from .gsplat2d import project_gaussians_cholesky, rasterize_gaussians
    targets, counts = [], []
    for i in range(n_img):
        h, w = synthetic.fit_shapes(i)
        h, w = max(16, int(round(h * size_scale))), max(16, int(round(w * size_scale)))
        nt = max(1, int(round(teacher_density * h * w)))
        mu, ch, co = synthetic.gaussians(nt, h, w, diag=diag, seed=1000 + i)
        with torch.no_grad():
            xys, ext, con, cnt = project_gaussians_cholesky(ch.to(device), mu.to(device), h, w,
                                                            block)
            img = rasterize_gaussians(xys, ext, con, cnt, co.to(device), None, h, w, block)[0]
            img = img + synthetic.white_noise(h, w, noise_std, seed=2000 + i).to(device)
        targets.append(torch.clamp(img, 0, 1).contiguous())
        counts.append(min(int(round(density * h * w)), cap))
    return targets, counts
