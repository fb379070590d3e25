"""Served reconstruction: a device-resident request loop with continuous batching.

Requests are FDK (fbp/reconFDK.m) or OS-PWLS (statsrecon/pwls/reconPwlsSeSqs.m,
initialised by reconFDK as the reference's scripts do) reconstructions, each with
its own geometry.  The server

* admits a request only when its HBM footprint fits the remaining budget and a
  slot is free (``hbm_budget`` bytes, ``max_active`` slots), in arrival order;
* gives each slot a persistent CUDA stream, and each admitted request its own
  stream-ordered projector plan (tables and scratch from the library pool,
  ctsim_plan_create_async), sinogram, weights and image, so requests never share
  mutable device memory and a result does not depend on what else runs;
* stores sinogram-sized data in float32, bfloat16 or float16 (FP32 arithmetic);
* issues work per request in units -- one FDK pass, or one OS-PWLS outer
  iteration (all subsets and the objective terms) -- with at most ``depth`` units
  in flight per request, so kernels of different requests overlap on the device
  and requests that arrive meanwhile are admitted as soon as slots and memory
  free up.  From the second iteration on, an OS-PWLS iteration is one replay of
  a CUDA graph captured from the first;
* records per-request latency (completion - arrival) for p50/p99;
* isolates failures: a request whose set-up or work raises, or whose plan reports a
  device-side error at retirement, ends as ``status == "failed"`` with the error text,
  and its slot and budget return to the server, while the other requests go on;
  ``cancel(rid)`` withdraws a request (pending: at once; active: after the units
  already on its stream).

OS-PWLS requests run a fixed number of iterations (the reference's stopping test
on the RMS change needs a host read per iteration).
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

from .geometry import CTGeometry, circular_betas


@dataclass
class ReconRequest:
    kind: str                      # "fdk" or "pwls"
    geom: CTGeometry
    sino: "object"                 # log sinogram, host numpy or device tensor [views, nu, nv]
    weights: "object" = None       # PWLS weights (reconPwlsSeSqs.m's w), same shape
    window: str = "hamming"        # FDK window (reconFDK.m default)
    beta: float = 1e3              # PWLS penalty weight
    delta: float = 0.01            # Huber parameter
    pfun: str = "huber"
    iterations: int = 10
    subsets: int = 12
    storage: str = "float32"       # storage type of the sinogram and weights on the device
    arrival: float = 0.0           # seconds, relative to the start of the run
    rid: int = 0
    # filled by the server
    result: "object" = None
    t_admit: float = float("nan")
    t_done: float = float("nan")
    status: str = "pending"        # "done", "failed" or "cancelled" when the server is through with it
    error: Optional[str] = None    # why it failed

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


STORAGE = ("float32", "bfloat16", "float16")


def _dtype(name):
    import torch
    return {"float32": torch.float32, "bfloat16": torch.bfloat16, "float16": torch.float16}[name]


def hbm_footprint(req: ReconRequest) -> int:
    """Upper bound of the device bytes a request holds while active: plan tables and
    prefix sums, FDK tables and filtered sinogram, the stored sinogram/weights and the FP32
    solver state.  Sinogram-sized data is held in the request's storage type (s bytes per
    pixel): the plan reads BF16/FP16 sinograms and pre-scaled residuals as they are, so
    no FP32 sinogram-sized scratch is allocated for a served request."""
    g = req.geom
    vox = g.nx * g.ny * g.nz
    pix = g.nu * g.nv * g.noViews
    s = 4 if req.storage == "float32" else 2
    L = 64
    while L < 2 * g.nu - 1:
        L *= 2
    xs = 8 * g.nx * g.ny * (g.nz + 4)  # column prefix sums (paired layout at most, or the padded plain one)
    plan = xs + 4 * g.nu * g.nv + g.nx * g.ny + 64 * g.noViews + 4096
    fdk = s * pix + 4 * g.nu * g.nv + 12 * L + 4 * g.nu * g.noViews + 4096  # filtered sinogram + tables
    image = 4 * vox
    if req.kind == "fdk":
        return plan + fdk + s * pix + image
    # while the solver is set up: the stored y and w (FP16 weights: FP32 until scaled) with
    # their per-subset copies, the FDK start image, one FP32 sinogram for A(1) and (w A(1))
    # ampv, the images x, x_new, x_old, precom, num (FP32) and the per-subset ax and wd
    w_in = 4 if req.storage == "float16" else s
    sub = 2 * 4 * g.nu * g.nv * math.ceil(g.noViews / req.subsets)
    return plan + fdk + (s + w_in + 2 * s + 4) * pix + 6 * image + sub + 4096


class _Active:
    """Device state and work of one admitted request (runs on its slot's stream)."""

    def __init__(self, req: ReconRequest, stream, device, graphs: bool = True, autotune: bool = False,
                 batched: bool = False):
        import torch
        self.req = req
        self.stream = stream
        self.device = device
        self.graphs = graphs
        self.events = deque()
        self.issued = 0
        self.solver = None
        self._graph = {}
        dt = _dtype(req.storage)
        self.plan = self.fdk = self.sino = None
        try:
            self._setup(req, stream, device, dt, autotune)
        except BaseException:
            self.release()  # what the set-up made so far (stream-ordered)
            raise
        # batched OS-PWLS: the server steps the request's sub-iterations together with the
        # other active requests' on its batch stream, after this set-up on the slot stream
        self.batched = batched and req.kind == "pwls"
        if self.batched:
            self.units = req.iterations * req.subsets
            self.sub = 0
            self.joined = False
            self.ready = torch.cuda.Event()
            self.ready.record(stream)

    def _setup(self, req, stream, device, dt, autotune):
        import torch
        from .fdk import FDK
        from .projector import Plan
        with torch.cuda.device(device), torch.cuda.stream(stream):
            self.plan = Plan(req.geom, device, stream=stream)
            self.fdk = FDK(req.geom, req.window, 1.0, device, plan=self.plan)
            # the sinogram goes to the device in its storage type (converted on the host:
            # half the copy for BF16/FP16, and no FP32 copy on the device)
            sino = _to_device(req.sino, device, dt)
            if req.kind == "fdk":
                self.sino = sino
                self.units = 1
            else:
                from .pwls import PwlsSolver
                # FP16 weights stay FP32 until the solver scales them into FP16's range
                w = _to_device(req.weights, device, torch.float32 if dt == torch.float16 else dt)
                x0 = self.fdk(sino)  # reconFDK start image, from the stored sinogram
                self.solver = PwlsSolver(sino, w, req.geom, req.beta, req.pfun, req.delta, req.subsets, x0,
                                         storage=dt, plan=self.plan, autotune=autotune)
                self.fdk.close()
                self.fdk = None
                self.units = req.iterations

    def in_flight(self) -> int:
        while self.events and self.events[0].query():
            self.events.popleft()
        return len(self.events)

    def _iteration(self):
        s = self.solver
        key = s.x.data_ptr()
        if self.issued == 0 or not self.graphs:
            for i in range(len(s.subsets)):
                s.subset_step(i)
            s.end_iteration()
            return
        g = self._graph.get(key)
        if g is None:
            import torch
            # record (nothing runs during capture), then replay; the swaps of x and
            # x_new done while recording leave the host-side pointers as after the run
            g = torch.cuda.CUDAGraph()
            g.capture_begin(capture_error_mode="thread_local")
            for i in range(len(s.subsets)):
                s.subset_step(i)
            s.end_iteration()
            g.capture_end()
            self._graph[key] = g
        else:
            for _ in range(len(s.subsets)):  # the pointer swaps of the replayed iteration
                s.x, s.xn = s.xn, s.x
        g.replay()

    def issue(self, to_host: bool = False):
        """Enqueue the next unit on this request's stream (asynchronous); after the last
        one, with ``to_host``, the copy of the image into pinned host memory."""
        import torch
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            if self.req.kind == "fdk":
                img = self.fdk(self.sino)
            else:
                self._iteration()
                img = self.solver.x
            if self.issued + 1 == self.units:
                if to_host:
                    host = torch.empty(img.shape, dtype=img.dtype, pin_memory=True)
                    host.copy_(img, non_blocking=True)
                    img = host
                self.req.result = img
            self.issued += 1
            ev = torch.cuda.Event()
            ev.record(self.stream)
            self.events.append(ev)

    def batch_pair(self):
        """(solver, subset index) of the next batched sub-iteration."""
        return self.solver, self.sub

    def batch_advance(self, to_host: bool, stream):
        """Book-keeping after a batched sub-iteration (on the batch stream): the
        iteration's objective terms after its last subset, the result after the last."""
        import torch
        self.sub += 1
        self.issued += 1
        if self.sub == self.req.subsets:
            self.sub = 0
            self.solver.end_iteration()
        if self.issued == self.units:
            img = self.solver.x
            if to_host:
                host = torch.empty(img.shape, dtype=img.dtype, pin_memory=True)
                host.copy_(img, non_blocking=True)
                img = host
            self.req.result = img
            ev = torch.cuda.Event()
            ev.record(stream)
            self.events.append(ev)

    def complete(self) -> bool:
        return self.issued == self.units and self.in_flight() == 0

    def check(self):
        """Raise if a kernel of this request set the plan's error flag (reads it on the
        request's stream, whose work is complete when this is called)."""
        self.plan.check()

    def release(self):
        """Free the request's device state (stream-ordered, no synchronisation)."""
        import torch
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            self._graph.clear()
            if self.fdk is not None:
                self.fdk.close()
                self.fdk = None
            self.solver = None
            self.sino = None
            if self.plan is not None:
                self.plan.close()


def _to_device(a, device, dtype=None):
    """A host array or tensor on the device, contiguous, converted to ``dtype`` (on the host
    for host data, rounding to nearest even as the device conversion does)."""
    import torch
    if isinstance(a, torch.Tensor):
        return a.to(device, dtype or a.dtype, non_blocking=True).contiguous()
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    if torch.cuda.is_available():
        t = t.pin_memory()
    return t.to(device, non_blocking=True)


class ReconServer:
    """Admission by HBM budget into ``max_active`` slots (one stream each); every tick
    issues one unit per active request with fewer than ``depth`` units in flight."""

    def __init__(self, hbm_budget: int = 150 * 2 ** 30, max_active: int = 8, depth: int = 2, device=None,
                 graphs: bool = True, activate: Optional[Callable] = None, clock: Optional[Callable] = None,
                 to_host: bool = False, admit_workers: int = 0, autotune: bool = False, batch_pwls: bool = False):
        self.budget = int(hbm_budget)
        self.max_active = int(max_active)
        self.depth = int(depth)
        self.graphs = graphs
        self.to_host = to_host
        self.pending = deque()
        self.active = []
        self.starting = []   # (future, request, slot): requests set up by the admission workers
        self._pool = None
        if admit_workers > 0:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(admit_workers, thread_name_prefix="ctsim-admit")
        self.used = 0
        self.peak_used = 0
        self.peak_active = 0       # the most requests set up or active at once
        self._active_sum = 0       # sum over ticks of the requests set up or active (mean concurrency)
        self._ticks = 0
        self.done = []
        self.failed = []      # requests that failed or were cancelled, in the order they ended
        self._cancel = set()  # rids to withdraw when their set-up finishes
        self.t0 = 0.0
        self._clock = clock or time.perf_counter
        if activate is None:
            import torch
            self.device = torch.device("cuda", torch.cuda.current_device() if device is None else
                                       (torch.device(device).index or 0))
            self.streams = [torch.cuda.Stream(device=self.device) for _ in range(self.max_active)]
            self.batch_stream = torch.cuda.Stream(device=self.device) if batch_pwls else None
            activate = lambda req, slot: _Active(req, self.streams[slot], self.device, self.graphs, autotune,
                                                 batch_pwls)
        else:
            self.streams = [None] * self.max_active
        self._activate = activate
        self.batch_pwls = batch_pwls
        self._tick_events = deque()
        self._free_slots = list(range(self.max_active))[::-1]
        self._slot_of = {}

    def now(self) -> float:
        return self._clock() - self.t0

    def submit(self, req: ReconRequest):
        if req.kind not in ("fdk", "pwls"):
            raise ValueError(f"unknown request kind {req.kind!r}")
        if req.storage not in STORAGE:
            raise ValueError(f"unknown storage type {req.storage!r}")
        if hbm_footprint(req) > self.budget:
            raise ValueError(f"request {req.rid} needs more than the whole HBM budget")
        self.pending.append(req)

    def _admit(self):
        while self.pending and self._free_slots:
            req = self.pending[0]
            if req.arrival > self.now():
                break
            need = hbm_footprint(req)
            if self.used + need > self.budget:
                break
            self.pending.popleft()
            req.t_admit = self.now()
            slot = self._free_slots.pop()
            self.used += need
            self.peak_used = max(self.peak_used, self.used)
            if self._pool is None:
                try:
                    a = self._activate(req, slot)
                except Exception as exc:  # this request only: its slot and budget return
                    self._end(req, slot, "failed", exc)
                    continue
                self._start(a, slot)
            else:
                self.starting.append((self._pool.submit(self._activate_in_worker, req, slot), req, slot))

    def _activate_in_worker(self, req, slot):
        # the set-up work is ordered on the slot's stream, ahead of the units the main
        # thread issues there later
        return self._activate(req, slot)

    def _start(self, a, slot):
        self._slot_of[id(a)] = slot
        self.active.append(a)

    def _end(self, req, slot, status, exc=None):
        """A request the server is through with other than by success: its slot and its
        share of the budget return."""
        req.status = status
        req.error = None if exc is None else f"{type(exc).__name__}: {exc}"
        req.t_done = self.now()
        req.result = None
        self.used -= hbm_footprint(req)
        self._free_slots.append(slot)
        self._cancel.discard(req.rid)
        self.failed.append(req)

    def _collect_started(self):
        keep = []
        for fut, req, slot in self.starting:
            if not fut.done():
                keep.append((fut, req, slot))
                continue
            try:
                a = fut.result()
            except Exception as exc:  # a set-up error ends this request only
                self._end(req, slot, "failed", exc)
                continue
            if req.rid in self._cancel:
                a.release()
                self._end(req, slot, "cancelled")
            else:
                self._start(a, slot)
        self.starting = keep

    def cancel(self, rid: int) -> bool:
        """Withdraw request ``rid``: a pending one at once, one being set up when its set-up
        finishes, an active one once the units already on its stream are done (no more
        are issued).  False if the server does not hold it (unknown or finished)."""
        for i, r in enumerate(self.pending):
            if r.rid == rid:
                del self.pending[i]  # by position: requests hold arrays, so no equality test
                r.status, r.t_done = "cancelled", self.now()
                self.failed.append(r)
                return True
        if any(req.rid == rid for _, req, _ in self.starting):
            self._cancel.add(rid)
            return True
        for a in self.active:
            if a.req.rid == rid:
                a.cancelled = True
                return True
        return False

    def _retire(self):
        keep = []
        for a in self.active:
            failed = getattr(a, "failed", None)
            cancelled = getattr(a, "cancelled", False)
            if failed is None and not (cancelled and a.in_flight() == 0) and not a.complete():
                keep.append(a)
                continue
            slot = self._slot_of.pop(id(a))
            if failed is None and not cancelled:
                try:
                    a.check()  # the plan's device-side error flag
                except Exception as exc:
                    failed = exc
            try:
                a.release()
            except Exception as exc:
                failed = failed or exc
            if failed is not None or cancelled:
                self._end(a.req, slot, "failed" if failed is not None else "cancelled", failed)
            else:
                a.req.t_done = self.now()
                a.req.status = "done"
                self.used -= hbm_footprint(a.req)
                self._free_slots.append(slot)
                self.done.append(a.req)
        self.active = keep

    @property
    def mean_active(self) -> float:
        """Requests set up or active per scheduler tick, on average."""
        return self._active_sum / self._ticks if self._ticks else 0.0

    def tick(self):
        self._admit()
        if self.starting:
            self._collect_started()
        n = len(self.active) + len(self.starting)
        self.peak_active = max(self.peak_active, n)
        self._active_sum += n
        self._ticks += 1
        for a in self.active:
            if getattr(a, "cancelled", False) or getattr(a, "failed", None) is not None:
                continue
            if not getattr(a, "batched", False) and a.issued < a.units and a.in_flight() < self.depth:
                try:
                    a.issue(self.to_host)
                except Exception as exc:  # retired (and released) as failed below
                    a.failed = exc
        if self.batch_pwls:
            self._batched_tick()
        self._retire()

    def _batched_tick(self):
        """One sub-iteration of every active OS-PWLS request in one batched A and one
        batched A^T launch on the batch stream (at most ``depth`` ticks in flight)."""
        import torch
        from .pwls import batched_subset_steps
        while self._tick_events and self._tick_events[0].query():
            self._tick_events.popleft()
        if len(self._tick_events) >= self.depth:
            return
        pw = [a for a in self.active if getattr(a, "batched", False) and a.issued < a.units and
              not getattr(a, "cancelled", False) and getattr(a, "failed", None) is None]
        if not pw:
            return
        bs = self.batch_stream
        with torch.cuda.device(self.device), torch.cuda.stream(bs):
            for a in pw:
                if not a.joined:
                    bs.wait_event(a.ready)
                    a.joined = True
            try:
                batched_subset_steps([a.batch_pair() for a in pw])
                for a in pw:
                    a.batch_advance(self.to_host, bs)
            except Exception as exc:  # the requests of this batched step fail together
                for a in pw:
                    a.failed = exc
                return
            ev = torch.cuda.Event()
            ev.record(bs)
            self._tick_events.append(ev)

    def close(self):
        if self._pool is not None:
            self._pool.shutdown(wait=True)
            self._pool = None

    def run(self, requests, time_limit: Optional[float] = None, idle_sleep: float = 2e-4):
        """Serve requests (by arrival time) until each is done, failed or cancelled; returns
        the ones that succeeded, in completion order (``failed`` holds the others)."""
        for r in sorted(requests, key=lambda r: r.arrival):
            self.submit(r)
        self.t0 = self._clock()
        try:
            while self.pending or self.active or self.starting:
                self.tick()
                if self.active or self.starting or (self.pending and self.pending[0].arrival > self.now()):
                    time.sleep(idle_sleep)
                if time_limit is not None and self.now() > time_limit:
                    break
        finally:
            self.close()
        return self.done


def serve_sequential(requests, device=None):
    """The plain single-instance path: one request at a time through the public FP32
    API (reconFDK, reconFDK + reconPwlsSeSqs), host arrays in and out.  Sets result,
    t_done (seconds from the start) and returns the requests."""
    from .fdk import reconFDK
    from .pwls import reconPwlsSeSqs
    t0 = time.perf_counter()
    for r in requests:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        r.t_admit = time.perf_counter() - t0
        y = np.asarray(r.sino, dtype=np.float32)
        if r.kind == "fdk":
            r.result = reconFDK(y, r.geom, r.window)
        else:
            import torch
            x0 = reconFDK(y, r.geom, r.window)
            x, _, _ = reconPwlsSeSqs(torch.from_numpy(y).cuda(), torch.from_numpy(np.asarray(r.weights)).cuda(),
                                     r.geom, r.beta, r.pfun, r.iterations, r.delta, r.subsets,
                                     torch.from_numpy(x0).cuda(), stopCrt=-1.0)
            r.result = x.cpu().numpy()
        r.t_done = time.perf_counter() - t0
        # the plans and FDK objects the public API cached on the geometry
        for f in r.geom.__dict__.pop("_fdk", {}).values():
            f.close()
        for p in r.geom.__dict__.pop("_plans", {}).values():
            p.close()
    return requests


def latency_stats(done, t_total: float):
    lat = np.array([r.latency for r in done])
    if lat.size == 0:
        return {"requests": 0}
    return {"requests": int(lat.size), "req_per_s": float(lat.size / t_total),
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3)}


# ---------------------------------------------------------------------------
# Seeded synthetic request stream
# ---------------------------------------------------------------------------
def random_geometry(rng, scale: float = 1.0) -> CTGeometry:
    """Uneven instance geometry: volumes 128^2x64 .. 384^2x160 (voxel 0.5-1.0 mm), 180-720
    views, detectors 256x64 .. 768x256 (0.8-1.6 mm); ~20% short scan, ~20% offset
    detector.  ``scale`` shrinks every size."""
    n = max(16, int(rng.integers(128, 385) * scale) // 16 * 16)
    nz = max(8, int(rng.integers(64, 161) * scale) // 8 * 8)
    vox = float(rng.uniform(0.5, 1.0))
    nu = max(32, int(rng.integers(256, 769) * scale) // 16 * 16)
    nv = max(16, int(rng.integers(64, 257) * scale) // 8 * 8)
    # detector pitch covering the volume at magnification 1.5
    du = max(0.8, min(1.6, 1.5 * n * vox * 1.5 / nu))
    dv = max(0.8, min(1.6, 1.5 * nz * vox * 1.6 / nv))
    views = max(8, int(rng.integers(180, 721) * scale) // 4 * 4)
    short = bool(rng.random() < 0.2)
    offset = (not short) and bool(rng.random() < 0.25)
    if short:
        fan = 2 * math.atan(nu * du / 2 / 1500.0)
        betas = np.linspace(0.0, math.pi + fan, views)
    else:
        betas = circular_betas(views)
    return CTGeometry((n, n, nz), (vox, vox, vox), (0, 0, 0), (nu, nv), (du, dv), (nu / 4.0 if offset else 0.0, 0),
                      1000.0, 500.0, 1500.0, betas, shortScan=short)


def config1_geometry() -> CTGeometry:
    """The plain small reconstruction: 128x128x64 at 1 mm, 360 views over 2 pi, flat
    256x96 detector at 1.6 mm, SAD 1000 mm, SDD 1500 mm."""
    return CTGeometry((128, 128, 64), (1.0, 1.0, 1.0), (0, 0, 0), (256, 96), (1.6, 1.6), (0, 0), 1000.0, 500.0,
                      1500.0, circular_betas(360))


def make_requests(n: int, seed: int = 0, fdk_fraction: float = 0.7, storage: str = "bfloat16", scale: float = 1.0,
                  iterations: int = 10, subsets: int = 12, rate: Optional[float] = None, i0: float = 1e5,
                  sizes: str = "uneven"):
    """``n`` requests (FDK with probability ``fdk_fraction``, else OS-PWLS) over
    random_geometry (``sizes="uneven"``) or the config-1 geometry (``sizes="config1"``),
    with Poisson arrivals at ``rate`` req/s (all at 0 if None).
    The data: a random ellipsoid phantom projected with the SF projector, Poisson
    counts at ``i0`` photons, y = log(i0 / max(counts, 10)) and w = counts
    (computeWeightsPwls with r = v = 0 on counts)."""
    import torch
    from .phantom import ellipsoid_phantom, to_projector_units
    from .projector import Plan
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    t, reqs = 0.0, []
    for rid in range(n):
        if rate is not None:
            t += float(rng.exponential(1.0 / rate))
        g = random_geometry(rng, scale) if sizes == "uneven" else config1_geometry()
        r_xy = 0.4 * g.nx * g.reconSpacing[0]
        x = to_projector_units(ellipsoid_phantom(g, 6, (0.015, 0.035), 0.02, r_xy, 0.6 * r_xy,
                                                 0.3 * g.nz * g.reconSpacing[2], (2.0, 8.0),
                                                 int(rng.integers(1 << 30))))
        p = Plan(g)
        line = p.project(torch.from_numpy(x).cuda(), "tf")
        p.close()
        counts = torch.poisson(i0 * torch.exp(-line), generator=gen)
        y = torch.log(i0 / torch.clamp(counts, min=10.0)).cpu().numpy()
        kind = "fdk" if rng.random() < fdk_fraction else "pwls"
        reqs.append(ReconRequest(kind, g, y, counts.cpu().numpy() if kind == "pwls" else None, storage=storage,
                                 arrival=t, rid=rid, iterations=iterations, subsets=subsets))
    return reqs
