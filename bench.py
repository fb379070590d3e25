#!/usr/bin/env python
"""Benchmark: distance-driven cone-beam A and A^T on one B200.

Workload (default): the full-size plain reconstruction geometry -- volume
512x512x256 at 0.5 mm (seeded ellipsoid phantom), 720 views over 2 pi, flat
detector 1024x384 at 0.8 mm, SAD 1000 mm, SDD 1500 mm.  One step = one
distance-driven forward projection A x plus one matched backprojection A^T y
(y = log-transformed Poisson data).  Metric: GVoxel-views/s = 2 * nx*ny*nz*views
per step / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: the projector does not exchange data between GPUs (replicas only):
every rank runs the same workload on its own GPU; the time is the max over
ranks and ``value`` counts the work of all ranks.

``--impl reference`` times the reference's own CPU C (geom/cbct, compiled
unmodified into oracle/_ref) over all host cores on a bounded sample of views
of the same workload (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GVoxel-views/s for DD A and A^T"
UNIT = "GVoxel-views/s"


def rank_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def max_over_ranks(ms: float, dist: bool, device) -> float:
    """The slowest rank's time: every rank of a replica run calls this in the same order
    (an all-reduce with MAX); a single process returns its own."""
    if not dist:
        return ms
    import torch
    import torch.distributed as td
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def replica_value(vv_per_step: float, steps: int, world: int, total_ms: float) -> float:
    """Whole-job GVoxel-views/s: every rank runs `steps` A + A^T steps of `vv_per_step`
    voxel-views each, and the job takes the slowest rank's `total_ms`."""
    return 2.0 * vv_per_step * steps * world / (total_ms / 1e3) / 1e9


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel: str):
    """DRAM bytes per launch recorded from an ncu capture (profiles/*.txt line 'traffic_bytes_per_launch <k> <n>')."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith(".txt"):
            continue
        with open(os.path.join(pdir, fn)) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 3 and parts[0] == "traffic_bytes_per_launch" and parts[1] == kernel:
                    return float(parts[2])
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        import torch
        uuid = None
        try:
            uuid = "GPU-" + str(torch.cuda.get_device_properties(self.dev).uuid)
        except Exception:
            pass
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
        if uuid:
            cmd += ["-i", uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        mhz, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [s.strip() for s in line.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(mhz)) if mhz else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(mhz)}


def make_workload(views: int = 0, consecutive: bool = False):
    """The benchmark workload; ``views`` > 0 keeps every (720/views)-th view, or with
    ``consecutive`` the first ``views`` views (profiling captures: the scan's own view
    spacing, so that neighbouring views share candidate columns in L2 as in a full run)."""
    from dataclasses import replace
    from ctsim_b200.phantom import config2, to_projector_units
    g, x_mm = config2(seed=2)
    if views:
        s = 1 if consecutive else max(1, g.noViews // views)
        g = replace(g, betas=g.betas[::s][:views].copy(), couchZ=g.couchZ[::s][:views].copy())
    return g, to_projector_units(x_mm)


def sample_views(g, nviews):
    """Indices of the CPU sample's views: every (views / nviews)-th view of the scan."""
    return np.arange(0, g.noViews, max(1, g.noViews // nviews))[:nviews]


def cpu_reference_sample(g, x, y, keep_outputs=False):
    """Time the reference C (all host cores) on a bounded sample of the workload's views.
    With ``keep_outputs`` the sample's A and A^T results come back too (under "outputs",
    with the view indices), for the parity check of the GPU step."""
    from oracle.bindings import ref_available, ref_cbct, oracle_cbct
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    nxyz = g.nx * g.ny * g.nz
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 16 << 30
    # the threaded backprojection keeps one image per thread
    threads = max(1, min(ncores, int(avail * 0.5 // (nxyz * 4))))
    from dataclasses import replace
    idx = sample_views(g, threads)
    if not ref_available():  # the oracle port, single-threaded, one view
        threads, idx = 1, idx[:1]
    gs = replace(g, betas=g.betas[idx].copy(), couchZ=g.couchZ[idx].copy())
    ys = np.ascontiguousarray(y[idx])
    if ref_available():
        kind = "reference"
        t0 = time.perf_counter()
        a = ref_cbct("proj,dd", gs, x, nthreads=threads)
        at = ref_cbct("back,dd", gs, ys, nthreads=threads)
        dt = time.perf_counter() - t0
    else:
        kind = "port"
        t0 = time.perf_counter()
        a = oracle_cbct("proj,dd", gs, x)
        at = oracle_cbct("back,dd", gs, ys)
        dt = time.perf_counter() - t0
    vv = 2.0 * nxyz * gs.noViews
    out = {"value": vv / dt / 1e9, "unit": UNIT, "cores": threads, "kind": kind,
           "sample": f"DD A then A^T of {gs.noViews} of the {g.noViews} views on the full "
                     f"{g.nx}x{g.ny}x{g.nz} volume ({dt:.1f} s)"}
    if keep_outputs:
        out["outputs"] = (idx, gs, a, at)
    return out


def rel_l2(a, b):
    a64, b64 = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a64 - b64) / max(np.linalg.norm(b64), 1e-300))


def step_parity(plan_cls, sino, yd, sample):
    """The timed step's own results against the reference C on the CPU sample's views:
    A from the step's sinogram at those views, A^T from a plan of those views over the
    step's data (the full A^T sums all views; the CPU sample backprojects its own)."""
    import torch
    idx, gs, ref_a, ref_at = sample
    ours_a = sino[torch.as_tensor(idx, device=sino.device)].cpu().numpy()
    ys = yd[torch.as_tensor(idx, device=yd.device)].contiguous()
    ours_at = plan_cls(gs).backproject(ys, "dd").cpu().numpy()
    return {"views": [int(i) for i in idx], "against": "reference C" if len(idx) > 1 else "oracle",
            "A_rel_l2": rel_l2(ours_a, ref_a), "AT_rel_l2": rel_l2(ours_at, ref_at), "bar": 1e-5}


def run_reference(args):
    rank, local, world = rank_info()
    if rank != 0:
        return
    g, x = make_workload()
    rng = np.random.default_rng(3)
    y = rng.random(g.sino_shape, dtype=np.float32)
    for _ in range(args.warmup):
        cpu_reference_sample(g, x, y)
    vals, cb = [], None
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cb = cpu_reference_sample(g, x, y)
        vals.append(cb["value"])
    wall = time.perf_counter() - t0
    value = float(np.mean(vals))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "DD A + A^T, 512x512x256 @0.5mm, 720 views, flat 1024x384 @0.8mm, SAD 1000, SDD 1500",
                       "sample": cb["sample"]},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cb["cores"], "kind": cb["kind"],
                             "sample": cb["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    from ctsim_b200 import _lib
    from ctsim_b200.projector import Plan

    rank, local, world = rank_info()
    dist = world > 1
    if dist:
        import torch.distributed as td
        from datetime import timedelta
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    g, x = make_workload(args.views, args.consecutive)
    vv = float(g.nx * g.ny * g.nz * g.noViews)
    plan = Plan(g)
    xd = torch.from_numpy(x).to(dev)
    # log-transformed Poisson data: counts ~ Poisson(I0 exp(-A x)), y = log(I0 / max(counts, 10))
    with torch.no_grad():
        p = plan.project(xd, "dd")
        gen = torch.Generator(device=dev)
        gen.manual_seed(1234 + rank)
        counts = torch.poisson(1e5 * torch.exp(-p), generator=gen)
        yd = torch.log(1e5 / torch.clamp(counts, min=10.0)).contiguous()
        del p, counts
    sino = torch.empty(g.sino_shape, dtype=torch.float32, device=dev)
    img = torch.empty(g.image_shape, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def step():
        plan.project(xd, "dd", out=sino)
        plan.backproject(yd, "dd", out=img)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    plan.check()

    # timed region
    K = args.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    clocks = ClockSampler(dev)
    if dist:
        td.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for i in range(K):
        ev[i][0].record(stream)
        plan.project(xd, "dd", out=sino)
        ev[i][1].record(stream)
        plan.backproject(yd, "dd", out=img)
        ev[i][2].record(stream)
    end.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist:
        td.barrier()
    total_ms = start.elapsed_time(end)
    t_a = float(np.mean([e[0].elapsed_time(e[1]) for e in ev]))
    t_b = float(np.mean([e[1].elapsed_time(e[2]) for e in ev]))
    total_ms = max_over_ranks(total_ms, dist, dev)
    ms_per_step = total_ms / K
    value = replica_value(vv, K, world, total_ms)

    # roofline of the dominant kernel (streaming model: every view reads the volume and writes/reads its view)
    peak, peak_src = measured_peaks()
    alg_bytes = g.noViews * (g.nx * g.ny * g.nz * 4 + g.nu * g.nv * 4)
    proj_name = "proj_staged_kernel" if plan.tuning["proj_layout"] == 3 else "proj_kernel"
    dom, t_dom = (proj_name, t_a) if t_a >= t_b else ("back_kernel", t_b)
    achieved = alg_bytes / (t_dom / 1e3) / 1e9
    traffic = profile_traffic(dom)

    # end to end through the drop-in C ABI with pinned host buffers (H2D/D2H inside the timed region)
    L = _lib.load()
    h_img = torch.from_numpy(x).pin_memory()
    h_sino_in = yd.cpu().pin_memory()
    h_sino_out = torch.empty(g.sino_shape, dtype=torch.float32).pin_memory()
    h_img_out = torch.empty(g.image_shape, dtype=torch.float32).pin_memory()
    betas = np.ascontiguousarray(g.betas)
    couch = np.ascontiguousarray(g.couchZ)
    mp = np.ascontiguousarray(g.map)
    sc = g.scalars()

    def e2e_step(img_in, sino_out, img_out, sino_in):
        ok1 = L.ctsim_proj_dd(*sc, betas.ctypes.data, couch.ctypes.data, g.flatPanel, img_in, sino_out,
                              mp.ctypes.data)
        ok2 = L.ctsim_back_dd(*sc, betas.ctypes.data, couch.ctypes.data, g.flatPanel, img_out, sino_in,
                              mp.ctypes.data)
        if not (ok1 and ok2):
            raise RuntimeError(_lib.last_error())

    pinned = (h_img.data_ptr(), h_sino_out.data_ptr(), h_img_out.data_ptr(), h_sino_in.data_ptr())
    e2e_val = e2e_pageable = None
    if not args.no_e2e:
        e2e_val, _ = run_e2e(lambda: e2e_step(*pinned), K, dist, dev, vv, world)
        # pageable host memory, what a MATLAB MEX caller hands over (mxArray data)
        p_img, p_sino_in = h_img.numpy().copy(), h_sino_in.numpy().copy()
        p_sino_out = np.empty(g.sino_shape, np.float32)
        p_img_out = np.empty(g.image_shape, np.float32)
        pageable = (p_img.ctypes.data, p_sino_out.ctypes.data, p_img_out.ctypes.data, p_sino_in.ctypes.data)
        e2e_pageable, _ = run_e2e(lambda: e2e_step(*pageable), K, dist, dev, vv, world)
        del p_img, p_sino_in, p_sino_out, p_img_out
    nbytes_img = g.nx * g.ny * g.nz * 4
    nbytes_sino = g.nu * g.nv * g.noViews * 4

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_sample(g, x, yd.cpu().numpy(), keep_outputs=True)
        parity = step_parity(Plan, sino, yd, cpu.pop("outputs"))

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
                "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "DD A + A^T, 512x512x256 @0.5mm, 720 views, flat 1024x384 @0.8mm, "
                                       "SAD 1000, SDD 1500 (seeded 20-ellipsoid phantom, log Poisson data I0=1e5)",
                           "parallelism": f"replicas x{world}",
                           "l2": "inputs larger than L2 (268 MB volume, 1.13 GB sinogram), no flush"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "kernel": dom,
                             "peak_source": peak_src,
                             "model": "views*(nx*ny*nz*4 + nu*nv*4) bytes per launch"},
                "kernels_ms": {"A (prefix+proj)": t_a, "A^T (back)": t_b},
                "A_gvv_s": vv / (t_a / 1e3) / 1e9, "AT_gvv_s": vv / (t_b / 1e3) / 1e9,
                "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": nbytes_img + nbytes_sino,
                        "d2h_bytes_per_step": nbytes_sino + nbytes_img, "steps": K,
                        "api": "ctsim_proj_dd + ctsim_back_dd (host pointers, pinned)",
                        "pageable_value": e2e_pageable},
                "parity": parity,
                "gpu_launches": 4 * K,
                "clocks": clk,
                "cpu_baseline": cpu}
        if args.extras:
            line["extras"] = extras(plan, xd, yd, sino, img, vv)
        if world == 1 and not (args.no_serving and args.no_config1):
            del plan, xd, yd, sino, img
            torch.cuda.empty_cache()
            if not args.no_config1:
                try:
                    line["config1"] = config1_leg(K)
                except Exception as exc:  # a side figure: the headline line is printed either way
                    line["config1"] = {"error": f"{type(exc).__name__}: {exc}"}
            if not args.no_serving:
                line["serving"] = serving_leg(args.seed)
        print(json.dumps(line), flush=True)
    if dist:
        td.destroy_process_group()


def run_e2e(e2e_step, K, dist, dev, vv, world):
    """K synchronous drop-in steps after one untimed call (wall clock: the C ABI returns
    after its device->host copies); the slowest rank's time."""
    e2e_step()
    if dist:
        import torch.distributed as td
        td.barrier()
    t0 = time.perf_counter()
    for _ in range(K):
        e2e_step()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / K * 1e3, dist, dev) / 1e3
    return replica_value(vv, 1, world, e2e_s * 1e3), e2e_s


def extras(plan, xd, yd, sino, img, vv):
    """Other rows of the path on the same workload: SF pair and FDK backprojection."""
    import torch
    out = {}
    for name, fn in (("SF A", lambda: plan.project(xd, "tf", out=sino)),
                     ("SF A^T", lambda: plan.backproject(yd, "tf", out=img)),
                     ("FDK back,hpd", lambda: plan.backproject(yd, "hpd", out=img))):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(3):
            fn()
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / 3
        out[name] = {"ms": ms, "gvv_s": vv / (ms / 1e3) / 1e9}
    return out


def config1_leg(steps: int):
    """DD A + A^T on the 128x128x64 / 360-view / 256x96 scan (volume 4 MB, sinogram 35 MB,
    both L2-resident): y = A x + N(0, 0.01^2), ``steps`` timed steps, each preceded by a
    512 MB write that flushes L2, so every step starts from HBM.  Events bracket A and
    A^T only, on the launching stream."""
    import torch
    from ctsim_b200.phantom import config1, to_projector_units
    from ctsim_b200.projector import Plan
    g, x_mm = config1(seed=1)
    vv = float(g.nx * g.ny * g.nz * g.noViews)
    plan = Plan(g)
    xd = torch.from_numpy(to_projector_units(x_mm)).cuda()
    gen = torch.Generator(device=xd.device)
    gen.manual_seed(11)
    with torch.no_grad():
        yd = plan.project(xd, "dd")
        yd = (yd + 0.01 * torch.randn(yd.shape, generator=gen, device=xd.device)).contiguous()
    sino = torch.empty_like(yd)
    img = torch.empty_like(xd)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=xd.device)
    stream = torch.cuda.current_stream()
    for _ in range(3):
        plan.project(xd, "dd", out=sino)
        plan.backproject(yd, "dd", out=img)
    torch.cuda.synchronize()
    plan.check()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    for e in ev:
        flush.fill_(1)
        e[0].record(stream)
        plan.project(xd, "dd", out=sino)
        e[1].record(stream)
        plan.backproject(yd, "dd", out=img)
        e[2].record(stream)
    torch.cuda.synchronize()
    t_a = float(np.mean([e[0].elapsed_time(e[1]) for e in ev]))
    t_b = float(np.mean([e[1].elapsed_time(e[2]) for e in ev]))
    ms = t_a + t_b
    out = {"workload": "DD A + A^T, 128x128x64 @1mm, 360 views, flat 256x96 @1.6mm, SAD 1000, SDD 1500 "
                       "(seeded 12-ellipsoid phantom, y = A x + N(0, 0.01^2))",
           "value": vv / (ms / 1e3) / 1e9, "unit": UNIT, "ms_per_step": ms, "steps": steps,
           "kernels_ms": {"A (prefix+proj)": t_a, "A^T (back)": t_b},
           "l2": "512 MB write before each step (volume 4 MB and sinogram 35 MB fit in L2)"}
    del plan, xd, yd, sino, img, flush
    torch.cuda.empty_cache()
    return out


def served_accuracy(served, plain):
    """Relative RMSE (||a - b|| / ||b||) of each served BF16-storage image against the plain
    FP32 path's image of the same request, per request kind (max and median).  The FP32
    path itself is within 2e-6 of the FP64 oracle on these shapes (tests/test_precision.py)."""
    ref = {r.rid: r for r in plain}
    errs = {"fdk": [], "pwls": []}
    for r in served:
        a = r.result
        a = a.float().numpy() if hasattr(a, "float") else np.asarray(a, np.float32)
        b = np.asarray(ref[r.rid].result, np.float64)
        errs[r.kind].append(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)))
    return {"against": "plain FP32 path, same requests", "metric": "relative RMSE",
            **{k: {"max": max(v), "median": float(np.median(v)), "n": len(v)} for k, v in errs.items() if v}}


def serving_leg(seed: int, unique: int = 40, total: int = 200, budget_s: float = 60.0):
    """The served stream at config-1 sizes (128^2 x 64, 360 views, 256 x 96): a seeded 70/30
    FDK / OS-PWLS (10 iterations x 12 subsets) mix of `total` requests (`unique` distinct
    phantoms, cycled), BF16 storage with FP32 arithmetic through ReconServer, against the
    plain single-instance FP32 path (reconFDK / reconPwlsSeSqs one request at a time, host
    arrays in and out) on the same requests.  Closed loop for req/s; Poisson arrivals at
    50% and 80% of the served capacity for p50/p99 latency.  Every arm runs the same
    requests after one untimed pass over the distinct ones; the leg stops short of
    `budget_s` seconds of serving (the arms it reached are reported)."""
    import copy
    import torch
    from ctsim_b200.serving import ReconServer, latency_stats, make_requests, serve_sequential
    t_start = time.perf_counter()
    base = make_requests(unique, seed=seed, sizes="config1", iterations=10, subsets=12)
    reqs = []
    for i in range(total):
        r = copy.copy(base[i % unique])
        r.rid = i
        reqs.append(r)

    def fresh(rs, storage, arrivals=None):
        out = []
        for i, r in enumerate(rs):
            c = copy.copy(r)
            c.storage, c.result, c.status = storage, None, "pending"
            c.arrival = 0.0 if arrivals is None else float(arrivals[i])
            out.append(c)
        return out

    def served(rs):
        srv = ReconServer(max_active=8, to_host=True, admit_workers=2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        done = srv.run(rs)
        torch.cuda.synchronize()
        return done, time.perf_counter() - t0

    serve_sequential(fresh(base, "float32"))  # warm-up: plans, pools, pinned buffers
    served(fresh(base, "bfloat16"))
    out = {"workload": "config-1 geometry (128^2x64 @1mm, 360 views, 256x96 @1.6mm), 70/30 FDK/OS-PWLS "
                       "(10 x 12 subsets), seeded ellipsoid phantoms, Poisson counts I0=1e5",
           "requests": total, "distinct": unique, "fdk": sum(r.kind == "fdk" for r in reqs),
           "pwls": sum(r.kind == "pwls" for r in reqs), "slots": 8}
    clocks = ClockSampler(0)
    clocks.start()
    t0 = time.perf_counter()
    plain = serve_sequential(fresh(reqs, "float32"))
    t_plain = time.perf_counter() - t0
    done16, t16 = served(fresh(reqs, "bfloat16"))
    cap = len(done16) / t16
    out.update({"plain_fp32_req_per_s": len(plain) / t_plain, "served_bf16_req_per_s": cap,
                "speedup_served_bf16_vs_plain_fp32": cap / (len(plain) / t_plain),
                "closed_loop": latency_stats(done16, t16),
                "accuracy": served_accuracy(done16, plain)})
    rng = np.random.default_rng(seed)
    sweep = []
    for frac in (0.5, 0.8):
        if time.perf_counter() - t_start > budget_s:
            break
        rate = frac * cap
        arr = np.cumsum(rng.exponential(1.0 / rate, size=total))
        d, t = served(fresh(reqs, "bfloat16", arr))
        st = latency_stats(d, t)
        st.update({"offered_req_per_s": rate, "load_fraction": frac})
        sweep.append(st)
    out["open_loop"] = sweep
    out["clocks"] = clocks.stop()
    out["seconds"] = time.perf_counter() - t_start
    return out


def run_serving(args):
    """Served reconstruction: a seeded mix of FDK and OS-PWLS requests (random_geometry:
    volumes 128^2x64 .. 384^2x160, 180-720 views, 20% short scan, 20% offset detector;
    70% FDK, 30% OS-PWLS with 12 subsets x 10 iterations) through ReconServer, against the
    plain single-instance FP32 path (serve_sequential: reconFDK / reconPwlsSeSqs one
    request at a time, host arrays in and out).  Closed loop (all requests queued at 0)
    for throughput, then Poisson arrivals at fractions of the served capacity for the
    p50/p99 latency."""
    import copy
    import torch
    from ctsim_b200.serving import ReconServer, latency_stats, make_requests, serve_sequential
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(args.seed)

    def fresh(reqs, storage, arrivals=None):
        out = []
        for i, r in enumerate(reqs):
            c = copy.copy(r)
            c.storage = storage
            c.arrival = 0.0 if arrivals is None else float(arrivals[i])
            c.result = None
            out.append(c)
        return out

    def served(reqs, **kw):
        srv = ReconServer(hbm_budget=int(args.budget_gb * 2 ** 30), max_active=args.slots, to_host=True,
                          admit_workers=2, batch_pwls=args.batch_pwls, **kw)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        done = srv.run(reqs)
        torch.cuda.synchronize()
        return done, time.perf_counter() - t0, srv

    reqs = make_requests(args.requests, seed=args.seed, scale=args.scale, iterations=10, subsets=12,
                         sizes=args.sizes)
    kinds = [r.kind for r in reqs]
    # untimed pass of every arm over the same requests: pinned host buffers, the memory
    # pools, graph instantiation and (with --autotune) the launch-shape records warm up
    serve_sequential(fresh(reqs, "float32"))
    served(fresh(reqs, "float32"))
    served(fresh(reqs, "bfloat16"), autotune=args.autotune)
    clocks = ClockSampler(0)
    clocks.start()
    t_plain = t32 = t16 = float("inf")
    for _ in range(2):  # the better of two timed passes per arm, arms interleaved
        plain = serve_sequential(fresh(reqs, "float32"))
        t_plain = min(t_plain, max(r.t_done for r in plain))
        d32, t, srv = served(fresh(reqs, "float32"))
        if t < t32:
            done32, t32, srv32 = d32, t, srv
        d16, t, srv = served(fresh(reqs, "bfloat16"), autotune=args.autotune)
        if t < t16:
            done16, t16, srv16 = d16, t, srv
    plain_rps = len(plain) / t_plain
    cap = len(done16) / t16
    sweep = []
    # the configured arrival rates (2-50 req/s) that the measured capacity can carry, and
    # 50% / 80% of the capacity
    rates = sorted({r for r in (2.0, 5.0, 10.0, 20.0, 50.0) if r <= 0.9 * cap} | {0.5 * cap, 0.8 * cap})
    for rate in rates:
        frac = rate / cap
        arr = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
        d, t, _ = served(fresh(reqs, "bfloat16", arr), autotune=args.autotune)
        st = latency_stats(d, t)
        st.update({"offered_req_per_s": rate, "load_fraction": frac})
        sweep.append(st)
    clk = clocks.stop()
    closed = latency_stats(done16, t16)
    line = {
        "metric": "served reconstructions/s (FDK + OS-PWLS mix)", "value": cap, "unit": "req/s",
        "impl": "serving", "n_gpus": 1, "higher_is_better": True, "dtype": "bf16 storage, fp32 arithmetic",
        "data": "synthetic (seeded ellipsoid phantoms, Poisson counts)",
        "config": {"workload": "random_geometry mix", "requests": len(reqs), "fdk": kinds.count("fdk"),
                   "pwls": kinds.count("pwls"), "pwls_iterations": 10, "pwls_subsets": 12, "slots": args.slots,
                   "scale": args.scale, "seed": args.seed, "autotune": bool(args.autotune), "sizes": args.sizes,
                   "batch_pwls_per_tick": bool(args.batch_pwls)},
        "plain_fp32_single_instance_req_per_s": plain_rps,
        "served_fp32_req_per_s": len(done32) / t32,
        "speedup_vs_plain_fp32": cap / plain_rps,
        "closed_loop": closed, "open_loop": sweep, "peak_hbm_admitted_bytes": srv16.peak_used,
        "hbm_budget_bytes": int(args.budget_gb * 2 ** 30),
        "concurrency": {"bf16_mean": srv16.mean_active, "bf16_peak": srv16.peak_active,
                        "fp32_mean": srv32.mean_active, "fp32_peak": srv32.peak_active},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_batched(args):
    """Batched uneven instances: OS-PWLS reconstructions of random_geometry instances
    (volumes 128^2x64 .. 384^2x160, 180-720 views, ~20% short scan, ~20% offset detector),
    10 iterations x 12 subsets each, Huber and quadratic penalties alternating, FP32.
    Arms: every instance solved on its own, one after another (reconPwlsSeSqs's loop), and
    all instances stepped together by BatchedPwls (one persistent A and one persistent A^T
    launch per sub-iteration and launch-shape class, CUDA-graph iterations).  Both arms
    start from the same FDK images and must end on identical images."""
    import torch
    from ctsim_b200.fdk import FDK
    from ctsim_b200.projector import Plan
    from ctsim_b200.pwls import BatchedPwls, PwlsSolver
    from ctsim_b200.serving import make_requests
    torch.cuda.set_device(0)
    reqs = make_requests(args.instances, seed=args.seed, fdk_fraction=0.0, storage="float32", scale=args.scale)
    solvers, starts = [], []
    for k, r in enumerate(reqs):
        plan = Plan(r.geom)
        if args.autotune:
            sub = -(-r.geom.noViews // 12)
            plan.autotune("proj,tf", sub)
            plan.autotune("back,tf", sub)
        y = torch.from_numpy(r.sino).cuda()
        w = torch.from_numpy(r.weights).cuda()
        f = FDK(r.geom, "hamming", 1.0, plan=plan)
        x0 = f(y)
        f.close()
        s = PwlsSolver(y, w, r.geom, 1e3 if k % 2 == 0 else 1e2, "huber" if k % 2 == 0 else "quad", 0.01, 12, x0,
                       plan=plan)
        solvers.append(s)
        starts.append(x0)
    its = 10

    def reset():
        for s, x0 in zip(solvers, starts):
            s.x.copy_(x0)
            s.itn = 0

    vv = sum(2 * its * r.geom.nx * r.geom.ny * r.geom.nz * r.geom.noViews for r in reqs)
    # warm-up of both arms (one iteration each)
    for s in solvers:
        s.step()
    reset()
    BatchedPwls(solvers).iteration()
    reset()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in solvers:
        for _ in range(its):
            s.step()
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    seq_images = [s.x.clone() for s in solvers]
    reset()
    b = BatchedPwls(solvers)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(its):
        b.iteration()
    torch.cuda.synchronize()
    t_bat = time.perf_counter() - t0
    same = all(torch.equal(s.x, x) for s, x in zip(solvers, seq_images))
    sizes = [(r.geom.nx, r.geom.nz, r.geom.noViews, r.geom.nu, r.geom.nv) for r in reqs]
    line = {
        "metric": "batched OS-PWLS reconstructions/s (uneven instances)", "value": len(reqs) / t_bat,
        "unit": "instances/s", "impl": "batched", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
        "data": "synthetic (seeded ellipsoid phantoms, Poisson counts)",
        "config": {"workload": "random_geometry instances", "instances": len(reqs), "iterations": its,
                   "subsets": 12, "scale": args.scale, "seed": args.seed, "autotune": bool(args.autotune)},
        "sequential_instances_per_s": len(reqs) / t_seq, "speedup_vs_sequential": t_seq / t_bat,
        "batched_s": t_bat, "sequential_s": t_seq, "gvoxel_views_per_s_batched": vv / t_bat / 1e9,
        "identical_images": bool(same), "sizes_nx_nz_views_nu_nv": sizes,
    }
    print(json.dumps(line), flush=True)


def run_reference_gpu(args):
    """The reference's own CUDA distance-driven pair (geom/dd_cuda: cbct_proj_dd_gpu and
    cbct_back_dd_gpu, compiled unmodified for sm_100a into oracle/_ref) on this GPU, through
    its synchronous host-pointer drivers, beside this project's drop-in host-pointer calls
    on the same inputs: one A and one A^T each, wall clock (both APIs are synchronous and
    include their host copies).  The two outputs are compared; the reference's GPU code
    is not the parity target (its CPU C is) and differs from it at the volume's z edges."""
    import ctypes as C
    import torch
    from ctsim_b200 import _lib
    from oracle.bindings import refgpu_available, refgpu_cbct
    rank, local, world = rank_info()
    if rank != 0:
        return
    if not refgpu_available():
        print(json.dumps({"impl": "reference-gpu", "unavailable": "oracle/_ref/librefgpu_dd.so was not built"}))
        return
    torch.cuda.set_device(0)
    g, x = make_workload(args.views)
    rng = np.random.default_rng(3)
    y = rng.random(g.sino_shape, dtype=np.float32)
    from dataclasses import replace
    warm = replace(g, betas=g.betas[:2].copy(), couchZ=g.couchZ[:2].copy())
    refgpu_cbct("proj,dd", warm, x)
    refgpu_cbct("back,dd", warm, y[:2])
    t0 = time.perf_counter()
    ref_a = refgpu_cbct("proj,dd", g, x)
    t1 = time.perf_counter()
    ref_at = refgpu_cbct("back,dd", g, y)
    t2 = time.perf_counter()
    L = _lib.load()
    betas, couch, mp = np.ascontiguousarray(g.betas), np.ascontiguousarray(g.couchZ), np.ascontiguousarray(g.map)
    ours_a = np.empty(g.sino_shape, np.float32)
    ours_at = np.empty(g.image_shape, np.float32)
    sc = g.scalars()

    def ours():
        ok = L.ctsim_proj_dd(*sc, betas.ctypes.data, couch.ctypes.data, g.flatPanel, x.ctypes.data,
                             ours_a.ctypes.data, mp.ctypes.data)
        ok = ok and L.ctsim_back_dd(*sc, betas.ctypes.data, couch.ctypes.data, g.flatPanel, ours_at.ctypes.data,
                                    y.ctypes.data, mp.ctypes.data)
        if not ok:
            raise RuntimeError(_lib.last_error())

    ours()
    t3 = time.perf_counter()
    ours()
    t4 = time.perf_counter()

    def rel(a, b):
        a64, b64 = a.astype(np.float64), b.astype(np.float64)
        return float(np.linalg.norm(a64 - b64) / max(np.linalg.norm(b64), 1e-300))

    # against the parity target, the reference's CPU C, on two views of the same volume
    from oracle.bindings import ref_available, ref_cbct
    cpu_check = None
    if ref_available():
        g2 = replace(g, betas=g.betas[:2].copy(), couchZ=g.couchZ[:2].copy())
        y2 = np.ascontiguousarray(y[:2])
        nthr = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        cpu_a = ref_cbct("proj,dd", g2, x, nthreads=2)
        cpu_at = ref_cbct("back,dd", g2, y2, nthreads=min(2, nthr))
        ours_at2 = np.empty(g2.image_shape, np.float32)
        b2, c2 = np.ascontiguousarray(g2.betas), np.ascontiguousarray(g2.couchZ)
        if not L.ctsim_back_dd(*g2.scalars(), b2.ctypes.data, c2.ctypes.data, g2.flatPanel, ours_at2.ctypes.data,
                               y2.ctypes.data, mp.ctypes.data):
            raise RuntimeError(_lib.last_error())
        cpu_check = {"views": 2,
                     "A": {"ours": rel(ours_a[:2], cpu_a), "reference_gpu": rel(ref_a[:2], cpu_a)},
                     "A^T": {"ours": rel(ours_at2, cpu_at),
                             "reference_gpu": rel(refgpu_cbct("back,dd", g2, y2), cpu_at)}}
    # FDK back,hpd: the reference's cbct_back_pd_gpu against the drop-in ctsim_back_pd
    fdk = None
    from oracle.bindings import REFGPU_PD_SO
    if os.path.exists(REFGPU_PD_SO):
        refgpu_cbct("back,hpd", warm, y[:2])
        t5 = time.perf_counter()
        ref_pd = refgpu_cbct("back,hpd", g, y)
        t6 = time.perf_counter()
        ours_pd = np.empty(g.image_shape, np.float32)

        def ours_hpd():
            if not L.ctsim_back_pd(*sc, betas.ctypes.data, couch.ctypes.data, g.flatPanel, ours_pd.ctypes.data,
                                   y.ctypes.data, mp.ctypes.data, False):
                raise RuntimeError(_lib.last_error())

        ours_hpd()
        t7 = time.perf_counter()
        ours_hpd()
        t8 = time.perf_counter()
        fdk = {"reference_gpu_ms": (t6 - t5) * 1e3, "ours_host_pointer_ms": (t8 - t7) * 1e3,
               "speedup": (t6 - t5) / (t8 - t7), "rel_l2_reference_gpu_vs_ours": rel(ref_pd, ours_pd)}
        if ref_available():
            cpu_pd = ref_cbct("back,hpd", g2, y2)  # one thread: the reference's own summation order
            ours_pd2 = np.empty(g2.image_shape, np.float32)
            if not L.ctsim_back_pd(*g2.scalars(), b2.ctypes.data, c2.ctypes.data, g2.flatPanel,
                                   ours_pd2.ctypes.data, y2.ctypes.data, mp.ctypes.data, False):
                raise RuntimeError(_lib.last_error())
            fdk["vs_reference_cpu_2_views"] = {"ours_bit_identical": bool(np.array_equal(ours_pd2, cpu_pd)),
                                               "ours": rel(ours_pd2, cpu_pd),
                                               "reference_gpu": rel(refgpu_cbct("back,hpd", g2, y2), cpu_pd)}
    # SF pair: the reference's cbct_proj_tf_gpu / cbct_back_tf_gpu against the drop-in
    # ctsim_proj_tf / ctsim_back_tf (host pointers, synchronous)
    sf = None
    from oracle.bindings import REFGPU_SF_SO
    if os.path.exists(REFGPU_SF_SO):
        refgpu_cbct("proj,tf", warm, x)
        refgpu_cbct("back,tf", warm, y[:2])
        s0 = time.perf_counter()
        ref_sa = refgpu_cbct("proj,tf", g, x)
        s1 = time.perf_counter()
        ref_sat = refgpu_cbct("back,tf", g, y)
        s2 = time.perf_counter()
        ours_sa = np.empty(g.sino_shape, np.float32)
        ours_sat = np.empty(g.image_shape, np.float32)

        def ours_sf():
            ok = L.ctsim_proj_tf(*sc, betas.ctypes.data, couch.ctypes.data, g.flatPanel, x.ctypes.data,
                                 ours_sa.ctypes.data, mp.ctypes.data)
            ok = ok and L.ctsim_back_tf(*sc, betas.ctypes.data, couch.ctypes.data, g.flatPanel,
                                        ours_sat.ctypes.data, y.ctypes.data, mp.ctypes.data)
            if not ok:
                raise RuntimeError(_lib.last_error())

        ours_sf()
        s3 = time.perf_counter()
        ours_sf()
        s4 = time.perf_counter()
        sf = {"reference_gpu_ms": {"A": (s1 - s0) * 1e3, "A^T": (s2 - s1) * 1e3},
              "ours_host_pointer_ms": (s4 - s3) * 1e3, "speedup": (s2 - s0) / (s4 - s3),
              "rel_l2_reference_gpu_vs_ours": {"A": rel(ref_sa, ours_sa), "A^T": rel(ref_sat, ours_sat)}}
        if ref_available():
            cpu_sa = ref_cbct("proj,tf", g2, x, nthreads=2)
            cpu_sat = ref_cbct("back,tf", g2, y2, nthreads=2)
            ours_sat2 = np.empty(g2.image_shape, np.float32)
            if not L.ctsim_back_tf(*g2.scalars(), b2.ctypes.data, c2.ctypes.data, g2.flatPanel,
                                   ours_sat2.ctypes.data, y2.ctypes.data, mp.ctypes.data):
                raise RuntimeError(_lib.last_error())
            sf["vs_reference_cpu_2_views"] = {
                "A": {"ours": rel(ours_sa[:2], cpu_sa), "reference_gpu": rel(ref_sa[:2], cpu_sa)},
                "A^T": {"ours": rel(ours_sat2, cpu_sat), "reference_gpu": rel(refgpu_cbct("back,tf", g2, y2), cpu_sat)}}
    vv = float(g.nx * g.ny * g.nz * g.noViews)
    line = {"metric": METRIC, "impl": "reference-gpu", "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "value": 2 * vv / (t2 - t0) / 1e9, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"DD A + A^T, {g.nx}x{g.ny}x{g.nz}, {g.noViews} views, {g.nu}x{g.nv} detector",
                       "api": "host pointers, synchronous (cbct_proj_dd_gpu / cbct_back_dd_gpu)"},
            "reference_gpu_ms": {"A": (t1 - t0) * 1e3, "A^T": (t2 - t1) * 1e3},
            "ours_host_pointer_ms": {"A+A^T": (t4 - t3) * 1e3},
            "ours_host_pointer_value": 2 * vv / (t4 - t3) / 1e9,
            "speedup": (t2 - t0) / (t4 - t3),
            "rel_l2_reference_gpu_vs_ours": {"A": rel(ref_a, ours_a), "A^T": rel(ref_at, ours_at)},
            "rel_l2_vs_reference_cpu": cpu_check, "fdk_back_hpd": fdk, "sf_pair": sf}
    print(json.dumps(line), flush=True)


def run_recon(args):
    """Config-2 reconstructions on the device: reconFDK ('hann' window, crop 1) and OS-SQS
    PWLS (reconPwlsSeSqs: SF pair, 24 ordered subsets, Huber delta 0.001, beta 5e4) started
    from the FDK image, from log Poisson data (I0 1e5, counts clamped at 10) with the
    weights w = counts (computeWeightsPwls(counts, 0, 0)).  FP32; CUDA-event timing of
    the FDK call, of the PWLS set-up (A 1 and A^T (w A 1), the subset copies) and of the
    outer iterations (each ends with the host read of phi and rmsd)."""
    import torch
    from ctsim_b200.fdk import FDK
    from ctsim_b200.projector import Plan
    from ctsim_b200.pwls import PwlsSolver
    torch.cuda.set_device(0)
    g, x = make_workload(args.views)
    plan = Plan(g)
    xd = torch.from_numpy(x).cuda()
    with torch.no_grad():
        p = plan.project(xd, "tf")
        gen = torch.Generator(device="cuda")
        gen.manual_seed(4321)
        counts = torch.poisson(1e5 * torch.exp(-p), generator=gen)
        y = torch.log(1e5 / torch.clamp(counts, min=10.0)).contiguous()
        w = counts.contiguous()
        del p

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        r = fn()
        b.record()
        torch.cuda.synchronize()
        return r, a.elapsed_time(b)

    def rel_rmse(img):
        return float(torch.sqrt(torch.mean((img - xd) ** 2)) / torch.sqrt(torch.mean(xd ** 2)))

    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    f = FDK(g, "hann", 1.0, plan=plan)
    f(y)
    torch.cuda.synchronize()
    fdk_ms = min(timed(lambda: f(y))[1] for _ in range(3))
    x0 = f(y)
    solver, setup_ms = timed(lambda: PwlsSolver(y, w, g, 5e4, "huber", 0.001, 24, x0, plan=plan,
                                                autotune=args.autotune))
    its = args.iterations
    phis, rmsds, it_ms = [], [], []
    for _ in range(its):
        (phi, rmsd), ms = timed(solver.step)
        phis.append(phi)
        rmsds.append(rmsd)
        it_ms.append(ms)
    ck = clocks.stop()
    vv = float(g.nx * g.ny * g.nz * g.noViews)
    steady = it_ms[1:] if len(it_ms) > 1 else it_ms
    line = {
        "metric": "config-2 reconstruction times", "unit": "ms", "impl": "ours", "n_gpus": 1, "dtype": "f32",
        "higher_is_better": False, "data": "synthetic (seeded 20-ellipsoid phantom, log Poisson data I0=1e5)",
        "config": {"workload": "reconFDK hann + OS-SQS PWLS (SF, 24 subsets, huber 0.001, beta 5e4)",
                   "volume": [g.nx, g.ny, g.nz], "views": g.noViews, "detector": [g.nu, g.nv],
                   "iterations": its, "autotune": bool(args.autotune), "tuning": plan.tuning},
        "fdk_ms": fdk_ms, "fdk_gvv_s": vv / (fdk_ms / 1e3) / 1e9,
        "pwls_setup_ms": setup_ms, "pwls_iteration_ms": float(np.mean(steady)),
        "pwls_iteration_gvv_s": 2 * vv / (float(np.mean(steady)) / 1e3) / 1e9,
        "pwls_iteration_ms_each": it_ms, "phi": phis, "rmsd": rmsds,
        "rel_rmse_vs_phantom": {"fdk": rel_rmse(x0), "pwls": rel_rmse(solver.x)},
        "clocks": ck,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", dest="no_cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--extras", action="store_true", help="also time SF A/A^T and FDK back,hpd")
    ap.add_argument("--views", type=int, default=0, help="keep only this many views (profiling captures)")
    ap.add_argument("--consecutive", action="store_true", help="with --views: the first views, not every n-th")
    ap.add_argument("--no-e2e", dest="no_e2e", action="store_true", help="skip the end-to-end host-buffer leg")
    ap.add_argument("--no-serving", dest="no_serving", action="store_true",
                    help="skip the bounded served-stream leg of the default run")
    ap.add_argument("--no-config1", dest="no_config1", action="store_true",
                    help="skip the 128x128x64 / 360-view DD step of the default run")
    ap.add_argument("--serving", action="store_true", help="served FDK/OS-PWLS request mix instead of A/A^T")
    ap.add_argument("--requests", type=int, default=24, help="requests of the serving run")
    ap.add_argument("--slots", type=int, default=8, help="concurrent requests of the serving run")
    ap.add_argument("--budget-gb", dest="budget_gb", type=float, default=150.0,
                    help="serving: HBM admission budget in GiB")
    ap.add_argument("--scale", type=float, default=1.0, help="size scale of the serving run's geometries")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--autotune", action="store_true", help="serving/batched: autotune launch shapes")
    ap.add_argument("--batched", action="store_true", help="batched uneven OS-PWLS instances instead of A/A^T")
    ap.add_argument("--sizes", choices=["config1", "uneven"], default="uneven", help="serving: request sizes")
    ap.add_argument("--batch-pwls", dest="batch_pwls", action="store_true",
                    help="serving: batch the OS-PWLS requests per scheduler tick")
    ap.add_argument("--instances", type=int, default=16, help="instances of the batched run")
    ap.add_argument("--recon", action="store_true", help="config-2 reconFDK and OS-SQS PWLS times")
    ap.add_argument("--reference-gpu", dest="reference_gpu", action="store_true",
                    help="the reference's own CUDA DD pair on this GPU beside the drop-in calls")
    ap.add_argument("--iterations", type=int, default=5, help="OS-SQS iterations of the --recon run")
    args = ap.parse_args()
    if args.reference_gpu:
        run_reference_gpu(args)
    elif args.recon:
        run_recon(args)
    elif args.batched:
        run_batched(args)
    elif args.serving:
        run_serving(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
