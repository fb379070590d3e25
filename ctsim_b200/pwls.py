"""OS-PWLS reconstruction on the device (statsrecon/pwls/reconPwlsSeSqs.m).

Mirrors the reference's MATLAB entry points with torch CUDA tensors:

* ``computeWeightsPwls(sino, r, v)``            statsrecon/pwls/computeWeightsPwls.m
* ``huberPenalty(x, mode, delta)``, ``quadPenalty(x, mode)``
                                                penalty/huberPenalty.m, penalty/quadPenalty.m
* ``loadPenaltyOperator(pfun, delta)``          penalty/loadPenaltyOperator.m ('huber', 'quad')
* ``reconPwlsSeSqs(y, w, geom, beta, pfun, itnlim, delta, numos, img0)``
                                                statsrecon/pwls/reconPwlsSeSqs.m
* ``reconPwlsSeNesterovSqs(y, w, geom, beta, pfun, itnlim, delta, numos, img0, imgOpt)``
                                                statsrecon/pwls/reconPwlsSeNesterovSqs.m
* ``BatchedPwls(solvers)``                      many reconPwlsSeSqs instances in batched launches

The projectors are the separable-footprint pair the reference's PWLS loads
(geom/shell/loadPojectors.m:8-11); all per-voxel and per-ray arithmetic runs in
CUDA kernels of libctsim_b200 (pwls.cu), reductions (cost, rmsd) in FP64.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from .geometry import CTGeometry
from .projector import plan_for

PENALTIES = {"huber": 0, "quad": 1}


def _torch():
    import torch
    return torch


def _stream(dev):
    return _torch().cuda.current_stream(dev).cuda_stream


def computeWeightsPwls(sino, r: float = 0.0, v: float = 0.0):
    """w = (sino - r).^2 ./ (sino + v), w(sino <= r) = 0 (single)."""
    torch = _torch()
    s = sino.contiguous()
    w = torch.empty_like(s)
    _lib.check(_lib.load().ctsim_pwls_weights(s.data_ptr(), float(r), float(v), w.data_ptr(), s.numel(),
                                              _stream(s.device)), "ctsim_pwls_weights")
    return w


def _penalty(x, kind: int, mode: int, delta: float):
    torch = _torch()
    x = x.contiguous()
    nz, ny, nx = x.shape
    L = _lib.load()
    if mode == 0:
        acc = torch.zeros(1, dtype=torch.float64, device=x.device)
        _lib.check(L.ctsim_penalty(kind, 0, float(delta), nx, ny, nz, x.data_ptr(), None, acc.data_ptr(),
                                   _stream(x.device)), "ctsim_penalty")
        return acc
    out = torch.empty_like(x)
    _lib.check(L.ctsim_penalty(kind, mode, float(delta), nx, ny, nz, x.data_ptr(), out.data_ptr(), None,
                               _stream(x.device)), "ctsim_penalty")
    return out


def huberPenalty(x, mode: int, delta: float = 0.001):
    """mode 0: value (FP64 scalar tensor), 1: gradient, 2: curvature."""
    return _penalty(x, 0, mode, delta)


def quadPenalty(x, mode: int):
    """mode 0: value, 1: gradient (dQuad(d) = d), 2: curvature (constant 4 + 4/sqrt(2) + 1)."""
    return _penalty(x, 1, mode, 0.0)


def loadPenaltyOperator(pfun: str, delta: float = 0.001):
    """(R, S, T): penalty value, gradient and curvature operators."""
    if pfun.lower() not in PENALTIES:
        raise ValueError("unknow penalty function")
    kind = PENALTIES[pfun.lower()]
    return (lambda x: _penalty(x, kind, 0, delta), lambda x: _penalty(x, kind, 1, delta),
            lambda x: _penalty(x, kind, 2, delta))


class PwlsSolver:
    """Device state of one OS-PWLS reconstruction: plan, subset data and buffers.

    ``step()`` runs one outer iteration (all ``numos`` subsets) and returns
    (phi, rmsd); ``reconPwlsSeSqs`` loops it like the reference.
    """

    def __init__(self, y, w, geom: CTGeometry, beta: float, pfun: str = "huber", delta: float = 0.001,
                 numos: int = 1, img0=None, method: str = "tf", storage=None, plan=None, autotune: bool = False):
        torch = _torch()
        if pfun.lower() not in PENALTIES:
            raise ValueError("unknow penalty function")
        self.geom, self.beta, self.delta, self.M = geom, float(beta), float(delta), int(numos)
        self.kind = PENALTIES[pfun.lower()]
        self.method = method
        self.plan = plan if plan is not None else plan_for(geom, y.device)
        if autotune:  # launch shapes timed on subset-sized launches (recorded per shape class)
            sub = max(1, -(-geom.noViews // self.M))
            self.plan.autotune(f"proj,{method}", sub)
            self.plan.autotune(f"back,{method}", sub)
        self.dev = self.plan.device
        self.L = _lib.load()
        # the measured data (y, w: the largest arrays) may be stored in bfloat16 or float16;
        # the image, the surrogate denominator and every residual stay FP32
        self.storage = storage or torch.float32
        from .projector import _DTYPES
        self.sdt = _DTYPES[self.storage]
        if img0 is None:
            from .fdk import reconFDK
            img0 = reconFDK(y.to(self.dev, torch.float32).contiguous(), geom)
        y = y.to(self.dev, self.storage).contiguous()
        # weights are photon counts (1e5 and more): FP16 stores them divided by a power of two
        self.w_scale = 1.0
        if self.storage == torch.float16:
            w32 = w.to(self.dev, torch.float32)
            wmax = float(w32.max().item())
            if wmax > 16384.0:
                self.w_scale = float(2.0 ** math.ceil(math.log2(wmax / 16384.0)))
            w = (w32 / self.w_scale).to(self.storage).contiguous()
            del w32
        else:
            w = w.to(self.dev, self.storage).contiguous()
        self.x = img0.to(self.dev, torch.float32).clone().contiguous()
        self.xn = torch.empty_like(self.x)
        self.xold = torch.empty_like(self.x)
        # precompute (reconPwlsSeSqs.m:40-41): a = A(1), precom = At(w .* a); w .* a is written
        # over a already times the axial amplitudes (the first product of At), so one FP32
        # sinogram-sized buffer serves both
        a = self.plan.project(torch.ones_like(self.x), method)
        _lib.check(self.L.ctsim_pwls_residual_scaled(self.plan._h, a.data_ptr(), None, w.data_ptr(), self.sdt,
                                                     self.w_scale, a.data_ptr(), geom.noViews, None,
                                                     _stream(self.dev)), "ctsim_pwls_residual_scaled")
        self.precom = self.plan.backproject(a, method, scaled=True)
        del a
        # subsets 1+mod(isub,M):M:end for isub = 1..M (0-based start isub % M)
        self.subsets = []
        for isub in range(1, self.M + 1):
            start = isub % self.M if self.M > 1 else 0
            count = len(range(start, geom.noViews, self.M))
            self.subsets.append((start, count, y[start::self.M].contiguous(), w[start::self.M].contiguous()))
        maxc = max(c for _, c, _, _ in self.subsets)
        self.ax = torch.empty((maxc, geom.nu, geom.nv), dtype=torch.float32, device=self.dev)
        self.wd = torch.empty_like(self.ax)
        self.num = torch.empty_like(self.x)
        self.acc = torch.zeros(3, dtype=torch.float64, device=self.dev)  # phi, rmsd sum, penalty value
        self.nx, self.ny, self.nz = geom.nx, geom.ny, geom.nz
        self.itn = 0

    def subset_step(self, i: int):
        """Sub-iteration i (0-based) of the current outer iteration, asynchronous on the
        current stream (reconPwlsSeSqs.m:57-66)."""
        st = _stream(self.dev)
        if i == 0:
            self.xold.copy_(self.x)
            self.acc.zero_()
        acc = self.acc.data_ptr()
        stride = 1 if self.M == 1 else self.M
        start, count, ys, ws = self.subsets[i]
        ax = self.ax[:count]
        wd = self.wd[:count]
        self.plan.project(self.x, self.method, start, stride, count, out=ax)
        self._residual(ax, ys, ws, wd, count, acc, st)
        self.plan.backproject(wd, self.method, start, stride, count, scale=float(self.M), out=self.num, scaled=True)
        _lib.check(self.L.ctsim_sqs_update(self.kind, self.beta, self.delta, self.nx, self.ny, self.nz,
                                           self.x.data_ptr(), self.xn.data_ptr(), self.num.data_ptr(),
                                           self.precom.data_ptr(), st), "ctsim_sqs_update")
        self.x, self.xn = self.xn, self.x

    def _residual(self, ax, ys, ws, wd, count, acc, st):
        """wd = (w (A_s x - y_s)) * ampv per pixel (the weighted residual with the first
        product of A^T applied: backprojected with scaled=True, no scaled copy), and the
        data term sum(w d^2) into the FP64 accumulator at acc (reconPwlsSeSqs.m:57-74)."""
        _lib.check(self.L.ctsim_pwls_residual_scaled(self.plan._h, ax.data_ptr(), ys.data_ptr(), ws.data_ptr(),
                                                     self.sdt, self.w_scale, wd.data_ptr(), count, acc, st),
                   "ctsim_pwls_residual_scaled")

    def end_iteration(self):
        """Penalty value and squared change of the iteration into the FP64 accumulators
        (asynchronous; ``step`` reads them)."""
        st = _stream(self.dev)
        acc = self.acc.data_ptr()
        _lib.check(self.L.ctsim_penalty(self.kind, 0, self.delta, self.nx, self.ny, self.nz, self.x.data_ptr(),
                                        None, acc + 16, st), "ctsim_penalty")
        _lib.check(self.L.ctsim_sqdiff(self.x.data_ptr(), self.xold.data_ptr(), self.x.numel(), acc + 8, st),
                   "ctsim_sqdiff")

    def step(self):
        """One outer iteration; returns (phi, rmsd) (synchronises)."""
        for i in range(len(self.subsets)):
            self.subset_step(i)
        self.end_iteration()
        a = self.acc.cpu().numpy()
        self.itn += 1
        phi = a[0] / 2 + self.beta * a[2]
        rmsd = math.sqrt(a[1] / self.x.numel())
        return phi, rmsd


def reconPwlsSeSqs(y, w, geom: CTGeometry, beta: float, pfun: str = "huber", itnlim: int = 10,
                   delta: float = 0.001, numos: int = 1, img0=None, stopCrt: float = 1e-5, storage=None):
    """statsrecon/pwls/reconPwlsSeSqs.m: returns (x, phis, rmsds).  ``storage`` (torch dtype)
    stores y and w in bfloat16/float16; arithmetic and the image stay FP32."""
    solver = PwlsSolver(y, w, geom, beta, pfun, delta, numos, img0, storage=storage)
    phis, rmsds = np.zeros(itnlim), np.zeros(itnlim)
    for itn in range(1, itnlim + 1):
        phi, rmsd = solver.step()
        phis[itn - 1], rmsds[itn - 1] = phi, rmsd
        if itn > 5 and rmsd < stopCrt:  # reconPwlsSeSqs.m:106
            break
    return solver.x, phis, rmsds


class PwlsNesterovSolver(PwlsSolver):
    """OS-SQS with Nesterov's momentum (statsrecon/pwls/reconPwlsSeNesterovSqs.m:41-136):
    the subsets project the extrapolated image z, the step is taken from z, and the
    momentum state s and scalar t follow Kim, Ramani and Fessler (2013) as the reference
    writes them.  ``img_opt`` (the converged image) switches the rmsd to the distance of the
    middle slice from it (reconPwlsSeNesterovSqs.m:102-113)."""

    def __init__(self, *args, img_opt=None, **kw):
        super().__init__(*args, **kw)
        torch = _torch()
        self.z = self.x.clone()
        self.s = self.x.clone()
        self.zn = torch.empty_like(self.x)
        self.t = 1.0
        self.img_opt = None
        if img_opt is not None:
            if self.nz % 2:
                raise ValueError("the rmsd against imgOpt compares slice end/2, which needs an even nz")
            k = self.nz // 2 - 1  # x(:,:,end/2), 0-based
            self._slice = k
            self.img_opt = img_opt.to(self.dev, torch.float32)[k].contiguous()

    def subset_step(self, i: int):
        st = _stream(self.dev)
        if i == 0:
            self.xold.copy_(self.x)
            self.acc.zero_()
        acc = self.acc.data_ptr()
        stride = 1 if self.M == 1 else self.M
        start, count, ys, ws = self.subsets[i]
        ax = self.ax[:count]
        wd = self.wd[:count]
        self.plan.project(self.z, self.method, start, stride, count, out=ax)        # Aos(z, isub)
        self._residual(ax, ys, ws, wd, count, acc, st)
        self.plan.backproject(wd, self.method, start, stride, count, scale=float(self.M), out=self.num, scaled=True)
        t_next = (1.0 + math.sqrt(1.0 + 4.0 * self.t * self.t)) / 2.0
        _lib.check(self.L.ctsim_nesterov_update(self.kind, self.beta, self.delta, self.nx, self.ny, self.nz,
                                                self.z.data_ptr(), self.x.data_ptr(), self.s.data_ptr(),
                                                self.num.data_ptr(), self.precom.data_ptr(), self.t, t_next,
                                                self.xn.data_ptr(), self.zn.data_ptr(), st),
                   "ctsim_nesterov_update")
        self.x, self.xn = self.xn, self.x
        self.z, self.zn = self.zn, self.z
        self.t = t_next

    def end_iteration(self):
        if self.img_opt is None:
            return super().end_iteration()
        st = _stream(self.dev)
        acc = self.acc.data_ptr()
        _lib.check(self.L.ctsim_penalty(self.kind, 0, self.delta, self.nx, self.ny, self.nz, self.x.data_ptr(),
                                        None, acc + 16, st), "ctsim_penalty")
        xs = self.x[self._slice]
        _lib.check(self.L.ctsim_sqdiff(xs.data_ptr(), self.img_opt.data_ptr(), xs.numel(), acc + 8, st),
                   "ctsim_sqdiff")

    def step(self):
        for i in range(len(self.subsets)):
            self.subset_step(i)
        self.end_iteration()
        a = self.acc.cpu().numpy()
        self.itn += 1
        phi = a[0] / 2 + self.beta * a[2]
        n = self.x.numel() if self.img_opt is None else self.img_opt.numel()
        return phi, math.sqrt(a[1] / n)

    def restart(self):
        """t = 1, z = x, s = x (reconPwlsSeNesterovSqs.m:132-136)."""
        self.t = 1.0
        self.z.copy_(self.x)
        self.s.copy_(self.x)


def reconPwlsSeNesterovSqs(y, w, geom: CTGeometry, beta: float, pfun: str = "huber", itnlim: int = 10,
                           delta: float = 0.001, numos: int = 1, img0=None, imgOpt=None, storage=None):
    """statsrecon/pwls/reconPwlsSeNesterovSqs.m: returns (x, phis, rmsds).  Stops after
    iteration 5 once rmsd < 1e-10; restarts the momentum every round(2 itnlim) iterations."""
    solver = PwlsNesterovSolver(y, w, geom, beta, pfun, delta, numos, img0, storage=storage, img_opt=imgOpt)
    stop_crt = 1e-10
    nrestart = int(round(itnlim * 2))
    phis, rmsds = np.zeros(itnlim), np.zeros(itnlim)
    for itn in range(1, itnlim + 1):
        phi, rmsd = solver.step()
        phis[itn - 1], rmsds[itn - 1] = phi, rmsd
        if itn > 5 and rmsd < stop_crt:
            break
        if itn % nrestart == 0:
            solver.restart()
    return solver.x, phis, rmsds


def batched_subset_steps(pairs):
    """Sub-iteration i_k of solver k for every (solver_k, i_k) in ``pairs`` -- solvers of
    different geometries and subset counts, each at its own place in its iteration --
    with one batched A and one batched A^T (reconPwlsSeSqs.m:57-66 for each solver).
    Asynchronous on the current stream; the solvers need distinct plans and one method."""
    from .projector import batch_backproject, batch_project
    if not pairs:
        return
    method = pairs[0][0].method
    fwd, back = [], []
    for s, i in pairs:
        if s.method != method:
            raise ValueError("batched solvers need the same projector method")
        if i == 0:
            s.xold.copy_(s.x)
            s.acc.zero_()
        start, count, _, _ = s.subsets[i]
        fwd.append((s.plan, s.x, s.ax[:count], start, 1 if s.M == 1 else s.M, count))
    batch_project(method, fwd)
    for s, i in pairs:
        start, count, ys, ws = s.subsets[i]
        ax, wd = s.ax[:count], s.wd[:count]
        s._residual(ax, ys, ws, wd, count, s.acc.data_ptr(), _stream(s.dev))
        back.append((s.plan, wd, s.num, start, 1 if s.M == 1 else s.M, count, float(s.M)))
    batch_backproject(method, back, scaled=True)
    for s, i in pairs:
        _lib.check(s.L.ctsim_sqs_update(s.kind, s.beta, s.delta, s.nx, s.ny, s.nz, s.x.data_ptr(),
                                        s.xn.data_ptr(), s.num.data_ptr(), s.precom.data_ptr(), _stream(s.dev)),
                   "ctsim_sqs_update")
        s.x, s.xn = s.xn, s.x


class BatchedPwls:
    """Many OS-PWLS reconstructions (reconPwlsSeSqs.m:57-66 each) stepped together.

    Every sub-iteration runs ONE persistent A launch over all instances' subset views
    (ctsim_batch_project, per launch-shape class), the per-instance residuals, ONE
    persistent A^T launch (ctsim_batch_backproject) and the per-instance SQS updates;
    with ``graphs`` an outer iteration of all instances is one CUDA-graph replay after
    the first.  The instances keep their own plans, data and state, so each result is
    the one its own solver would compute.  All solvers use the same projector method
    and number of subsets.
    """

    def __init__(self, solvers, graphs: bool = True):
        if not solvers:
            raise ValueError("no solvers")
        self.solvers = list(solvers)
        self.M = self.solvers[0].M
        self.method = self.solvers[0].method
        if any(s.M != self.M or s.method != self.method for s in self.solvers):
            raise ValueError("batched solvers need the same method and number of subsets")
        if len({id(s.plan) for s in self.solvers}) != len(self.solvers):
            raise ValueError("each batched solver needs its own plan")
        self.graphs = graphs
        self._graph = {}
        self.itn = 0

    def subset_step(self, i: int):
        batched_subset_steps([(s, i) for s in self.solvers])

    def _eager_iteration(self):
        for i in range(self.M):
            self.subset_step(i)
        for s in self.solvers:
            s.end_iteration()

    def iteration(self):
        """One outer iteration of every instance (asynchronous, ordered after the work
        already queued on the current stream; graphs are captured on a private stream)."""
        torch = _torch()
        cur = torch.cuda.current_stream(self.solvers[0].dev)
        if not hasattr(self, "_stream"):
            self._stream = torch.cuda.Stream(device=self.solvers[0].dev)
        self._stream.wait_stream(cur)
        with torch.cuda.stream(self._stream):
            self._iteration_on_stream(torch)
        cur.wait_stream(self._stream)
        self.itn += 1
        for s in self.solvers:
            s.itn += 1

    def _iteration_on_stream(self, torch):
        if not self.graphs or self.itn == 0:
            self._eager_iteration()
        else:
            key = tuple(s.x.data_ptr() for s in self.solvers)
            g = self._graph.get(key)
            if g is None:
                # recorded, not run: the pointer swaps leave the host side as after the run
                g = torch.cuda.CUDAGraph()
                g.capture_begin(capture_error_mode="thread_local")
                self._eager_iteration()
                g.capture_end()
                self._graph[key] = g
            else:
                for s in self.solvers:
                    for _ in range(self.M):
                        s.x, s.xn = s.xn, s.x
            g.replay()

    def step(self):
        """One outer iteration; returns [(phi, rmsd)] per instance (synchronises)."""
        self.iteration()
        out = []
        for s in self.solvers:
            a = s.acc.cpu().numpy()
            out.append((a[0] / 2 + s.beta * a[2], math.sqrt(a[1] / s.x.numel())))
        return out
