"""Served reconstruction (ctsim_b200.serving): admission by HBM budget and slots,
continuous issue across requests, and results that do not depend on the mix."""
import copy

import numpy as np
import pytest

from ctsim_b200 import CTGeometry, circular_betas
from ctsim_b200.serving import ReconRequest, ReconServer, hbm_footprint


def _geom(n, nz, nu, nv, views):
    return CTGeometry((n, n, nz), (1.0, 1.0, 1.0), (0, 0, 0), (nu, nv), (1.2, 1.2), (0, 0), 1000.0, 500.0, 1500.0,
                      circular_betas(views))


class _FakeActive:
    """Host-only stand-in for a request's device state: each unit takes `lag` ticks."""

    def __init__(self, req, slot, log, lag=2):
        self.req, self.slot, self.log, self.lag = req, slot, log, lag
        self.units = req.iterations if req.kind == "pwls" else 1
        self.issued = 0
        self.pending = []
        self.released = False

    def in_flight(self):
        self.pending = [t - 1 for t in self.pending if t > 1]
        return len(self.pending)

    def issue(self, to_host=False):
        self.issued += 1
        self.pending.append(self.lag)
        self.log.append(("issue", self.req.rid, self.slot))

    def complete(self):
        return self.issued == self.units and self.in_flight() == 0

    def release(self):
        self.released = True
        self.log.append(("release", self.req.rid, self.slot))

    def check(self):
        pass


class _Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.001
        return self.t


def _requests():
    rng = np.random.default_rng(3)
    reqs = []
    for rid in range(14):
        g = _geom(int(rng.choice([32, 64, 96])), 16, 64, 24, int(rng.choice([24, 48])))
        kind = "pwls" if rid % 3 == 0 else "fdk"
        reqs.append(ReconRequest(kind, g, None, storage=["float32", "bfloat16", "float16"][rid % 3],
                                 arrival=0.002 * rid, rid=rid, iterations=3))
    return reqs


def test_footprint_grows_with_storage_and_kind():
    g = _geom(64, 32, 128, 32, 60)
    f32 = hbm_footprint(ReconRequest("fdk", g, None, storage="float32"))
    b16 = hbm_footprint(ReconRequest("fdk", g, None, storage="bfloat16"))
    p32 = hbm_footprint(ReconRequest("pwls", g, None, storage="float32"))
    assert b16 < f32 < p32
    # at least the plan scratch, the stored sinogram and the image
    pix, vox = 128 * 32 * 60, 64 * 64 * 32
    assert f32 >= 4 * pix + 4 * pix + 4 * vox


def test_admission_respects_budget_slots_and_arrival_order():
    reqs = _requests()
    need = sorted(hbm_footprint(r) for r in reqs)
    budget = need[-1] + need[-2]  # never room for every request at once
    log = []
    srv = ReconServer(hbm_budget=budget, max_active=3, activate=lambda r, s: _FakeActive(r, s, log),
                      clock=_Clock())
    active_max = 0
    for r in sorted(reqs, key=lambda r: r.arrival):
        srv.submit(r)
    srv.t0 = srv._clock()
    while srv.pending or srv.active:
        srv.tick()
        active_max = max(active_max, len(srv.active))
        assert srv.used <= budget
        assert len({srv._slot_of[id(a)] for a in srv.active}) == len(srv.active)  # one slot each
    assert srv.peak_used <= budget and active_max <= 3
    assert sorted(r.rid for r in srv.done) == list(range(len(reqs)))
    admit_order = [r.rid for r in sorted(reqs, key=lambda r: r.t_admit)]
    assert admit_order == sorted(admit_order)  # first come, first admitted
    assert all(r.t_admit >= r.arrival for r in reqs)
    assert all(r.t_done >= r.t_admit for r in reqs)
    # a PWLS request's units are issued one per tick while other requests progress
    issues = [e for e in log if e[0] == "issue"]
    assert len(issues) == sum(3 if r.kind == "pwls" else 1 for r in reqs)
    assert srv.used == 0


def test_submit_rejects_bad_requests():
    g = _geom(32, 16, 64, 24, 24)
    srv = ReconServer(hbm_budget=1 << 16, activate=lambda r, s: None)
    with pytest.raises(ValueError, match="budget"):
        srv.submit(ReconRequest("fdk", g, None))
    srv = ReconServer(hbm_budget=1 << 40, activate=lambda r, s: None)
    with pytest.raises(ValueError, match="kind"):
        srv.submit(ReconRequest("sart", g, None))
    with pytest.raises(ValueError, match="storage"):
        srv.submit(ReconRequest("fdk", g, None, storage="int8"))


# ---------------------------------------------------------------------------
# On the device
# ---------------------------------------------------------------------------
def _device_requests(storage="float32"):
    from ctsim_b200.serving import make_requests
    reqs = make_requests(7, seed=11, fdk_fraction=0.5, storage=storage, scale=0.15, iterations=3, subsets=4)
    kinds = ["fdk", "pwls", "fdk", "pwls", "pwls", "fdk", "pwls"]
    for r, k in zip(reqs, kinds):
        r.kind = k
        if k == "pwls" and r.weights is None:
            y = np.asarray(r.sino)
            r.weights = (1e5 * np.exp(-y)).astype(np.float32)
    reqs[4].subsets = 3  # odd subset count: the two x buffers alternate between iterations
    return reqs


def _result(r):
    import torch
    x = r.result
    return x.cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


@pytest.mark.gpu
def test_served_results_do_not_depend_on_the_mix():
    """Bit-identical images whether a request is served alone, in a mix of seven on four
    slots, without CUDA graphs, with set-up on admission threads and delivery to host
    memory, with the OS-PWLS requests batched per tick, or through the plain
    single-instance FP32 API."""
    from ctsim_b200.serving import serve_sequential
    reqs = _device_requests()
    mixed = copy.deepcopy(reqs)
    done = ReconServer(max_active=4).run(mixed)
    assert len(done) == len(reqs)
    eager = copy.deepcopy(reqs)
    ReconServer(max_active=4, graphs=False).run(eager)
    threaded = copy.deepcopy(reqs)
    ReconServer(max_active=3, to_host=True, admit_workers=2).run(threaded)
    batched = copy.deepcopy(reqs)
    ReconServer(max_active=5, to_host=True, admit_workers=2, batch_pwls=True).run(batched)
    plain = serve_sequential(copy.deepcopy(reqs))
    for i, r in enumerate(reqs):
        alone = copy.deepcopy(r)
        ReconServer(max_active=1).run([alone])
        a = _result(alone)
        assert a.shape == r.geom.image_shape and np.isfinite(a).all() and np.abs(a).max() > 0
        assert np.array_equal(_result(mixed[i]), a), (i, r.kind)
        assert np.array_equal(_result(eager[i]), a), (i, r.kind)
        assert not threaded[i].result.is_cuda and np.array_equal(_result(threaded[i]), a), (i, r.kind)
        assert np.array_equal(_result(batched[i]), a), (i, r.kind)
        assert np.array_equal(_result(plain[i]), a), (i, r.kind)


@pytest.mark.gpu
def test_served_low_precision_storage_close_to_fp32():
    """bfloat16/float16 storage of sinogram and weights (FP32 arithmetic) against FP32
    storage: relative RMS error of the images."""
    ref = _device_requests("float32")
    ReconServer(max_active=4).run(ref)
    for storage, tol in (("bfloat16", 1e-2), ("float16", 2e-3)):
        reqs = _device_requests(storage)
        ReconServer(max_active=4).run(reqs)
        for a, b in zip(reqs, ref):
            x, x0 = _result(a), _result(b)
            err = np.sqrt(np.mean((x - x0) ** 2)) / np.sqrt(np.mean(x0 ** 2))
            assert err < tol, (storage, a.rid, a.kind, err)


@pytest.mark.gpu
def test_served_footprint_bounds_device_memory():
    """The admission estimate bounds what a request allocates (torch tensors and the
    library pool): measured on an otherwise idle device, request by request."""
    import torch
    from ctsim_b200.serving import _Active
    reqs = _device_requests("bfloat16")[:2]
    s = torch.cuda.Stream()
    for r in reqs:
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats()
        base = torch.cuda.memory_allocated()
        a = _Active(r, s, torch.device("cuda", 0))
        while not a.complete():
            if a.issued < a.units:
                a.issue()
        torch.cuda.synchronize()
        torch_peak = torch.cuda.max_memory_allocated() - base
        used = torch_peak + a.plan.device_bytes
        a.release()
        torch.cuda.synchronize()
        assert used <= hbm_footprint(r), (r.kind, used, hbm_footprint(r))


# ---------------------------------------------------------------------------
# Failure isolation (host-side injection only: no GPU fault is made)
# ---------------------------------------------------------------------------
class _FailingIssue(_FakeActive):
    def issue(self, to_host=False):
        if self.issued == 1:
            raise RuntimeError("injected failure of the second unit")
        super().issue(to_host)


def _serve_with_faults(admit_workers):
    reqs = _requests()
    log = []

    def activate(r, s):
        if r.rid == 2:
            raise MemoryError("injected set-up failure")
        if r.rid == 6:
            return _FailingIssue(r, s, log)  # a PWLS request (3 units) that fails at its second
        return _FakeActive(r, s, log)

    srv = ReconServer(hbm_budget=1 << 40, max_active=3, activate=activate, clock=_Clock(),
                      admit_workers=admit_workers)
    for r in sorted(reqs, key=lambda r: r.arrival):
        srv.submit(r)
    srv.t0 = srv._clock()
    cancelled = set()
    ticks = 0
    while srv.pending or srv.active or srv.starting:
        srv.tick()
        ticks += 1
        if ticks == 3:  # one request still pending, one active mid-run
            assert srv.cancel(13) and srv.pending[-1].rid != 13
            act = [a.req.rid for a in srv.active if a.issued > 0 and a.req.kind == "pwls" and a.req.rid != 6]
            if act:
                assert srv.cancel(act[0])
                cancelled.add(act[0])
            cancelled.add(13)
        assert srv.used >= 0 and len(srv._free_slots) + len(srv.active) + len(srv.starting) == 3
    srv.close()
    return reqs, srv, cancelled, log


@pytest.mark.parametrize("admit_workers", [0, 2])
def test_failures_and_cancellations_stay_with_their_requests(admit_workers):
    reqs, srv, cancelled, log = _serve_with_faults(admit_workers)
    assert len(cancelled) == 2  # one pending, one active mid-run
    by = {r.rid: r for r in reqs}
    assert by[2].status == "failed" and "MemoryError" in by[2].error and by[2].result is None
    assert by[6].status == "failed" and "second unit" in by[6].error
    for rid in cancelled:
        assert by[rid].status == "cancelled"
    assert srv.cancel(13) is False  # no longer held
    others = [r for r in reqs if r.rid not in cancelled | {2, 6}]
    assert all(r.status == "done" for r in others)
    assert sorted(r.rid for r in srv.done) == sorted(r.rid for r in others)
    assert sorted(r.rid for r in srv.failed) == sorted(cancelled | {2, 6})
    # every slot and byte of budget came back; no work was issued for a withdrawn request after it ended
    assert srv.used == 0 and len(srv._free_slots) == 3
    assert all(e[1] not in (2, 13) for e in log if e[0] == "issue")
    # the released device state of a request that failed mid-run
    assert ("release", 6) in {(e[0], e[1]) for e in log}


def test_a_request_whose_plan_reports_an_error_fails_at_retirement():
    log = []

    class _Flagged(_FakeActive):
        def check(self):
            raise RuntimeError("a footprint exceeded the kernel's row buffer")

    srv = ReconServer(hbm_budget=1 << 40, max_active=2, clock=_Clock(),
                      activate=lambda r, s: (_Flagged if r.rid == 1 else _FakeActive)(r, s, log))
    reqs = _requests()[:4]
    done = srv.run(reqs)
    assert sorted(r.rid for r in done) == [0, 2, 3]
    assert reqs[1].status == "failed" and "row buffer" in reqs[1].error and srv.used == 0


@pytest.mark.gpu
def test_served_failure_and_cancellation_leave_other_results_unchanged():
    """On the device: one request's set-up raises (injected on the host, before any device
    work of its own), another is cancelled after its first unit; the rest finish with
    images bit-identical to their solo runs, and the budget is whole again."""
    reqs = _device_requests()
    solo = []
    for r in reqs:
        alone = copy.deepcopy(r)
        ReconServer(max_active=1).run([alone])
        solo.append(_result(alone))
    mixed = copy.deepcopy(reqs)
    fail_rid = mixed[1].rid
    cancel_rid = mixed[3].rid  # an OS-PWLS request (3 iterations)
    srv = ReconServer(max_active=3, admit_workers=2, to_host=True)
    default = srv._activate

    def activate(r, slot):
        if r.rid == fail_rid:
            raise MemoryError("injected set-up failure")
        return default(r, slot)

    srv._activate = activate
    for r in mixed:
        srv.submit(r)
    srv.t0 = srv._clock()
    cancelled = False
    while srv.pending or srv.active or srv.starting:
        srv.tick()
        if not cancelled and any(a.req.rid == cancel_rid and a.issued >= 1 for a in srv.active):
            cancelled = srv.cancel(cancel_rid)
    srv.close()
    assert cancelled
    by = {r.rid: r for r in mixed}
    assert by[fail_rid].status == "failed" and "MemoryError" in by[fail_rid].error
    assert by[cancel_rid].status == "cancelled" and by[cancel_rid].result is None
    assert srv.used == 0
    for i, r in enumerate(mixed):
        if r.rid in (fail_rid, cancel_rid):
            continue
        assert r.status == "done" and np.array_equal(_result(r), solo[i]), (i, r.kind)
