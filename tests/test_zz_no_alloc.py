"""The backprojection entry point that allocates no device memory.

ctsim_back_dd_noalloc serves callers that cannot allocate device memory
themselves (a framework owning all device memory through its own pool, a
serving loop with a fixed budget, code that cannot afford the device
synchronisation of cudaMalloc/cudaFree).  It keeps its tables in one fixed
device array shared by all calls, so the GPU test calls it twice in a row with
different sinograms, on a flat detector and on a curved one with couch shifts,
and checks each result against the plan API's matched distance-driven
backprojection and against the oracle, with the parity tolerance of the other
tests.  Collected last so that a failure here comes after every other test has
run.
"""
import ctypes

import numpy as np
import pytest

from ctsim_b200 import CTGeometry, _lib, circular_betas

REL_L2 = 1e-5


def _geom_struct(g):
    return _lib.CtsimGeom(*g.scalars()[:18], g.noViews, int(g.flatPanel))


def _rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _flat():
    return CTGeometry((96, 80, 40), (1.0, 1.0, 1.0), (0.5, -0.25, 0.0), (192, 72), (1.6, 1.6), (1.0, 0.0), 1000.0,
                      500.0, 1500.0, circular_betas(90), map=np.random.default_rng(4).random((80, 96)) > 0.1)


def _curved_couch():
    n = 60
    return CTGeometry((72, 88, 36), (1.0, 1.0, 1.2), (-1.0, 0.5, 2.0), (160, 64), (1.4, 1.5), (-2.0, 1.5), 1000.0,
                      500.0, 1500.0, circular_betas(n), couchZ=np.linspace(-6.0, 6.0, n).astype(np.float32),
                      flatPanel=0)


@pytest.mark.gpu
@pytest.mark.parametrize("make", [_flat, _curved_couch], ids=["flat", "curved_couch"])
def test_noalloc_backprojection_matches_plan_on_two_calls(make):
    import torch
    from ctsim_b200.projector import Plan
    from oracle.bindings import oracle_cbct

    g = make()
    L = _lib.load()
    gs = _geom_struct(g)
    betas = np.ascontiguousarray(g.betas)
    couch = np.ascontiguousarray(g.couchZ)
    mp = np.ascontiguousarray(g.map)
    plan = Plan(g)
    rng = np.random.default_rng(12)
    stream = torch.cuda.current_stream()
    for call in range(2):
        y_host = rng.random(g.sino_shape, dtype=np.float32) * (call + 1)
        y = torch.from_numpy(y_host).cuda()
        want = plan.backproject(y, "dd").cpu().numpy()
        out = torch.full(g.image_shape, float("nan"), dtype=torch.float32, device="cuda")
        st = L.ctsim_back_dd_noalloc(ctypes.byref(gs), betas.ctypes.data, couch.ctypes.data, mp.ctypes.data,
                                     y.data_ptr(), out.data_ptr(), stream.cuda_stream)
        assert st == 0, _lib.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        err = _rel_l2(got, want)
        assert err <= REL_L2, f"call {call}: rel L2 {err:.2e} against the plan API"
        err = _rel_l2(got, oracle_cbct("back,dd", g, y_host))
        assert err <= REL_L2, f"call {call}: rel L2 {err:.2e} against the oracle"
        assert np.all(got[:, ~g.map] == 0)


def test_noalloc_rejects_geometry_beyond_its_scratch():
    """The size check comes before any device work: a geometry whose tables exceed
    the fixed scratch is refused with a clear error."""
    g = CTGeometry((2048, 2048, 4), (0.1, 0.1, 0.1), (0, 0, 0), (2048, 1024), (0.2, 0.2), (0, 0), 1000.0, 500.0,
                   1500.0, circular_betas(4))
    L = _lib.load()
    gs = _geom_struct(g)
    betas = np.ascontiguousarray(g.betas)
    couch = np.ascontiguousarray(g.couchZ)
    buf = np.zeros(4, np.float32)
    st = L.ctsim_back_dd_noalloc(ctypes.byref(gs), betas.ctypes.data, couch.ctypes.data, None, buf.ctypes.data,
                                 buf.ctypes.data, None)
    assert st == 1
    assert "8 MiB" in _lib.last_error()
