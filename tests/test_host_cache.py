"""The host-pointer entry points keep the last geometry's plan and buffers between calls
and return the forward projection in view chunks.  Neither may change a result: every
call must equal a fresh, uncached call and the device-plan path bit for bit."""
import numpy as np
import pytest

from cases import KINDS, case_inputs, make_cases
from ctsim_b200 import CTGeometry, circular_betas
from ctsim_b200 import _lib
from ctsim_b200.projector import Plan, cbct_geom_mex

pytestmark = pytest.mark.gpu


def mex(kind, g, data):
    return cbct_geom_mex(kind, g.reconSize, g.reconSpacing, g.reconOffset, g.detSize, g.detSpacing, g.detOffset,
                         g.SAD, g.ADD, g.SDD, g.noViews, g.betas, g.couchZ, g.flatPanel, data, g.map)


def _geom(views, offset=0.0, turn=0.0, map=None, size=(96, 80, 24)):
    return CTGeometry(size, (1.0, 1.0, 1.0), (0.5, -0.25, 0), (160, 40), (1.2, 1.2), (offset, 0), 1000.0,
                      500.0, 1500.0, circular_betas(views) + turn, map=map)


def _uncached(kind, g, data):
    L = _lib.load()
    L.ctsim_host_cache_enable(0)
    try:
        return mex(kind, g, data)
    finally:
        L.ctsim_host_cache_enable(1)


@pytest.mark.parametrize("views,size", [(1, (96, 80, 24)), (5, (96, 80, 24)), (37, (96, 80, 24)),
                                        (11, (7, 3, 40)), (70, (96, 80, 24))])
def test_cached_calls_equal_uncached_and_plan(views, size):
    """Chunks of one view, fewer views than chunks, uneven chunks; fewer image rows than
    y slabs; with 64 views or more a short first (A^T) or last (A) chunk."""
    import torch
    g = _geom(views, size=size)
    x, y = case_inputs(g, seed=views)
    plan = Plan(g)
    _lib.load().ctsim_host_cache_release()
    for kind in KINDS:
        src = x if kind.startswith("proj") else y
        fresh = _uncached(kind, g, src)
        first = mex(kind, g, src)   # builds the cache (or reuses it from the previous kind)
        again = mex(kind, g, src)   # reuses it
        assert np.array_equal(first, fresh), kind
        assert np.array_equal(again, fresh), kind
        method = kind.split(",")[1]
        if kind.startswith("proj"):
            dev = plan.project(torch.from_numpy(x).cuda(), method).cpu().numpy()
        else:
            dev = plan.backproject(torch.from_numpy(y).cuda(), method).cpu().numpy()
        assert np.array_equal(first, dev), kind
    plan.close()


def test_geometry_change_rebuilds():
    """Alternating geometries (views, a detector offset, betas, a map) never serve a
    result from the other geometry's tables."""
    m = np.ones((80, 96), dtype=bool)
    m[:10] = False
    g1, g2, g3, g4, g5 = _geom(12), _geom(12, offset=1.5), _geom(13), _geom(12, turn=0.01), _geom(12, map=m)
    x, _ = case_inputs(g1, seed=2)
    want = {id(g): _uncached("proj,dd", g, x) for g in (g1, g2, g3, g4, g5)}
    assert not np.array_equal(want[id(g1)], want[id(g2)])
    assert not np.array_equal(want[id(g1)], want[id(g4)])
    assert not np.array_equal(want[id(g1)], want[id(g5)])
    for g in (g1, g2, g1, g3, g3, g4, g1, g5, g1):
        assert np.array_equal(mex("proj,dd", g, x), want[id(g)])
    _lib.load().ctsim_host_cache_release()
    assert np.array_equal(mex("proj,dd", g1, x), want[id(g1)])


@pytest.mark.parametrize("name", ["ragged", "offsets_curved"])
def test_reference_cases_through_the_cache(name):
    g = make_cases()[name]
    x, y = case_inputs(g, seed=9)
    for kind in KINDS:
        src = x if kind.startswith("proj") else y
        assert np.array_equal(mex(kind, g, src), _uncached(kind, g, src)), (name, kind)


def test_threads_with_different_geometries():
    """Threads calling the drop-in functions at once, each with its own geometry, on one
    device: every result equals the uncached one."""
    from concurrent.futures import ThreadPoolExecutor
    gs = [_geom(9), _geom(10, offset=0.5), _geom(9, turn=0.2)]
    x, y = case_inputs(gs[0], seed=4)
    want = [(_uncached("proj,dd", g, x), _uncached("back,tf", g, case_inputs(g, seed=4)[1])) for g in gs]

    def work(k):
        g = gs[k % len(gs)]
        yk = case_inputs(g, seed=4)[1]
        return k, [(mex("proj,dd", g, x), mex("back,tf", g, yk)) for _ in range(3)]

    with ThreadPoolExecutor(4) as ex:
        for k, outs in ex.map(work, range(8)):
            for a, b in outs:
                assert np.array_equal(a, want[k % len(gs)][0]) and np.array_equal(b, want[k % len(gs)][1]), k


def test_pageable_buffers_match_pinned_buffers():
    """Pageable caller buffers go through pinned staging buffers (32 MB pieces, four of them,
    filled and drained by a host thread pool); page-locked buffers are copied directly.
    A 164 MB image takes six pieces each way, so every staging buffer is reused.  Both
    routes give the device plan's result bit for bit."""
    import torch
    g = CTGeometry((320, 320, 400), (0.5, 0.5, 0.5), (0.25, 0, 0), (512, 640), (0.8, 0.8), (0, 0), 1000.0, 500.0,
                   1500.0, circular_betas(4))
    x, y = case_inputs(g, seed=41)
    L = _lib.load()
    sc = g.scalars()
    betas = np.ascontiguousarray(g.betas)
    couch = np.ascontiguousarray(g.couchZ)
    mp = np.ascontiguousarray(g.map)

    def run(img_in, sino_out, img_out, sino_in):
        assert L.ctsim_proj_dd(*sc, betas.ctypes.data, couch.ctypes.data, g.flatPanel, img_in.ctypes.data,
                               sino_out.ctypes.data, mp.ctypes.data), _lib.last_error()
        assert L.ctsim_back_dd(*sc, betas.ctypes.data, couch.ctypes.data, g.flatPanel, img_out.ctypes.data,
                               sino_in.ctypes.data, mp.ctypes.data), _lib.last_error()

    pageable = (np.ascontiguousarray(x), np.empty(g.sino_shape, np.float32), np.empty(g.image_shape, np.float32),
                np.ascontiguousarray(y))
    pin = [torch.from_numpy(pageable[0]).pin_memory(), torch.empty(g.sino_shape).pin_memory(),
           torch.empty(g.image_shape).pin_memory(), torch.from_numpy(pageable[3]).pin_memory()]
    pinned = tuple(t.numpy() for t in pin)
    run(*pageable)
    run(*pinned)
    assert np.array_equal(pageable[1], pinned[1])
    assert np.array_equal(pageable[2], pinned[2])
    plan = Plan(g)
    assert np.array_equal(pageable[1], plan.project(torch.from_numpy(x).cuda(), "dd").cpu().numpy())
    assert np.array_equal(pageable[2], plan.backproject(torch.from_numpy(y).cuda(), "dd").cpu().numpy())
    plan.close()
    L.ctsim_host_cache_release()
