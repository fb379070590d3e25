"""Batched launches: the A / A^T of many plans (different geometries) in one persistent
grid per launch-shape class, and OS-PWLS instances stepped together -- each result equal,
bit for bit, to what its own plan or solver computes."""
import numpy as np
import pytest

from cases import case_inputs, make_cases

pytestmark = pytest.mark.gpu


def _plans():
    from ctsim_b200 import Plan
    cases = make_cases()
    names = ["basic", "offsets_curved", "couch_map", "thick_slices", "ragged", "short_scan", "tall_curved"]
    return [(cases[n], Plan(cases[n])) for n in names]


@pytest.mark.parametrize("staged", [False, True])
@pytest.mark.parametrize("method", ["dd", "tf"])
def test_batched_launches_equal_per_plan_calls(method, staged):
    import torch
    from ctsim_b200.projector import batch_backproject, batch_project
    gp = _plans()
    if staged:  # forward projections staged through shared memory: two slot counts and the plans' defaults mixed
        for k, (g, p) in enumerate(gp):
            if k % 3 != 2:
                p.set_tuning(proj_layout=3, proj_slots=8 if k % 3 == 0 else 2)
    xs, ys = [], []
    for k, (g, p) in enumerate(gp):
        x, y = case_inputs(g, seed=20 + k)
        xs.append(torch.from_numpy(x).cuda())
        ys.append(torch.from_numpy(y).cuda())
    # full view sets and ordered subsets (start 1, stride 3)
    for vb, vs in ((0, 1), (1, 3)):
        outs, ents = [], []
        for (g, p), x in zip(gp, xs):
            vc = len(range(vb, g.noViews, vs))
            o = torch.full((vc, g.nu, g.nv), float("nan"), device="cuda")
            outs.append(o)
            ents.append((p, x, o, vb, vs, vc))
        batch_project(method, ents)
        for (g, p), x, o, e in zip(gp, xs, outs, ents):
            assert torch.equal(o, p.project(x, method, vb, vs, e[5]))
        imgs, ents = [], []
        for (g, p), y in zip(gp, ys):
            vc = len(range(vb, g.noViews, vs))
            ysub = y[vb::vs].contiguous()
            o = torch.full(g.image_shape, float("nan"), device="cuda")
            imgs.append((o, ysub))
            ents.append((p, ysub, o, vb, vs, vc, 2.5))
        batch_backproject(method, ents)
        for (g, p), (o, ysub), e in zip(gp, imgs, ents):
            assert torch.equal(o, p.backproject(ysub, method, vb, vs, e[5], scale=2.5))


@pytest.mark.parametrize("method", ["dd", "tf"])
def test_batched_backprojection_with_different_row_buffers(method):
    """Plans whose A^T row buffers differ (detector height and magnification) in one
    persistent grid, with ragged column tiles (nx not a multiple of 8); the 160 x 162
    image (over four waves of the single-plan kernel) runs on that kernel instead."""
    import torch
    from ctsim_b200 import CTGeometry, Plan, circular_betas
    from ctsim_b200.projector import batch_backproject
    ents, refs = [], []
    for k, (n, nz, nv, dz) in enumerate([(21, 40, 96, 1.0), (19, 8, 24, 1.0), (27, 60, 200, 0.5), (13, 20, 48, 2.0),
                                         (30, 33, 140, 1.0), (17, 70, 260, 0.7), (160, 16, 48, 1.0)]):
        g = CTGeometry((n, n + 2, nz), (1.0, 1.0, dz), (0, 0, 0), (40, nv), (1.6, 1.0), (0, 0), 1000.0, 500.0, 1500.0,
                       circular_betas(9 + k))
        p = Plan(g)
        y = torch.rand(g.sino_shape, device="cuda")
        o = torch.empty(g.image_shape, device="cuda")
        ents.append((p, y, o, 0, 1, g.noViews, 1.0))
        refs.append((p, y))
    batch_backproject(method, ents)
    for (p, y), e in zip(refs, ents):
        assert torch.equal(e[2], p.backproject(y, method))


def test_batch_larger_than_one_launch_and_errors():
    """70 plans: more than the 64 tasks one launch carries; duplicates and mixed devices refused."""
    import torch
    from ctsim_b200 import CTGeometry, Plan, circular_betas
    from ctsim_b200._lib import CtsimError
    from ctsim_b200.projector import batch_project
    rng = np.random.default_rng(3)
    ents, refs = [], []
    for k in range(70):
        n = int(rng.integers(6, 14))
        g = CTGeometry((n, n + 1, 5), (1.0, 1.0, 1.0), (0, 0, 0), (24, 8), (1.6, 1.6), (0, 0), 1000.0, 500.0, 1500.0,
                       circular_betas(int(rng.integers(3, 7))))
        p = Plan(g)
        x = torch.rand(g.image_shape, device="cuda")
        o = torch.empty((g.noViews, g.nu, g.nv), device="cuda")
        ents.append((p, x, o, 0, 1, g.noViews))
        refs.append((p, x))
    batch_project("dd", ents)
    for (p, x), e in zip(refs, ents):
        assert torch.equal(e[2], p.project(x, "dd"))
    with pytest.raises(CtsimError, match="once"):
        batch_project("dd", [ents[0], ents[0]])


def test_batched_pwls_equals_each_solver():
    """Three OS-PWLS instances of different geometries stepped together (graphs after the
    first iteration) give exactly the images of three separate reconPwlsSeSqs runs."""
    import torch
    from ctsim_b200 import Plan
    from ctsim_b200.pwls import BatchedPwls, PwlsSolver, reconPwlsSeSqs
    cases = make_cases()
    inst = []
    for k, n in enumerate(["basic", "short_scan", "ragged"]):
        g = cases[n]
        x, _ = case_inputs(g, seed=40 + k)
        p = Plan(g)
        line = p.project(torch.from_numpy(x * 0.02).cuda(), "tf")
        counts = torch.poisson(1e4 * torch.exp(-line))
        y = torch.log(1e4 / counts.clamp(min=10.0))
        inst.append((g, y, counts, torch.full(g.image_shape, 0.01, device="cuda")))
    solvers = [PwlsSolver(y, w, g, 2.0, "huber", 0.01, 4, x0, plan=Plan(g)) for g, y, w, x0 in inst]
    b = BatchedPwls(solvers)
    hist = [b.step() for _ in range(3)]
    for s, (g, y, w, x0), k in zip(solvers, inst, range(3)):
        x_ref, phis, rmsds = reconPwlsSeSqs(y, w, g, 2.0, "huber", 3, 0.01, 4, x0, stopCrt=-1.0)
        assert torch.equal(s.x, x_ref)
        assert np.allclose([h[k][0] for h in hist], phis, rtol=1e-9)


@pytest.mark.parametrize("method", ["dd", "tf"])
def test_batched_low_precision_storage_equals_per_plan_calls(method):
    """bfloat16 / float16 / float32 buffers per item (FP32 arithmetic): each result equals
    its plan's own _ex call bit for bit, for A and A^T, in both directions of widening."""
    import torch
    from ctsim_b200.projector import batch_backproject, batch_project
    gp = _plans()[:4]
    dts = [(torch.bfloat16, torch.float32), (torch.float16, torch.float16), (torch.float32, torch.bfloat16),
           (torch.bfloat16, torch.bfloat16)]
    fwd, back, refs = [], [], []
    for k, ((g, p), (din, dout)) in enumerate(zip(gp, dts)):
        x, y = case_inputs(g, seed=40 + k)
        xd = torch.from_numpy(x).cuda().to(din)
        yd = torch.from_numpy(y).cuda().to(din)
        so = torch.empty(g.sino_shape, dtype=dout, device="cuda")
        io = torch.empty(g.image_shape, dtype=dout, device="cuda")
        fwd.append((p, xd, so, 0, 1, g.noViews))
        back.append((p, yd, io, 0, 1, g.noViews, 0.5))
        refs.append((p, xd, yd, dout))
    batch_project(method, fwd)
    batch_backproject(method, back)
    for (p, xd, yd, dout), f, b in zip(refs, fwd, back):
        assert torch.equal(f[2], p.project(xd, method, out_dtype=dout))
        assert torch.equal(b[2], p.backproject(yd, method, scale=0.5, out_dtype=dout))
