"""Parity of the CUDA projectors with the oracle (GPU).

Tolerance (FP32 projectors): relative L2 error <= 1e-5 against the reference's
own outputs; matched-adjoint identity <A x, y> = <x, A^T y> to 1e-6 relative for
the CUDA pair.  The voxel-driven FDK backprojection accumulates views in the
reference's order with the same float operations and is checked bit-for-bit on
flat panels.
"""
import glob
import os

import numpy as np
import pytest

from cases import ARC_KINDS, KINDS, case_inputs, make_arc_cases, make_cases
from ctsim_b200 import CTGeometry, circular_betas
from ctsim_b200.projector import Plan, cbct_geom_mex
from oracle.bindings import oracle_cbct

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
ADJ = 1e-6
GOLDEN_DIR = os.path.join(os.path.dirname(__file__), "golden")
CASES = make_cases()


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    n = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (n if n > 0 else 1.0)


def mex(kind, g, data):
    return cbct_geom_mex(kind, g.reconSize, g.reconSpacing, g.reconOffset, g.detSize, g.detSpacing, g.detOffset,
                         g.SAD, g.ADD, g.SDD, g.noViews, g.betas, g.couchZ, g.flatPanel, data, g.map)


@pytest.mark.parametrize("name", sorted(CASES))
def test_cuda_matches_golden(name):
    g = CASES[name]
    d = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    for k in KINDS:
        src = d["image_in"] if k.startswith("proj") else d["sino_in"]
        ref = d[k.replace(",", "_")]
        got = mex(k, g, src)
        err = rel_l2(got, ref)
        assert err <= REL_L2, f"{name} {k}: rel L2 {err:.3e}"
        if k in ("back,pd", "back,hpd", "back,var") and g.flatPanel == 1:
            assert np.array_equal(got, ref), f"{name} {k}: not bit-identical (max {np.abs(got - ref).max():.3e})"


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("slots", [1, 8])
def test_staged_forward_projector_matches_golden(name, slots):
    """The forward projector with the candidates' prefix columns staged in shared memory
    (layout 3), whatever the plan's default, against the reference's outputs."""
    import torch
    g = CASES[name]
    d = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    plan = Plan(g)
    plan.set_tuning(proj_layout=3, proj_slots=slots)
    xd = torch.from_numpy(np.ascontiguousarray(d["image_in"])).cuda()
    for m in ("dd", "tf"):
        got = plan.project(xd, m).cpu().numpy()
        plan.check()
        err = rel_l2(got, d[f"proj_{m}"])
        assert err <= REL_L2, f"{name} proj,{m} (staged, {slots} slots): rel L2 {err:.3e}"


@pytest.mark.parametrize("name", ["basic", "offsets_curved", "thick_slices", "ragged"])
def test_device_plan_matches_oracle_and_is_adjoint(name):
    import torch
    g = CASES[name]
    x, y = case_inputs(g, seed=5)
    plan = Plan(g)
    xd = torch.from_numpy(x).cuda()
    yd = torch.from_numpy(y).cuda()
    for m in ("dd", "tf"):
        ax = plan.project(xd, m).cpu().numpy()
        aty = plan.backproject(yd, m).cpu().numpy()
        plan.check()
        assert rel_l2(ax, oracle_cbct(f"proj,{m}", g, x)) <= REL_L2
        assert rel_l2(aty, oracle_cbct(f"back,{m}", g, y)) <= REL_L2
        lhs = float(np.sum(ax.astype(np.float64) * y))
        rhs = float(np.sum(x.astype(np.float64) * aty))
        assert abs(lhs - rhs) / abs(lhs) <= ADJ, f"{m}: adjoint mismatch {abs(lhs - rhs) / abs(lhs):.2e}"


def test_ordered_subsets_on_device():
    import torch
    g = CASES["short_scan"]
    x, y = case_inputs(g, seed=9)
    plan = Plan(g)
    xd = torch.from_numpy(x).cuda()
    M = 4
    for isub in range(M):
        gs = g.subset(M, isub)
        start = isub % M
        got = plan.project(xd, "tf", start, M).cpu().numpy()
        assert rel_l2(got, oracle_cbct("proj,tf", gs, x)) <= REL_L2
        ysub = np.ascontiguousarray(y[start::M])
        got = plan.backproject(torch.from_numpy(ysub).cuda(), "tf", start, M, scale=float(M)).cpu().numpy()
        assert rel_l2(got, M * oracle_cbct("back,tf", gs, ysub)) <= REL_L2


def test_launch_order_is_result_neutral():
    """Blocks run in groups of 32 consecutive launch views with a shorter last group; every
    block is independent, so one launch over 70 views (32 + 32 + 6), a strided subset
    launch and single-view launches give the same bits, for both prefix layouts."""
    import torch
    g = CTGeometry((20, 18, 12), (1.0, 1.0, 1.0), (0.2, -0.1, 0), (40, 24), (1.2, 1.2), (0, 0), 1000.0, 500.0,
                   1500.0, circular_betas(70))
    x, _ = case_inputs(g, seed=31)
    xd = torch.from_numpy(x).cuda()
    plan = Plan(g)
    for layout, slots in ((2, 0), (3, 8)):
        plan.set_tuning(proj_layout=layout, proj_slots=slots)
        for m in ("dd", "tf"):
            full = plan.project(xd, m).cpu().numpy()
            assert rel_l2(full, oracle_cbct(f"proj,{m}", g, x)) <= REL_L2
            single = np.stack([plan.project(xd, m, v, 1, 1).cpu().numpy()[0] for v in range(g.noViews)])
            assert np.array_equal(full, single)
            sub = plan.project(xd, m, 3, 4).cpu().numpy()  # views 3, 7, ..., 67
            assert np.array_equal(sub, full[3::4])


def config1_geometry(n_views):
    """Config-1 shapes (128^2 x 64 at 1 mm; flat 256 x 96 detector at 1.6 mm; SAD 1000, SDD 1500)."""
    return CTGeometry((128, 128, 64), (1.0, 1.0, 1.0), (0, 0, 0), (256, 96), (1.6, 1.6), (0, 0), 1000.0, 500.0,
                      1500.0, circular_betas(360)[:: 360 // n_views][:n_views])


@pytest.mark.parametrize("kind", KINDS)
def test_config1_shapes(kind):
    g = config1_geometry(12)
    x, y = case_inputs(g, seed=1)
    src = x if kind.startswith("proj") else y
    err = rel_l2(mex(kind, g, src), oracle_cbct(kind, g, src))
    assert err <= REL_L2, f"{kind}: rel L2 {err:.3e}"


def projectors_3d_geometry(views=120):
    """The reference's own projector regression geometry (geom/test_projectors_3d.m:41-66):
    256 x 256 x 128 voxels of 1 mm offset by (10, 10, 0) voxels, a curved 512 x 256
    detector of 0.7 x 0.58 mm offset by (10, 0) pixels, SAD 1000, SDD 1500, 120 views
    over the full turn (every 120/views-th of them here)."""
    b = (np.arange(120) * 2 * np.pi / 120)[:: 120 // views][:views]
    return CTGeometry((256, 256, 128), (1.0, 1.0, 1.0), (10, 10, 0), (512, 256), (0.7, 0.58), (10, 0), 1000.0,
                      500.0, 1500.0, b, flatPanel=0)


def projectors_3d_phantom(n=256):
    """The script's phantom (geom/test_projectors_3d.m:4-40): three discs (values 1, 2, 5)
    stacked over n/2 slices, halved from slice 3n/8 (1-based) up; [nz, ny, nx]."""
    ix = np.arange(1, n + 1) + 0.5
    iix = np.ones((n, 1)) * ix  # MATLAB iix(i, j) = ix(j)
    iiy = iix.T
    I = np.zeros((n, n))
    I[np.sqrt((iix - round(n / 2)) ** 2 + (iiy - round(n / 2)) ** 2) < round(n / 3)] = 1
    I[np.sqrt((iix - round(n * 2 / 3)) ** 2 + (iiy - round(n / 2)) ** 2) < round(n / 12)] = 2
    I[np.sqrt((iix - round(n / 2)) ** 2 + (iiy - round(n / 3)) ** 2) < round(n / 32)] = 5
    # MATLAB img(:, :, k) = I is [x y] with x = first index: I's rows are x
    img = np.repeat(I.T[None].astype(np.float32), n // 2, axis=0)
    img[n // 8 * 3 - 1:] /= 2
    return np.ascontiguousarray(img)


@pytest.mark.parametrize("kind", KINDS)
def test_reference_regression_geometry(kind):
    """geom/test_projectors_3d.m's geometry and phantom, 12 of its 120 views, against the
    oracle; the sinogram of the back kinds is the oracle's own SF projection."""
    g = projectors_3d_geometry(12)
    x = projectors_3d_phantom()
    src = x if kind.startswith("proj") else oracle_cbct("proj,tf", g, x)
    err = rel_l2(mex(kind, g, src), oracle_cbct(kind, g, src))
    assert err <= REL_L2, f"{kind}: rel L2 {err:.3e}"


def test_reference_regression_geometry_adjoint():
    """All 120 views of geom/test_projectors_3d.m: <A x, y> = <x, A^T y> for both pairs."""
    import torch
    g = projectors_3d_geometry(120)
    plan = Plan(g)
    x = torch.from_numpy(projectors_3d_phantom()).cuda()
    y = torch.rand(g.sino_shape, device="cuda", generator=torch.Generator(device="cuda").manual_seed(3))
    for m in ("dd", "tf"):
        ax = plan.project(x, m).double()
        aty = plan.backproject(y, m).double()
        lhs, rhs = float((ax * y.double()).sum()), float((x.double() * aty).sum())
        assert abs(lhs - rhs) <= ADJ * abs(lhs), (m, lhs, rhs)
    plan.close()


def test_map_off_columns_are_zero_and_skipped():
    import torch
    g = CASES["couch_map"]
    x, y = case_inputs(g, seed=2)
    plan = Plan(g)
    img = plan.backproject(torch.from_numpy(y).cuda(), "dd").cpu().numpy()
    assert np.all(img[:, ~g.map] == 0)
    # image content in map-off columns must not reach the sinogram
    x2 = x.copy()
    x2[:, ~g.map] = 123.0
    a = plan.project(torch.from_numpy(x).cuda(), "dd").cpu().numpy()
    b = plan.project(torch.from_numpy(x2).cuda(), "dd").cpu().numpy()
    assert np.array_equal(a, b)


def test_single_view_and_empty_volume():
    import torch
    g = CASES["basic"]
    g1 = g.subset(11, 3)
    x = np.zeros(g1.image_shape, np.float32)
    assert np.count_nonzero(mex("proj,dd", g1, x)) == 0
    y = np.ones(g1.sino_shape, np.float32)
    assert rel_l2(mex("back,dd", g1, y), oracle_cbct("back,dd", g1, y)) <= REL_L2


@pytest.mark.parametrize("name", sorted(make_arc_cases()))
def test_arc_detector_matches_reference(name):
    """Arc detector (detector_type 2): the DD pair against the reference's cbct_proj3.c /
    cbct_back3.c fixtures and adjoint; the other methods are refused."""
    import torch
    from ctsim_b200._lib import CtsimError
    g = make_arc_cases()[name]
    d = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    for k in ARC_KINDS:
        src = d["image_in"] if k.startswith("proj") else d["sino_in"]
        err = rel_l2(mex(k, g, src), d[k.replace(",", "_")])
        assert err <= REL_L2, f"{name} {k}: rel L2 {err:.3e}"
    x, y = case_inputs(g, seed=4)
    plan = Plan(g)
    ax = plan.project(torch.from_numpy(x).cuda(), "dd").cpu().numpy()
    aty = plan.backproject(torch.from_numpy(y).cuda(), "dd").cpu().numpy()
    lhs = float(np.sum(ax.astype(np.float64) * y))
    rhs = float(np.sum(x.astype(np.float64) * aty))
    assert abs(lhs - rhs) / abs(lhs) <= ADJ
    for m in ("tf", "pd", "hpd", "var"):
        with pytest.raises(CtsimError, match="arc"):
            plan.backproject(torch.from_numpy(y).cuda(), m)
    with pytest.raises(CtsimError, match="arc"):
        plan.project(torch.from_numpy(x).cuda(), "tf")


def test_helical_scan_matches_oracle():
    """A three-turn helical scan (loadProjectionGeometryHelicalCT.m): every method through
    the couch shifts against the oracle."""
    from ctsim_b200.geometry import helical_geometry
    g = helical_geometry((20, 20, 16), (1.0, 1.0, 1.0), (0, 0, 0), (40, 12), (1.6, 1.6), (0, 0), 1000.0, 500.0,
                         16, 3, 1.0)
    assert g.noViews == 49 and abs(float(g.couchZ[-1]) - 24 * 12 * 1.6 / 16) < 1e-4
    x, y = case_inputs(g, seed=6)
    for k in KINDS:
        src = x if k.startswith("proj") else y
        err = rel_l2(mex(k, g, src), oracle_cbct(k, g, src))
        assert err <= REL_L2, f"{k}: rel L2 {err:.3e}"


def test_launch_shapes_keep_parity_and_autotune():
    """Every valid launch shape stays within the parity bar (the FDK kernel's z blocks are
    bit-neutral); the autotuner picks a valid shape and records it for the shape class."""
    import torch
    from ctsim_b200._lib import CtsimError
    # a tall detector (160 rows: 64 row threads cover it in one pass, 32 walk the shadows)
    g = CTGeometry((14, 12, 30), (1.0, 1.0, 1.0), (0.3, 0, 0), (36, 160), (1.6, 0.5), (0, 0), 1000.0, 500.0, 1500.0,
                   circular_betas(7))
    x, y = case_inputs(g, seed=12)
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    plan = Plan(g)
    hpd0 = plan.backproject(yd, "hpd").cpu().numpy()
    for G in (1, 2, 4, 8):
        # plain prefix sums / (sum, slope) pairs / plain sums staged in shared memory (1 or 8 slots)
        for layout, slots in ((1, 0), (2, 0), (3, 1), (3, 8)):
            same = None
            for R in (64, 32):  # fewer row threads than rows: passes; 32: walks each candidate's rows
                try:
                    plan.set_tuning(proj_groups=G, proj_rows=R, proj_layout=layout, proj_slots=slots)
                except CtsimError:
                    continue
                for m in ("dd", "tf"):
                    a = plan.project(xd, m).cpu().numpy()
                    assert rel_l2(a, oracle_cbct(f"proj,{m}", g, x)) <= REL_L2
                    if m == "dd":  # the row mapping does not change the arithmetic
                        assert same is None or np.array_equal(a, same)
                        same = a
    for mz in (1, 2, 4, 8):
        plan.set_tuning(pd_mz=mz)
        assert np.array_equal(plan.backproject(yd, "hpd").cpu().numpy(), hpd0)
        try:
            plan.set_tuning(back_mz=mz, back_mz_tf=mz)
        except CtsimError:
            continue
        for m in ("dd", "tf"):
            assert rel_l2(plan.backproject(yd, m).cpu().numpy(), oracle_cbct(f"back,{m}", g, y)) <= REL_L2
    with pytest.raises(CtsimError):
        plan.set_tuning(proj_groups=3)
    t = Plan(g).autotune("proj,tf", 4)
    assert t["proj_groups"] in (1, 2, 4, 8)
    t2 = Plan(g).autotune("back,tf", 4)
    assert t2["back_mz_tf"] in (1, 2, 4, 8)
