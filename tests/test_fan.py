"""2-D fan-beam DD/SF pair (geom/fbct) on the device against the reference's fixtures."""
import os

import numpy as np
import pytest

from cases import FAN_KINDS, case_inputs, make_fan_cases

GOLDEN_DIR = os.path.join(os.path.dirname(__file__), "golden")
CASES = make_fan_cases()


def _mex(kind, g, data):
    from ctsim_b200.fan import fbct_geom_mex
    return fbct_geom_mex(kind, g.reconSize, g.reconSpacing, g.reconOffset, g.nu, g.du, g.detOffset, g.SAD, g.ADD,
                         g.SDD, g.noViews, g.betas, g.flatPanel, data)


def test_fan_mex_rejects_bad_arguments():
    g = CASES["fan_basic"]
    x, y = case_inputs(g)
    with pytest.raises(ValueError, match="unknown geom type"):
        _mex("proj,rd", g, x)
    with pytest.raises(ValueError, match="shape"):
        _mex("proj,dd", g, x.T)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_fan_matches_reference(name):
    """Flat detectors: bit-identical to the reference's C (same operations, same order);
    curved: within 1e-5 (the atan of the CUDA and C math libraries may differ in the last
    bit of a double)."""
    g = CASES[name]
    d = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    for k in FAN_KINDS:
        src = d["image_in"] if k.startswith("proj") else d["sino_in"]
        ref = d[k.replace(",", "_")]
        got = _mex(k, g, src)
        if g.flatPanel == 1:
            assert np.array_equal(got, ref), f"{name} {k}: max {np.abs(got - ref).max():.3e}"
        else:
            err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert err <= 1e-5, f"{name} {k}: rel L2 {err:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fan_basic", "fan_offsets_curved"])
def test_fan_plan_adjoint_and_subsets(name):
    import torch
    from ctsim_b200.fan import FanPlan
    from oracle.bindings import oracle_fbct
    g = CASES[name]
    x, y = case_inputs(g, seed=8)
    p = FanPlan(g)
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    for m in ("dd", "tf"):
        ax32 = p.project(xd, m).cpu().numpy()
        ax = ax32.astype(np.float64)
        aty = p.backproject(yd, m).cpu().numpy().astype(np.float64)
        lhs, rhs = float(np.sum(ax * y)), float(np.sum(x * aty))
        # the SF back-projector's bin range ends at ceil where the projector's ends at
        # floor; the extra bin carries zero weight, so the pair stays adjoint
        assert abs(lhs - rhs) <= 1e-6 * abs(lhs), (m, lhs, rhs)
        M = 3
        for s in range(M):
            sub = p.project(xd, m, s, M).cpu().numpy()
            assert np.array_equal(sub, ax32[s::M])
            ys = np.ascontiguousarray(y[s::M])
            bs = p.backproject(torch.from_numpy(ys).cuda(), m, s, M, scale=2.0).cpu().numpy()
            from ctsim_b200.geometry import FanGeometry
            gs = FanGeometry(g.reconSize, g.reconSpacing, g.reconOffset, g.nu, g.du, g.detOffset, g.SAD, g.ADD, g.SDD,
                             g.betas[s::M], g.flatPanel)
            want = 2.0 * oracle_fbct(f"back,{m}", gs, ys)
            assert np.linalg.norm(bs - want) <= 1e-5 * np.linalg.norm(want)
