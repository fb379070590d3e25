"""The oracle is pinned before it is trusted.

* against the golden fixtures (outputs of the reference's own compiled C,
  tests/golden/make_golden.py): bit-identical;
* against the reference library itself on fresh seeded inputs, where it is
  available (oracle/_ref): bit-identical;
* a planted mistake in the oracle's inputs is caught (the comparison is live).
"""
import glob
import os

import numpy as np
import pytest

from cases import ARC_KINDS, FAN_KINDS, KINDS, case_inputs, make_arc_cases, make_cases, make_fan_cases
from oracle.bindings import oracle_cbct, ref_available, ref_cbct

GOLDEN_DIR = os.path.join(os.path.dirname(__file__), "golden")
# the arc-detector (DD only) and fan-beam fixtures are checked on their own below
GOLDEN = sorted(p for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz"))
                if not os.path.basename(p).startswith(("arc_", "fan_")))
CASES = make_cases()


def test_golden_fixtures_present():
    names = {os.path.basename(p)[:-4] for p in GOLDEN}
    assert names == set(CASES), "regenerate with tests/golden/make_golden.py"


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_golden(path):
    name = os.path.basename(path)[:-4]
    g = CASES[name]
    d = np.load(path)
    assert np.array_equal(d["betas"], g.betas) and np.array_equal(d["map"], g.map)
    for k in KINDS:
        src = d["image_in"] if k.startswith("proj") else d["sino_in"]
        got = oracle_cbct(k, g, src)
        assert np.array_equal(got, d[k.replace(",", "_")]), f"{name} {k}: oracle differs from the reference output"


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
@pytest.mark.parametrize("name", ["basic", "offsets_curved", "couch_map", "thick_slices"])
def test_oracle_matches_reference_library(name):
    g = CASES[name]
    x, y = case_inputs(g, seed=7)
    for k in KINDS:
        src = x if k.startswith("proj") else y
        assert np.array_equal(oracle_cbct(k, g, src), ref_cbct(k, g, src)), k


def _bench_geometry(which: str, nviews: int):
    """The benchmark scans with ``nviews`` of their views (0, 45, 90, 135 degrees, ...):
    128x128x64 / 256x96 / 360 views, and 512x512x256 / 1024x384 / 720 views."""
    from dataclasses import replace
    from ctsim_b200.phantom import config1, config2, to_projector_units
    g, x_mm = (config1(seed=1) if which == "config1" else config2(seed=2))
    s = g.noViews // 8
    g = replace(g, betas=g.betas[::s][:nviews].copy(), couchZ=g.couchZ[::s][:nviews].copy())
    return g, to_projector_units(x_mm)


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
@pytest.mark.parametrize("which,nviews", [("config1", 4), ("config2", 2)])
def test_oracle_matches_reference_library_on_bench_scans(which, nviews):
    """Bit-identical at the benchmark geometries too (sizes, pitches and magnification of
    the timed runs), on the seeded phantom and a seeded sinogram, for the DD and SF pairs."""
    g, x = _bench_geometry(which, nviews)
    y = np.random.default_rng(3).uniform(0.0, 2.0, g.sino_shape).astype(np.float32)
    for k in ("proj,dd", "back,dd", "proj,tf", "back,tf"):
        src = x if k.startswith("proj") else y
        assert np.array_equal(oracle_cbct(k, g, src), ref_cbct(k, g, src, nthreads=8)
                              if k.startswith("proj") else ref_cbct(k, g, src)), k


def test_planted_mistake_is_detected():
    g = CASES["basic"]
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "basic.npz"))
    x = d["image_in"].copy()
    x[3, 4, 5] += 0.25  # planted on the CPU, in the oracle's input
    assert not np.array_equal(oracle_cbct("proj,dd", g, x), d["proj_dd"])


@pytest.mark.skipif(not ref_available(), reason="reference library not built")
def test_reference_threaded_harness_matches_single_thread():
    g = CASES["couch_map"]
    x, y = case_inputs(g, seed=3)
    a = ref_cbct("proj,dd", g, x)
    b = ref_cbct("proj,dd", g, x, nthreads=4)
    assert np.array_equal(a, b)  # disjoint view slices: identical
    a = ref_cbct("back,tf", g, y)
    b = ref_cbct("back,tf", g, y, nthreads=4)
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6)  # per-thread images summed: reassociated


def test_oracle_adjointness():
    """<A x, y> == <x, A^T y> for the oracle's DD and SF pairs (FP64 dot products)."""
    g = CASES["basic"]
    x, y = case_inputs(g, seed=11)
    for f, b in (("proj,dd", "back,dd"), ("proj,tf", "back,tf")):
        ax = oracle_cbct(f, g, x).astype(np.float64)
        aty = oracle_cbct(b, g, y).astype(np.float64)
        lhs = float(np.sum(ax * y))
        rhs = float(np.sum(x.astype(np.float64) * aty))
        assert abs(lhs - rhs) / abs(lhs) < 1e-6


@pytest.mark.parametrize("name", sorted(make_arc_cases()))
def test_oracle_arc_detector_matches_reference(name):
    """The arc-detector DD pair (detector_type 2) against the reference's cbct_proj3.c /
    cbct_back3.c fixtures: bit-exact; and the pair is adjoint."""
    g = make_arc_cases()[name]
    d = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    for k in ARC_KINDS:
        src = d["image_in"] if k.startswith("proj") else d["sino_in"]
        assert np.array_equal(oracle_cbct(k, g, src), d[k.replace(",", "_")]), k
    x, y = case_inputs(g, seed=3)
    lhs = float(np.sum(oracle_cbct("proj,dd", g, x).astype(np.float64) * y))
    rhs = float(np.sum(x.astype(np.float64) * oracle_cbct("back,dd", g, y)))
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


@pytest.mark.parametrize("name", sorted(make_fan_cases()))
def test_oracle_fan_beam_matches_reference(name):
    """The 2-D fan-beam DD/SF pair against the reference's geom/fbct fixtures: bit-exact."""
    from oracle.bindings import oracle_fbct
    g = make_fan_cases()[name]
    d = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    for k in FAN_KINDS:
        src = d["image_in"] if k.startswith("proj") else d["sino_in"]
        assert np.array_equal(oracle_fbct(k, g, src), d[k.replace(",", "_")]), k
