"""The C-ABI library builds, loads and exports every symbol include/ctsim_b200.h
declares; the reference-facing Python API validates its arguments like the MEX
gateway and reports errors without killing the process.  No GPU needed."""
import ctypes
import os
import re

import numpy as np
import pytest

import ctsim_b200
from ctsim_b200 import _lib
from ctsim_b200.projector import cbct_geom_mex
from cases import make_cases

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "ctsim_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ctsim_[a-z_]+)\s*\(", text)))


def test_library_loads_and_exports_header_symbols():
    L = _lib.load()
    names = header_functions()
    assert len(names) >= 14
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.EXPORTED)
    assert b"sm_100a" in L.ctsim_version()


def test_library_is_in_tree():
    assert os.path.exists(_lib.lib_path())
    assert os.path.dirname(_lib.lib_path()).endswith(os.path.join("ctsim_b200", "_lib"))


def _args(g):
    return (g.reconSize, g.reconSpacing, g.reconOffset, g.detSize, g.detSpacing, g.detOffset, g.SAD, g.ADD, g.SDD,
            g.noViews, g.betas, g.couchZ, g.flatPanel)


def test_mex_argument_checks():
    g = make_cases()["basic"]
    x = np.zeros(g.image_shape, np.float32)
    with pytest.raises(ValueError, match="unknown geom type"):
        cbct_geom_mex("proj,rd", *_args(g), x, g.map)
    with pytest.raises(ValueError, match="mx_betas"):
        a = list(_args(g))
        a[10] = g.betas.astype(np.float32)
        cbct_geom_mex("proj,dd", *a, x, g.map)
    with pytest.raises(ValueError, match="mx_image"):
        cbct_geom_mex("proj,dd", *_args(g), x[:-1], g.map)
    with pytest.raises(ValueError, match="mx_proj"):
        cbct_geom_mex("back,dd", *_args(g), x, g.map)
    with pytest.raises(ValueError, match="mx_map"):
        cbct_geom_mex("back,dd", *_args(g), np.zeros(g.sino_shape, np.float32), g.map.T)


def test_errors_are_reported_not_fatal():
    """Bad arguments come back as false/status codes with a message (the reference exit()s)."""
    L = _lib.load()
    g = _lib.CtsimGeom(0, 4, 4, 1, 1, 1, 0, 0, 0, 8, 8, 1, 1, 0, 0, 1000, 500, 1500, 1, 1)
    h = ctypes.c_void_p()
    b = np.zeros(1)
    c = np.zeros(1, np.float32)
    st = L.ctsim_plan_create(ctypes.byref(g), b.ctypes.data, c.ctypes.data, None, ctypes.byref(h))
    assert st == 1 and "positive" in _lib.last_error()
    st = L.ctsim_plan_create(None, None, None, None, ctypes.byref(h))
    assert st == 1
    ok = L.ctsim_cbct_geom(b"proj,xx", 4, 4, 4, 1, 1, 1, 0, 0, 0, 8, 8, 1, 1, 0, 0, 1000, 500, 1500, 1,
                           b.ctypes.data, c.ctypes.data, 1, c.ctypes.data, c.ctypes.data, None)
    assert not ok and "unknown geom type" in _lib.last_error()


def test_subset_selection_matches_reference_indexing():
    g = make_cases()["basic"]
    for M in (1, 2, 3, 4):
        for i in range(M + 2):
            s = g.subset(M, i)
            # MATLAB: betas(1+mod(i,M):M:end)
            want = g.betas[(1 + (i % M)) - 1::M] if M > 1 else g.betas
            assert np.array_equal(s.betas, want)
    y = np.arange(11 * 2 * 3).reshape(11, 2, 3)
    assert np.array_equal(ctsim_b200.orderedSubset(y, 4, 5), y[1::4])


def test_helical_geometry_follows_the_loader():
    """parameters/loadProjectionGeometryHelicalCT.m:26-57 restated by hand for a small scan."""
    from ctsim_b200.geometry import helical_geometry
    g = helical_geometry((8, 6, 4), (0.5, 0.5, 1.0), (0, 0, 0), (30, 10), (1.2, 2.0), (0, 0), 900.0, 600.0, 10, 2,
                         1.5, flatPanel=0)
    n = 10 * 2 + 1
    k = np.arange(1, n + 1) - (n + 1) / 2
    assert g.noViews == n and g.SDD == 1500.0 and g.shortScan
    assert np.allclose(g.betas, k * 2 * np.pi / 10 + np.pi)
    assert np.allclose(g.couchZ, k * (1.5 * 10 * 2.0 / 10), atol=1e-5)
    fov = 2 * np.sin(30 * 1.2 / 2 / 1500) * 900
    r = max(8, fov / 0.5) / 2
    xx = np.arange(8) - 3.5
    yy = np.arange(6) - 2.5
    assert np.array_equal(g.map, np.hypot(xx[None, :], yy[:, None]) < r)
