"""The MEX gateways (ctsim_b200/mex/: cone beam and 2-D fan beam), linked and called.

MATLAB is not available here, so each gateway is compiled with a test-side
implementation of the mx* functions it uses (tests/mex_stub/mex_fake.c: arrays with a
class, dimensions and data; mexErrMsgTxt jumps back to the caller) into a shared
library linked against libctsim_b200.so, and its mexFunction is called through
ctypes with the 16 (cone beam) or 14 (fan beam) MATLAB arguments:

* on the CPU: the usage text of a call with no arguments (the reference prints its
  help, geom/cbct/cbct_geom_mex.c:317-320) and the argument checks with the
  reference's messages (geom/cbct/cbct_geom_mex.c:78-107, :190-221);
* on the GPU: every geometry type through mexFunction against the reference's own
  outputs (the golden fixtures), in MATLAB's array layouts.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from cases import FAN_KINDS, KINDS, make_cases, make_fan_cases

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")
STUB = os.path.join(ROOT, "tests", "mex_stub")
LIBDIR = os.path.join(ROOT, "ctsim_b200", "_lib")
DOUBLE, SINGLE, INT32, LOGICAL, CHAR = 0, 1, 2, 3, 4
REL_L2 = 1e-5


@pytest.mark.parametrize("name", ["cbct_geom_mex_b200.c", "fbct_geom_mex_b200.c"])
def test_mex_gateway_compiles(name):
    src = os.path.join(ROOT, "ctsim_b200", "mex", name)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", STUB,
                        "-I", os.path.join(ROOT, "include"), src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_header_is_plain_c():
    hdr = os.path.join(ROOT, "include", "ctsim_b200.h")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-x", "c", hdr],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


class Gateway:
    """One gateway linked with the fake MEX API; call() runs its mexFunction."""

    def __init__(self, path):
        L = C.CDLL(path)
        L.fake_array.restype = C.c_void_p
        L.fake_array.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_size_t), C.c_void_p]
        L.fake_data.restype = C.c_void_p
        L.fake_data.argtypes = [C.c_void_p]
        L.fake_numel.restype = C.c_size_t
        L.fake_numel.argtypes = [C.c_void_p]
        L.fake_free.argtypes = [C.c_void_p]
        L.fake_error.restype = C.c_char_p
        L.fake_output.restype = C.c_char_p
        L.fake_call.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]
        self.L = L

    def array(self, cls, dims, data=None):
        d = (C.c_size_t * len(dims))(*dims)
        buf = None
        if data is not None:
            data = np.ascontiguousarray(data)
            buf = data.ctypes.data
        return self.L.fake_array(cls, len(dims), d, buf)

    def string(self, s):
        b = s.encode()
        return self.array(CHAR, (1, len(b)), np.frombuffer(b, np.uint8))

    def call(self, args, nlhs=1):
        prhs = (C.c_void_p * max(1, len(args)))(*args)
        plhs = (C.c_void_p * 1)()
        rc = self.L.fake_call(nlhs, plhs, len(args), prhs)
        for a in args:
            self.L.fake_free(a)
        return rc, plhs[0], self.L.fake_error().decode(), self.L.fake_output().decode()

    def result(self, arr, shape):
        n = self.L.fake_numel(arr)
        out = np.ctypeslib.as_array(C.cast(self.L.fake_data(arr), C.POINTER(C.c_float)), shape=(n,)).copy()
        self.L.fake_free(arr)
        return out.reshape(shape)


@pytest.fixture(scope="module")
def gateways(tmp_path_factory):
    from ctsim_b200 import _lib
    _lib.load()  # builds libctsim_b200.so if it is missing
    out = {}
    d = tmp_path_factory.mktemp("mex")
    for name in ("cbct", "fbct"):
        so = str(d / f"{name}_mex_test.so")
        cmd = ["gcc", "-std=c99", "-O1", "-shared", "-fPIC", "-I", STUB, "-I", os.path.join(ROOT, "include"),
               os.path.join(ROOT, "ctsim_b200", "mex", f"{name}_geom_mex_b200.c"), os.path.join(STUB, "mex_fake.c"),
               "-L", LIBDIR, "-lctsim_b200", f"-Wl,-rpath,{LIBDIR}", "-o", so]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        out[name] = Gateway(so)
    return out


def cbct_args(gw, kind, g, data, betas=None, map_=None):
    """The 16 MATLAB arguments of the cone-beam gateway; data in the repository's C-order
    layouts (image [nz][ny][nx] = MATLAB [nx ny nz], sinogram [views][nu][nv] = [nv nu views])."""
    betas = g.betas if betas is None else betas
    map_ = g.map if map_ is None else map_
    f32 = lambda v: np.asarray(v, np.float32)
    dims = np.shape(data)[::-1]  # MATLAB's column-major dimensions of the C-order array
    return [gw.string(kind),
            gw.array(INT32, (1, 3), np.array(g.reconSize, np.int32)),
            gw.array(SINGLE, (1, 3), f32(g.reconSpacing)), gw.array(SINGLE, (1, 3), f32(g.reconOffset)),
            gw.array(INT32, (1, 2), np.array(g.detSize, np.int32)),
            gw.array(SINGLE, (1, 2), f32(g.detSpacing)), gw.array(SINGLE, (1, 2), f32(g.detOffset)),
            gw.array(SINGLE, (1, 1), f32([g.SAD])), gw.array(SINGLE, (1, 1), f32([g.ADD])),
            gw.array(SINGLE, (1, 1), f32([g.SDD])), gw.array(INT32, (1, 1), np.array([g.noViews], np.int32)),
            gw.array(DOUBLE, (len(betas), 1), np.asarray(betas, np.float64)),
            gw.array(SINGLE, (g.noViews, 1), f32(g.couchZ)),
            gw.array(INT32, (1, 1), np.array([g.flatPanel], np.int32)),
            gw.array(SINGLE, dims, f32(data)),
            gw.array(LOGICAL, map_.shape[::-1], np.asarray(map_, np.uint8))]


def test_cbct_gateway_usage_without_arguments(gateways):
    rc, _, err, out = gateways["cbct"].call([], nlhs=0)
    assert rc == 0 and err == ""
    assert "cbct_geom_mex_b200(type" in out and "back,var" in out


def test_fbct_gateway_usage_without_arguments(gateways):
    rc, _, err, out = gateways["fbct"].call([], nlhs=0)
    assert rc == 0 and "fbct_geom_mex_b200(type" in out


def test_cbct_gateway_argument_checks(gateways):
    gw = gateways["cbct"]
    g = make_cases()["basic"]
    x = np.zeros(g.image_shape, np.float32)
    cases = []
    a = cbct_args(gw, "proj,dd", g, x)
    gw.L.fake_free(a[0])
    a[0] = gw.array(DOUBLE, (1, 1), np.array([1.0]))
    cases.append((a, "The 1st argument is invalid!"))
    cases.append((cbct_args(gw, "proj,rd", g, x), "Error: unknown geom type."))
    cases.append((cbct_args(gw, "proj,dd", g, x, betas=g.betas[:-1]), "mx_betas must have noviews X 1 double"))
    cases.append((cbct_args(gw, "proj,dd", g, x, map_=g.map[:-1]), "mx_map must have [nx ny] bool array"))
    cases.append((cbct_args(gw, "proj,dd", g, x[:-1]), "mx_image must have [nx ny nz] float array"))
    y = np.zeros(g.sino_shape, np.float32)
    cases.append((cbct_args(gw, "back,dd", g, y[:-1]), "mx_proj must have [nv nu noviews] float array"))
    a = cbct_args(gw, "proj,dd", g, x)
    gw.L.fake_free(a.pop())
    cases.append((a, "The 1st argument is invalid!"))  # 15 arguments
    for args, msg in cases:
        rc, _, err, _ = gw.call(args)
        assert rc == 1 and msg in err, (msg, err)


def test_cbct_gateway_reports_a_failed_projection(gateways):
    """A call the checks accept but the library refuses ends in the reference's error
    message (geom/cbct/cbct_geom_mex.c:322-323), with the library's reason printed first:
    an axial footprint wider than 10 detector rows on a GPU, the missing device here."""
    import torch
    from ctsim_b200 import CTGeometry, circular_betas
    gw = gateways["cbct"]
    g = CTGeometry((16, 16, 8), (1.0, 1.0, 20.0), (0, 0, 0), (32, 16), (1.0, 1.0), (0, 0), 1000.0, 500.0, 1500.0,
                   circular_betas(4))
    rc, _, err, out = gw.call(cbct_args(gw, "proj,dd", g, np.ones(g.image_shape, np.float32)))
    assert rc == 1 and "cbct_geom_mex() failed" in err
    assert ("10 detector rows" if torch.cuda.is_available() else "no CUDA device") in out


def fbct_args(gw, kind, g, data, betas=None):
    betas = g.betas if betas is None else betas
    f32 = lambda v: np.asarray(v, np.float32)
    dims = np.shape(data)[::-1]
    return [gw.string(kind), gw.array(INT32, (1, 2), np.array(g.reconSize, np.int32)),
            gw.array(SINGLE, (1, 2), f32(g.reconSpacing)), gw.array(SINGLE, (1, 2), f32(g.reconOffset)),
            gw.array(INT32, (1, 1), np.array([g.nu], np.int32)), gw.array(SINGLE, (1, 1), f32([g.du])),
            gw.array(SINGLE, (1, 1), f32([g.detOffset])), gw.array(SINGLE, (1, 1), f32([g.SAD])),
            gw.array(SINGLE, (1, 1), f32([g.ADD])), gw.array(SINGLE, (1, 1), f32([g.SDD])),
            gw.array(INT32, (1, 1), np.array([g.noViews], np.int32)),
            gw.array(DOUBLE, (len(betas), 1), np.asarray(betas, np.float64)),
            gw.array(INT32, (1, 1), np.array([g.flatPanel], np.int32)), gw.array(SINGLE, dims, f32(data))]


def test_fbct_gateway_argument_checks(gateways):
    gw = gateways["fbct"]
    g = make_fan_cases()["fan_basic"]
    x = np.zeros(g.image_shape, np.float32)
    for args, msg in ((fbct_args(gw, "proj,rd", g, x), "unknown geom type"),
                      (fbct_args(gw, "proj,dd", g, x, betas=g.betas[:-1]), "mx_betas must have noviews X 1"),
                      (fbct_args(gw, "proj,dd", g, x[:-1]), "mx_image must have [nx ny] float array"),
                      (fbct_args(gw, "proj,dd", g, x)[:13], "incorrect number of arguments")):
        rc, _, err, _ = gw.call(args)
        assert rc == 1 and msg in err, (msg, err)


def _rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["basic", "offsets_curved", "couch_map", "ragged"])
def test_cbct_gateway_matches_reference_outputs(gateways, name):
    gw = gateways["cbct"]
    g = make_cases()[name]
    d = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    for k in KINDS:
        src = d["image_in"] if k.startswith("proj") else d["sino_in"]
        rc, arr, err, out = gw.call(cbct_args(gw, k, g, src))
        assert rc == 0, (k, err, out)
        shape = g.sino_shape if k.startswith("proj") else g.image_shape
        got = gw.result(arr, shape)
        ref = d[k.replace(",", "_")]
        assert _rel_l2(got, ref) <= REL_L2, f"{name} {k}: rel L2 {_rel_l2(got, ref):.2e}"
        if k in ("back,pd", "back,hpd", "back,var") and g.flatPanel == 1:
            assert np.array_equal(got, ref), f"{name} {k}: not bit-identical"


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(make_fan_cases()))
def test_fbct_gateway_matches_reference_outputs(gateways, name):
    gw = gateways["fbct"]
    g = make_fan_cases()[name]
    d = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    for k in FAN_KINDS:
        src = d["image_in"] if k.startswith("proj") else d["sino_in"]
        rc, arr, err, out = gw.call(fbct_args(gw, k, g, src))
        assert rc == 0, (k, err, out)
        shape = (g.noViews, g.nu) if k.startswith("proj") else g.image_shape
        got = gw.result(arr, shape)
        ref = d[k.replace(",", "_")]
        assert _rel_l2(got, ref) <= REL_L2, f"{name} {k}: rel L2 {_rel_l2(got, ref):.2e}"
