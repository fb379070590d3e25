"""ctypes bindings to the oracle libraries (TEST INFRASTRUCTURE ONLY).

* ``oracle_cbct``  -> this project's CPU restatement, ``_build/libcbct_oracle.so``
* ``ref_cbct``     -> the reference's own geom/cbct C, ``_ref/libcbct_ref.so``
                      (single-threaded, or over view chunks with ``nthreads``)
* ``ref3_cbct``    -> the reference's arc-detector DD pair (geom/cbct/cbct_proj3.c,
                      cbct_back3.c), ``_ref/libcbct_ref3.so``
* ``refgpu_cbct``  -> the reference's CUDA DD pair (geom/dd_cuda), SF pair (geom/sf_cuda) and
                      FDK backprojection (geom/fdk_cuda), ``_ref/librefgpu_{dd,sf,pd}.so``:
                      timing baselines on the GPU, not parity targets

Both take and return numpy arrays in the package conventions
(image ``[nz, ny, nx]``, sino ``[noViews, nu, nv]``, float32).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libcbct_oracle.so")
ORACLE64_SO = os.path.join(HERE, "_build", "libcbct_oracle64.so")
REF_SO = os.path.join(HERE, "_ref", "libcbct_ref.so")
REF3_SO = os.path.join(HERE, "_ref", "libcbct_ref3.so")
REFGPU_SO = os.path.join(HERE, "_ref", "librefgpu_dd.so")
REFGPU_PD_SO = os.path.join(HERE, "_ref", "librefgpu_pd.so")
REFGPU_SF_SO = os.path.join(HERE, "_ref", "librefgpu_sf.so")

KINDS = {"proj,dd": 0, "proj,tf": 1, "back,dd": 2, "back,tf": 3,
         "back,pd": 4, "back,hpd": 5, "back,var": 6}

_f = C.c_float
_i = C.c_int
_p = C.c_void_p
_GEOM_ARGS = [_i, _i, _i, _f, _f, _f, _f, _f, _f, _i, _i, _f, _f, _f, _f, _f, _f, _f, _i, _p, _p, _i, _p, _p, _p]

_libs = {}


def build():
    """Build the oracle libraries (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load(path):
    if path not in _libs:
        if not os.path.exists(path):
            build()
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        if path in (ORACLE_SO, ORACLE64_SO):
            lib.orc_proj.argtypes = [_i] + _GEOM_ARGS
            lib.orc_back.argtypes = [_i] + _GEOM_ARGS
            lib.orc_back_pd.argtypes = _GEOM_ARGS + [_i]
            lib.orc_back_var.argtypes = _GEOM_ARGS
            for fn in (lib.orc_proj, lib.orc_back, lib.orc_back_pd, lib.orc_back_var):
                fn.restype = _i
        elif path == REF3_SO:
            lib.ref3_cbct_call.argtypes = [_i] + _GEOM_ARGS
            lib.ref3_cbct_call.restype = _i
        elif path == REFGPU_SO:
            for fn in (lib.refgpu_proj_dd, lib.refgpu_back_dd):
                fn.argtypes = _GEOM_ARGS
                fn.restype = C.c_bool
        elif path == REFGPU_PD_SO:
            lib.refgpu_back_pd.argtypes = _GEOM_ARGS + [C.c_bool]
            lib.refgpu_back_pd.restype = C.c_bool
        elif path == REFGPU_SF_SO:
            for fn in (lib.refgpu_proj_tf, lib.refgpu_back_tf):
                fn.argtypes = _GEOM_ARGS
                fn.restype = C.c_bool
        else:
            lib.ref_cbct_call.argtypes = [_i] + _GEOM_ARGS
            lib.ref_cbct_call.restype = _i
            lib.ref_cbct_call_mt.argtypes = [_i, _i] + _GEOM_ARGS
            lib.ref_cbct_call_mt.restype = _i
        _libs[path] = lib
    return _libs[path]


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _prep(kind, geom, data, dtype=np.float32):
    if kind not in KINDS:
        raise ValueError(f"unknown geom type {kind!r}")
    data = np.ascontiguousarray(data, dtype=dtype)
    if kind.startswith("proj"):
        if data.shape != geom.image_shape:
            raise ValueError("image must have shape (nz, ny, nx)")
        out = np.zeros(geom.sino_shape, dtype=dtype)
    else:
        if data.shape != geom.sino_shape:
            raise ValueError("sinogram must have shape (noViews, nu, nv)")
        out = np.zeros(geom.image_shape, dtype=dtype)
    betas = np.ascontiguousarray(geom.betas, dtype=np.float64)
    couch = np.ascontiguousarray(geom.couchZ, dtype=np.float32)
    mp = np.ascontiguousarray(geom.map, dtype=np.bool_)
    tail = (betas.ctypes.data, couch.ctypes.data, int(geom.flatPanel), data.ctypes.data, out.ctypes.data,
            mp.ctypes.data)
    keep = (data, betas, couch, mp)
    return data, out, tuple(geom.scalars()) + tail, keep


def oracle_cbct(kind: str, geom, data, fp64: bool = False) -> np.ndarray:
    """Run this project's CPU restatement of one reference projector (bit-exact FP32), or
    with ``fp64`` the same control flow in double (float64 arrays in and out)."""
    lib = _load(ORACLE64_SO if fp64 else ORACLE_SO)
    data, out, args, keep = _prep(kind, geom, data, np.float64 if fp64 else np.float32)
    if kind.startswith("proj"):
        ok = lib.orc_proj(KINDS[kind], *args)
    elif kind in ("back,dd", "back,tf"):
        ok = lib.orc_back(KINDS[kind] - 2, *args)
    elif kind in ("back,pd", "back,hpd"):
        ok = lib.orc_back_pd(*args, 1 if kind == "back,pd" else 0)
    elif kind == "back,var":
        ok = lib.orc_back_var(*args)
    else:
        raise NotImplementedError(kind)
    if not ok:
        raise RuntimeError("oracle call failed")
    return out


def oracle_cbct_mt(kind: str, geom, data, nthreads: int = 0) -> np.ndarray:
    """``oracle_cbct`` over contiguous view chunks in host threads (ctypes releases the
    GIL), like the reference harness ``ref_cbct_call_mt`` (oracle/ref_shim.c): forward
    projections fill disjoint view slices, backprojections fill one image per chunk and
    the images are summed in chunk order (so only the view-sum order differs from the
    single-thread oracle)."""
    from concurrent.futures import ThreadPoolExecutor
    from dataclasses import replace

    if nthreads < 1:
        nthreads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    n = geom.noViews
    chunks = max(1, min(nthreads, n))
    bounds = [n * c // chunks for c in range(chunks + 1)]
    data = np.ascontiguousarray(data, dtype=np.float32)

    def part(c):
        b, e = bounds[c], bounds[c + 1]
        g = replace(geom, betas=np.ascontiguousarray(geom.betas[b:e]), couchZ=np.ascontiguousarray(geom.couchZ[b:e]))
        return oracle_cbct(kind, g, data if kind.startswith("proj") else data[b:e])

    with ThreadPoolExecutor(chunks) as ex:
        parts = list(ex.map(part, range(chunks)))
    if kind.startswith("proj"):
        return np.concatenate(parts, axis=0)
    out = np.zeros(geom.image_shape, np.float32)
    for p in parts:
        out += p
    return out


def ref_cbct(kind: str, geom, data, nthreads: int = 1) -> np.ndarray:
    """Run the reference's own compiled geom/cbct projector (needs _ref/libcbct_ref.so)."""
    lib = _load(REF_SO)
    data, out, args, keep = _prep(kind, geom, data)
    if nthreads <= 1:
        ok = lib.ref_cbct_call(KINDS[kind], *args)
    else:
        ok = lib.ref_cbct_call_mt(int(nthreads), KINDS[kind], *args)
    if not ok:
        raise RuntimeError("reference call failed")
    return out


def ref3_cbct(kind: str, geom, data) -> np.ndarray:
    """The reference's arc-detector variants of proj,dd / back,dd (needs _ref/libcbct_ref3.so)."""
    if kind not in ("proj,dd", "back,dd"):
        raise ValueError("the reference's arc-detector code covers proj,dd and back,dd")
    lib = _load(REF3_SO)
    data, out, args, keep = _prep(kind, geom, data)
    if not lib.ref3_cbct_call(KINDS[kind], *args):
        raise RuntimeError("reference call failed")
    return out


def refgpu_available() -> bool:
    return os.path.exists(REFGPU_SO)


def refgpu_cbct(kind: str, geom, data) -> np.ndarray:
    """The reference's own GPU drivers cbct_proj_dd_gpu / cbct_back_dd_gpu
    (geom/dd_cuda/cbct_dd_proj.c:407, cbct_dd_back.c:299), cbct_proj_tf_gpu /
    cbct_back_tf_gpu (geom/sf_cuda/cbct_sf_proj.c:443, cbct_sf_back.c:334) and
    cbct_back_pd_gpu (geom/fdk_cuda/cbct_back_pd.c:230) on the current CUDA device:
    host arrays in and out, synchronous."""
    if kind not in ("proj,dd", "back,dd", "proj,tf", "back,tf", "back,pd", "back,hpd"):
        raise ValueError("the reference GPU builds cover proj,dd, back,dd, proj,tf, back,tf, back,pd and back,hpd")
    data, out, args, keep = _prep(kind, geom, data)
    a = list(args)
    if not kind.startswith("proj"):  # the back drivers take (image, proj): the output image first
        a[-3], a[-2] = a[-2], a[-3]
    if kind == "proj,dd":
        ok = _load(REFGPU_SO).refgpu_proj_dd(*a)
    elif kind == "back,dd":
        ok = _load(REFGPU_SO).refgpu_back_dd(*a)
    elif kind == "proj,tf":
        ok = _load(REFGPU_SF_SO).refgpu_proj_tf(*a)
    elif kind == "back,tf":
        ok = _load(REFGPU_SF_SO).refgpu_back_tf(*a)
    else:
        ok = _load(REFGPU_PD_SO).refgpu_back_pd(*a, kind == "back,pd")
    if not ok:
        raise RuntimeError("reference GPU call failed")
    return out


FBCT_ORACLE_SO = os.path.join(HERE, "_build", "libfbct_oracle.so")
FBCT_REF_SO = os.path.join(HERE, "_ref", "libfbct_ref.so")
FAN_KINDS = {"proj,dd": 0, "proj,tf": 1, "back,dd": 2, "back,tf": 3}
_FAN_ARGS = [_i, _i, _f, _f, _f, _f, _i, _f, _f, _f, _f, _f, _i, _p, _i, _p, _p]


def _fan_call(path, fn_name, kind, geom, data):
    if kind not in FAN_KINDS:
        raise ValueError(f"unknown fan-beam geom type {kind!r}")
    if path not in _libs:
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        for n in ("fbo_proj", "fbo_back", "ref_fbct_call"):
            if hasattr(lib, n):
                getattr(lib, n).argtypes = [_i] + _FAN_ARGS
                getattr(lib, n).restype = _i
        _libs[path] = lib
    lib = _libs[path]
    data = np.ascontiguousarray(data, dtype=np.float32)
    proj = kind.startswith("proj")
    if data.shape != (geom.image_shape if proj else geom.sino_shape):
        raise ValueError("data has the wrong shape")
    out = np.zeros(geom.sino_shape if proj else geom.image_shape, dtype=np.float32)
    betas = np.ascontiguousarray(geom.betas, dtype=np.float64)
    args = tuple(geom.scalars()) + (betas.ctypes.data, int(geom.flatPanel), data.ctypes.data, out.ctypes.data)
    k = FAN_KINDS[kind]
    if fn_name == "ref_fbct_call":
        ok = lib.ref_fbct_call(k, *args)
    else:
        ok = (lib.fbo_proj if proj else lib.fbo_back)(k & 1, *args)
    if not ok:
        raise RuntimeError("fan-beam call failed")
    return out


def oracle_fbct(kind: str, geom, data) -> np.ndarray:
    """This project's restatement of the geom/fbct DD/SF pair (bit-exact FP32)."""
    return _fan_call(FBCT_ORACLE_SO, "fbo", kind, geom, data)


def ref_fbct(kind: str, geom, data) -> np.ndarray:
    """The reference's own geom/fbct C (needs _ref/libfbct_ref.so)."""
    return _fan_call(FBCT_REF_SO, "ref_fbct_call", kind, geom, data)
