"""Reference-facing projector API.

Mirrors the reference's MATLAB/MEX interface for the cone-beam projector path:

* ``cbct_geom_mex(type, nxyz, dxyz, cxyz, nuv, duv, cuv, SAD, ADD, SDD, noViews,
  betas, couchZ, flatPanel, data, map)`` -- the MEX gateway
  (geom/cbct/cbct_geom_mex.c:253-326), host arrays in and out, through the C ABI;
* ``forwardProjectMex`` / ``backProjectMex`` -- the MATLAB shell
  (geom/shell/forwardProjectMex.m, geom/shell/backProjectMex.m) including the
  ordered-subset view selection ``1+mod(i,M):M:end`` and the ``M *`` scaling of
  subset backprojections;
* ``loadPojectors`` -- the closures of geom/shell/loadPojectors.m;
* ``Plan`` -- device-resident projector plan (torch CUDA tensors, no host copies).

Host numpy arrays go through the drop-in C entry points (one synchronous call,
like the MEX); torch CUDA tensors go through a cached device plan.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .geometry import CTGeometry

PROJ_TYPES = ("proj,dd", "proj,tf")


class _DTypeMap(dict):
    """torch dtype -> ctsim_dtype, built lazily (torch is optional for the host API)."""

    def _fill(self):
        if not self:
            import torch
            self.update({torch.float32: 0, torch.bfloat16: 1, torch.float16: 2})

    def __getitem__(self, k):
        self._fill()
        return dict.__getitem__(self, k)

    def __contains__(self, k):
        self._fill()
        return dict.__contains__(self, k)


_DTYPES = _DTypeMap()
BACK_TYPES = ("back,dd", "back,tf", "back,pd", "back,hpd", "back,var")


def _torch():
    import torch
    return torch


def _is_cuda_tensor(x) -> bool:
    try:
        torch = _torch()
    except ImportError:
        return False
    return isinstance(x, torch.Tensor) and x.is_cuda


# ---------------------------------------------------------------------------
# MEX gateway (host arrays)
# ---------------------------------------------------------------------------
def cbct_geom_mex(projType, nxyz, dxyz, cxyz, nuv, duv, cuv, SAD, ADD, SDD, noViews, betas, couchZ, flatPanel,
                  data, map=None):
    """Argument-for-argument mirror of the reference MEX ``cbct_geom_mex``.

    ``data`` is the image ``float32[nz, ny, nx]`` for ``proj,*`` and the sinogram
    ``float32[noViews, nu, nv]`` for ``back,*``; returns the sinogram or image.
    The shape/type checks and their messages follow
    geom/cbct/cbct_geom_mex.c:78-107 and :190-221.
    """
    if not isinstance(projType, str):
        raise ValueError("The 1st argument is invalid! ")
    if projType not in PROJ_TYPES + BACK_TYPES:
        raise ValueError("Error: unknown geom type. ")
    nx, ny, nz = (int(v) for v in np.asarray(nxyz).reshape(-1)[:3])
    nu, nv = (int(v) for v in np.asarray(nuv).reshape(-1)[:2])
    dx, dy, dz = (float(np.float32(v)) for v in np.asarray(dxyz).reshape(-1)[:3])
    ox, oy, oz = (float(np.float32(v)) for v in np.asarray(cxyz).reshape(-1)[:3])
    du, dv = (float(np.float32(v)) for v in np.asarray(duv).reshape(-1)[:2])
    ou, ov = (float(np.float32(v)) for v in np.asarray(cuv).reshape(-1)[:2])
    noViews = int(np.asarray(noViews).reshape(-1)[0])
    betas = np.asarray(betas)
    if betas.size != noViews or betas.dtype != np.float64:
        raise ValueError("Error: mx_betas must have noviews X 1 double array.")
    couchZ = np.asarray(couchZ)
    if couchZ.size != noViews or couchZ.dtype != np.float32:
        raise ValueError("Error: mx_couchz must have noviews X 1 double array.")
    if map is None:
        map = np.ones((ny, nx), dtype=bool)
    map = np.asarray(map)
    if map.shape != (ny, nx) or map.dtype != np.bool_:
        raise ValueError("Error: mx_map must have [nx ny] bool array.")
    data = np.asarray(data)
    if projType.startswith("proj"):
        if data.shape != (nz, ny, nx) or data.dtype != np.float32:
            raise ValueError("Error: mx_image must have [nx ny nz] float array.")
        out = np.empty((noViews, nu, nv), dtype=np.float32)
    else:
        if data.shape != (noViews, nu, nv) or data.dtype != np.float32:
            raise ValueError("Error: mx_proj must have [nv nu noviews] float array.")
        out = np.empty((nz, ny, nx), dtype=np.float32)
    L = _lib.load()
    data = np.ascontiguousarray(data)
    betas = np.ascontiguousarray(betas.reshape(-1))
    couchZ = np.ascontiguousarray(couchZ.reshape(-1))
    map = np.ascontiguousarray(map)
    ok = L.ctsim_cbct_geom(projType.encode(), nx, ny, nz, dx, dy, dz, ox, oy, oz, nu, nv, du, dv, ou, ov,
                           float(np.float32(SAD)), float(np.float32(ADD)), float(np.float32(SDD)), noViews,
                           betas.ctypes.data, couchZ.ctypes.data, int(flatPanel), data.ctypes.data, out.ctypes.data,
                           map.ctypes.data)
    if not ok:
        raise _lib.CtsimError("Error: cbct_geom_mex() failed. " + _lib.last_error())
    return out


def _mex_call(projType, geom: CTGeometry, data):
    return cbct_geom_mex(projType, geom.reconSize, geom.reconSpacing, geom.reconOffset, geom.detSize,
                         geom.detSpacing, geom.detOffset, geom.SAD, geom.ADD, geom.SDD, geom.noViews, geom.betas,
                         geom.couchZ, geom.flatPanel, data, geom.map)


# ---------------------------------------------------------------------------
# Device plans
# ---------------------------------------------------------------------------
def _tuning_dict(t) -> dict:
    return {"proj_groups": t.proj_groups, "proj_rows": t.proj_rows, "proj_layout": t.proj_layout,
            "proj_slots": t.proj_slots, "back_mz": t.back_mz, "back_mz_tf": t.back_mz_tf, "pd_mz": t.pd_mz}


class Plan:
    """Device-resident projector plan for one geometry (all of its views).

    Holds the per-view tables and scratch on one GPU; ``project``/``backproject``
    take and return torch CUDA tensors and run on the current torch stream.
    With ``stream`` (a torch.cuda.Stream) the plan is stream-ordered: its memory is
    allocated and freed on that stream from the library pool, without a device-wide
    synchronisation (ctsim_plan_create_async); all work on it must then be ordered
    on that stream.
    """

    def __init__(self, geom: CTGeometry, device=None, stream=None):
        torch = _torch()
        self.geom = geom
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else
                                   torch.device(device).index or 0)
        L = _lib.load()
        g = _lib.CtsimGeom(*geom.scalars()[:18], geom.noViews, int(geom.flatPanel))
        self._betas = np.ascontiguousarray(geom.betas, dtype=np.float64)
        self._couch = np.ascontiguousarray(geom.couchZ, dtype=np.float32)
        self._map = np.ascontiguousarray(geom.map, dtype=np.bool_)
        h = C.c_void_p()
        self.stream = stream
        with torch.cuda.device(self.device):
            if stream is None:
                _lib.check(L.ctsim_plan_create(C.byref(g), self._betas.ctypes.data, self._couch.ctypes.data,
                                               self._map.ctypes.data, C.byref(h)), "ctsim_plan_create")
            else:
                _lib.check(L.ctsim_plan_create_async(C.byref(g), self._betas.ctypes.data, self._couch.ctypes.data,
                                                     self._map.ctypes.data, stream.cuda_stream, C.byref(h)),
                           "ctsim_plan_create_async")
        self._h = h
        self._L = L

    @property
    def tuning(self) -> dict:
        """Launch shapes: forward candidate groups, A^T and FDK z-pass depths."""
        t = _lib.CtsimTuning()
        _lib.check(self._L.ctsim_plan_get_tuning(self._h, C.byref(t)), "ctsim_plan_get_tuning")
        return _tuning_dict(t)

    def set_tuning(self, proj_groups: int = 0, back_mz: int = 0, pd_mz: int = 0, back_mz_tf: int = 0,
                   proj_rows: int = 0, proj_layout: int = 0, proj_slots: int = 0):
        t = _lib.CtsimTuning(int(proj_groups), int(back_mz), int(pd_mz), int(back_mz_tf), int(proj_rows),
                             int(proj_layout), int(proj_slots))
        _lib.check(self._L.ctsim_plan_set_tuning(self._h, C.byref(t)), "ctsim_plan_set_tuning")

    def autotune(self, method: str, sample_views: int = 0) -> dict:
        """Time every valid launch shape of ``method`` on a sample of views and keep the
        fastest (recorded per shape class for the process); synchronises the stream."""
        torch = _torch()
        m = {"proj,dd": 0, "proj,tf": 1, "back,dd": 2, "back,tf": 3, "back,pd": 4, "back,hpd": 5,
             "back,var": 6}[method]
        t = _lib.CtsimTuning()
        st = torch.cuda.current_stream(self.device).cuda_stream
        with torch.cuda.device(self.device):
            _lib.check(self._L.ctsim_plan_autotune(self._h, m, int(sample_views), st, C.byref(t)),
                       "ctsim_plan_autotune")
        return _tuning_dict(t)

    @property
    def device_bytes(self) -> int:
        return int(self._L.ctsim_plan_device_bytes(self._h))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.ctsim_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _views(self, view_begin, view_stride, view_count):
        if view_count is None:
            view_count = len(range(view_begin, self.geom.noViews, view_stride))
        return int(view_begin), int(view_stride), int(view_count)

    def _check_tensor(self, t, shape, name):
        torch = _torch()
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype in _DTYPES):
            raise TypeError(f"{name} must be a float32, bfloat16 or float16 CUDA tensor")
        if t.device != self.device:
            raise ValueError(f"{name} is on {t.device}, the plan on {self.device}")
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")
        return t.contiguous()

    def project(self, image, method: str = "dd", view_begin: int = 0, view_stride: int = 1, view_count=None,
                out=None, out_dtype=None):
        """A x for the selected views -> [view_count, nu, nv] of ``out_dtype`` (default: the
        image's storage type; float32, bfloat16 or float16, FP32 accumulation)."""
        torch = _torch()
        vb, vs, vc = self._views(view_begin, view_stride, view_count)
        image = self._check_tensor(image, self.geom.image_shape, "image")
        if out is None:
            out = torch.empty((vc, self.geom.nu, self.geom.nv), dtype=out_dtype or image.dtype, device=self.device)
        else:
            out = self._check_tensor(out, (vc, self.geom.nu, self.geom.nv), "out")
        m = {"dd": 0, "tf": 1, "proj,dd": 0, "proj,tf": 1}[method]
        st = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._L.ctsim_plan_project_ex(self._h, m, image.data_ptr(), _DTYPES[image.dtype], out.data_ptr(),
                                                 _DTYPES[out.dtype], vb, vs, vc, st), "ctsim_plan_project")
        return out

    def backproject(self, sino, method: str = "dd", view_begin: int = 0, view_stride: int = 1, view_count=None,
                    scale: float = 1.0, out=None, out_dtype=None, scaled: bool = False):
        """scale * A^T y (or the FDK pd/hpd, or the variance backprojection) -> [nz, ny, nx] of ``out_dtype``
        (default: the sinogram's storage type).  ``scaled``: the FP32 sinogram is already
        multiplied by the plan's axial amplitudes (CTSIM_INPUT_SCALED, dd/tf)."""
        torch = _torch()
        vb, vs, vc = self._views(view_begin, view_stride, view_count)
        sino = self._check_tensor(sino, (vc, self.geom.nu, self.geom.nv), "sino")
        if out is None:
            out = torch.empty(self.geom.image_shape, dtype=out_dtype or sino.dtype, device=self.device)
        else:
            out = self._check_tensor(out, self.geom.image_shape, "out")
        m = {"dd": 2, "tf": 3, "pd": 4, "hpd": 5, "var": 6, "back,dd": 2, "back,tf": 3, "back,pd": 4, "back,hpd": 5,
             "back,var": 6}[method] | (_lib.INPUT_SCALED if scaled else 0)
        st = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._L.ctsim_plan_backproject_ex(self._h, m, sino.data_ptr(), _DTYPES[sino.dtype],
                                                     out.data_ptr(), _DTYPES[out.dtype], vb, vs, vc, float(scale),
                                                     st), "ctsim_plan_backproject")
        return out

    def check(self):
        """Synchronise and raise if a kernel flagged an oversized footprint."""
        _lib.check(self._L.ctsim_plan_check(self._h), "ctsim_plan_check")


def plan_for(geom: CTGeometry, device=None) -> Plan:
    """Cached device plan of a geometry (one per device)."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else torch.device(device).index or 0)
    cache = geom.__dict__.setdefault("_plans", {})
    p = cache.get(dev)
    if p is None:
        p = Plan(geom, dev)
        cache[dev] = p
    return p


# ---------------------------------------------------------------------------
# MATLAB shell mirrors
# ---------------------------------------------------------------------------
def _subset(geom: CTGeometry, M: int, i: int):
    """Views 1+mod(i,M):M:end (1-based) == start mod(i,M), stride M (0-based)."""
    if M == 1:
        return 0, 1, geom.noViews
    start = i % M
    return start, M, len(range(start, geom.noViews, M))


def forwardProjectMex(img, geom: CTGeometry, M: int = 1, i: int = 0, projType: str = "proj,dd", map=None):
    """geom/shell/forwardProjectMex.m: forward projection of subset i of M."""
    if projType not in PROJ_TYPES:
        raise ValueError("Error: unknown geom type. ")
    if map is not None:
        geom = _with_map(geom, map)
    if _is_cuda_tensor(img):
        vb, vs, vc = _subset(geom, M, i)
        return plan_for(geom, img.device).project(img, projType, vb, vs, vc)
    g = geom.subset(M, i)
    return _mex_call(projType, g, np.asarray(img, dtype=np.float32))


def backProjectMex(sino, geom: CTGeometry, M: int = 1, i: int = 0, projType: str = "back,dd", map=None):
    """geom/shell/backProjectMex.m: backprojection of subset i of M, scaled by M when M != 1."""
    if projType not in BACK_TYPES:
        raise ValueError("Error: unknown geom type. ")
    if map is not None:
        geom = _with_map(geom, map)
    if _is_cuda_tensor(sino):
        vb, vs, vc = _subset(geom, M, i)
        return plan_for(geom, sino.device).backproject(sino, projType, vb, vs, vc, scale=float(M))
    g = geom.subset(M, i)
    img = _mex_call(projType, g, np.asarray(sino, dtype=np.float32))
    if M != 1:
        img = img * np.float32(M)
    return img


def _with_map(geom: CTGeometry, map):
    from dataclasses import replace
    return replace(geom, map=np.asarray(map, dtype=bool))


def orderedSubset(x, M: int, isub: int):
    """penalty/orderedSubset.m: views 1+mod(isub,M):M:end of a sinogram [views, nu, nv]."""
    if M == 1:
        return x
    return x[isub % M::M]


def loadPojectors(geom: CTGeometry, numos: int = 1):
    """geom/shell/loadPojectors.m: the separable-footprint (tf) closures used by PWLS."""
    Aos = lambda x, isub: forwardProjectMex(x, geom, numos, isub, "proj,tf")
    Atos = lambda y, isub: backProjectMex(y, geom, numos, isub, "back,tf")
    A = lambda x: forwardProjectMex(x, geom, 1, 0, "proj,tf")
    At = lambda y: backProjectMex(y, geom, 1, 0, "back,tf")
    Os = lambda x, isub: orderedSubset(x, numos, isub)
    return A, At, Aos, Atos, Os


def _batch(fn_name, method_id, entries):
    """entries: (plan, in_tensor, out_tensor, view_begin, view_stride, view_count, scale)."""
    torch = _torch()
    L = _lib.load()
    n = len(entries)
    if n == 0:
        return
    arr = (_lib.CtsimBatchItem * n)()
    keep = []
    for k, (plan, x, y, vb, vs, vc, scale) in enumerate(entries):
        for t in (x, y):
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype in _DTYPES and t.is_contiguous()):
                raise TypeError("batched launches take contiguous float32, bfloat16 or float16 CUDA tensors")
        arr[k] = _lib.CtsimBatchItem(plan._h, x.data_ptr(), y.data_ptr(), int(vb), int(vs), int(vc), float(scale),
                                     _DTYPES[x.dtype], _DTYPES[y.dtype])
        keep.append(plan)
    st = torch.cuda.current_stream(entries[0][0].device).cuda_stream
    _lib.check(getattr(L, fn_name)(method_id, arr, n, st), fn_name)


def batch_project(method: str, entries):
    """A of many plans in one persistent launch per launch-shape class: entries are
    (plan, image, out_sino, view_begin, view_stride, view_count) (ctsim_batch_project)."""
    _batch("ctsim_batch_project", {"dd": 0, "tf": 1}[method], [e + (1.0,) if len(e) == 6 else e for e in entries])


def batch_backproject(method: str, entries, scaled: bool = False):
    """scale * A^T of many plans: entries are (plan, sino, out_image, view_begin,
    view_stride, view_count, scale) (ctsim_batch_backproject); ``scaled`` as in
    Plan.backproject."""
    _batch("ctsim_batch_backproject", {"dd": 2, "tf": 3}[method] | (_lib.INPUT_SCALED if scaled else 0), entries)
