"""2-D fan-beam projectors on the device (geom/fbct): the distance-driven and
separable-footprint pair behind the reference's fbct_geom_mex.

* ``fbct_geom_mex(projType, nxy, dxy, cxy, nu, du, cu, SAD, ADD, SDD, noViews, betas, flatPanel, data)``
      the MEX call (geom/fbct/fbct_geom_mex.c:225-278) for "proj,dd", "proj,tf", "back,dd",
      "back,tf": numpy in, numpy out (image [ny, nx], sinogram [noViews, nu]).
* ``FanPlan(geom)``  device plan of a FanGeometry; ``project``/``backproject`` take torch CUDA
      tensors, with ordered-subset view selection like the cone-beam Plan.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .geometry import FanGeometry

FAN_TYPES = ("proj,dd", "proj,tf", "back,dd", "back,tf")


def fbct_geom_mex(projType, nxy, dxy, cxy, nu, du, cu, SAD, ADD, SDD, noViews, betas, flatPanel, data):
    if projType not in FAN_TYPES:
        raise ValueError("Error: unknown geom type.")
    nx, ny = int(nxy[0]), int(nxy[1])
    betas = np.ascontiguousarray(betas, dtype=np.float64).reshape(-1)
    if betas.size != int(noViews):
        raise ValueError("Error: mx_betas must have noviews X 1 double array.")
    data = np.ascontiguousarray(data, dtype=np.float32)
    fwd = projType.startswith("proj")
    want = (ny, nx) if fwd else (int(noViews), int(np.atleast_1d(nu)[0]))
    if data.shape != want:
        raise ValueError(f"data must have shape {want}")
    nu0 = int(np.atleast_1d(nu)[0])
    out = np.zeros((int(noViews), nu0) if fwd else (ny, nx), dtype=np.float32)
    f32 = lambda v, i=0: float(np.float32(np.atleast_1d(v)[i]))
    ok = _lib.load().ctsim_fbct_geom(projType.encode(), nx, ny, f32(dxy, 0), f32(dxy, 1), f32(cxy, 0), f32(cxy, 1),
                                     nu0, f32(du), f32(cu), f32(SAD), f32(ADD), f32(SDD), int(noViews),
                                     betas.ctypes.data, int(np.atleast_1d(flatPanel)[0]), data.ctypes.data,
                                     out.ctypes.data)
    if not ok:
        raise _lib.CtsimError("fbct_geom_mex: " + _lib.last_error())
    return out


class FanPlan:
    """Device plan of one fan-beam geometry (all of its views) on one GPU."""

    def __init__(self, geom: FanGeometry, device=None):
        import torch
        self.geom = geom
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else
                                   torch.device(device).index or 0)
        s = geom.scalars()
        g = _lib.CtsimFanGeom(s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7], s[8], s[9], s[10], s[11], s[12],
                              int(geom.flatPanel))
        self._betas = np.ascontiguousarray(geom.betas, dtype=np.float64)
        self._L = _lib.load()
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self._L.ctsim_fan_plan_create(C.byref(g), self._betas.ctypes.data, C.byref(h)),
                       "ctsim_fan_plan_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.ctsim_fan_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _views(self, vb, vs, vc):
        if vc is None:
            vc = len(range(vb, self.geom.noViews, vs))
        return int(vb), int(vs), int(vc)

    def _check(self, t, shape, name):
        import torch
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32):
            raise TypeError(f"{name} must be a float32 CUDA tensor")
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"{name} must have shape {tuple(shape)}")
        return t.contiguous()

    def project(self, image, method="dd", view_begin=0, view_stride=1, view_count=None, out=None):
        import torch
        vb, vs, vc = self._views(view_begin, view_stride, view_count)
        image = self._check(image, self.geom.image_shape, "image")
        out = torch.empty((vc, self.geom.nu), dtype=torch.float32, device=self.device) if out is None else out
        m = {"dd": 0, "tf": 1, "proj,dd": 0, "proj,tf": 1}[method]
        st = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._L.ctsim_fan_project(self._h, m, image.data_ptr(), out.data_ptr(), vb, vs, vc, st),
                   "ctsim_fan_project")
        return out

    def backproject(self, sino, method="dd", view_begin=0, view_stride=1, view_count=None, scale=1.0, out=None):
        import torch
        vb, vs, vc = self._views(view_begin, view_stride, view_count)
        sino = self._check(sino, (vc, self.geom.nu), "sino")
        out = torch.empty(self.geom.image_shape, dtype=torch.float32, device=self.device) if out is None else out
        m = {"dd": 2, "tf": 3, "back,dd": 2, "back,tf": 3}[method]
        st = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._L.ctsim_fan_backproject(self._h, m, sino.data_ptr(), out.data_ptr(), vb, vs, vc,
                                                 float(scale), st), "ctsim_fan_backproject")
        return out
