"""FDK reconstruction on the device (fbp/reconFDK.m).

``reconFDK(sino, geom, window, crop)`` keeps the reference's signature: the log
sinogram ``float32[noViews, nu, nv]`` and the geometry in, the attenuation image
``float32[nz, ny, nx]`` out (1/cm when the sinogram holds line integrals of
1/cm -- the reference's units).  Weighting, Parker short-scan weights, the
ramp x window row filter and the ``back,hpd`` backprojection all run on the GPU
(ctsim_fdk_* in include/ctsim_b200.h).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .geometry import CTGeometry
from .projector import plan_for, _is_cuda_tensor

WINDOWS = ("ram-lak", "shepp-logan", "cosine", "hamming", "hann", "hann50", "hann75", "hann80", "B50", "B75", "B80",
           "C50", "C75", "C80")


def design_filter(nu: int, du: float, sdd: float, flat: bool, window: str = "hamming", crop: float = 1.0):
    """Frequency response of fbp/filter/designFilter2.m (flat) or designEquiangularFilter2.m
    (curved), gamma = du, as computed by the library (float64[order])."""
    L = _lib.load()
    order = C.c_int()
    _lib.check(L.ctsim_fdk_design_filter(int(nu), float(du), float(sdd), 1 if flat else 0, window.encode(),
                                         float(crop), None, C.byref(order)), "ctsim_fdk_design_filter")
    H = np.zeros(order.value, dtype=np.float64)
    _lib.check(L.ctsim_fdk_design_filter(int(nu), float(du), float(sdd), 1 if flat else 0, window.encode(),
                                         float(crop), H.ctypes.data, C.byref(order)), "ctsim_fdk_design_filter")
    return H


class FDK:
    """Device FDK reconstructor for one geometry, window and crop."""

    def __init__(self, geom: CTGeometry, window: str = "hamming", crop: float = 1.0, device=None, plan=None):
        if window not in WINDOWS:
            raise ValueError("Invalid window selected.")
        self.geom = geom
        self.plan = plan if plan is not None else plan_for(geom, device)
        L = _lib.load()
        h = C.c_void_p()
        import torch
        with torch.cuda.device(self.plan.device):
            _lib.check(L.ctsim_fdk_create(self.plan._h, window.encode(), float(crop), 1 if geom.shortScan else 0,
                                          C.byref(h)), "ctsim_fdk_create")
        self._h = h
        self._L = L

    @property
    def dbeta(self) -> float:
        return float(self._L.ctsim_fdk_dbeta(self._h))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.ctsim_fdk_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def filter(self, sino, out=None):
        """Cosine/Parker-weighted, ramp-filtered sinogram (reconFDK.m:51-76)."""
        import torch
        sino = self.plan._check_tensor(sino, self.geom.sino_shape, "sino")
        if out is None:
            out = torch.empty(sino.shape, dtype=torch.float32, device=sino.device)
        st = torch.cuda.current_stream(self.plan.device).cuda_stream
        from .projector import _DTYPES
        _lib.check(self._L.ctsim_fdk_filter_ex(self._h, sino.data_ptr(), _DTYPES[sino.dtype], out.data_ptr(), st),
                   "ctsim_fdk_filter")
        return out

    def __call__(self, sino, out=None):
        """The reconstructed image (reconFDK.m:84)."""
        import torch
        sino = self.plan._check_tensor(sino, self.geom.sino_shape, "sino")
        if out is None:
            out = torch.empty(self.geom.image_shape, dtype=torch.float32, device=self.plan.device)
        st = torch.cuda.current_stream(self.plan.device).cuda_stream
        from .projector import _DTYPES
        _lib.check(self._L.ctsim_fdk_run_ex(self._h, sino.data_ptr(), _DTYPES[sino.dtype], out.data_ptr(), st),
                   "ctsim_fdk_run")
        return out


def reconFDK(sino, geom: CTGeometry, window: str = "hamming", crop: float = 1.0):
    """fbp/reconFDK.m.  Torch CUDA tensors stay on the device; numpy arrays go in and come out."""
    key = (window, float(crop))
    cache = geom.__dict__.setdefault("_fdk", {})
    if _is_cuda_tensor(sino):
        f = cache.get((key, sino.device))
        if f is None:
            f = cache[(key, sino.device)] = FDK(geom, window, crop, sino.device)
        return f(sino)
    import torch
    s = torch.from_numpy(np.ascontiguousarray(sino, dtype=np.float32)).cuda()
    f = cache.get((key, s.device))
    if f is None:
        f = cache[(key, s.device)] = FDK(geom, window, crop, s.device)
    return f(s).cpu().numpy()
