"""Cone-beam geometry, mirroring the reference's MATLAB ``geom`` struct.

The reference builds this struct in ``parameters/loadProjectionGeometryCT.m``
and passes its fields to the MEX projectors in a fixed order
(``geom/shell/forwardProjectMex.m:82-85``)::

    <mex>(type, int32(reconSize), single(reconSpacing), single(reconOffset),
          int32(detSize), single(detSpacing), single(detOffset),
          single(SAD), single(ADD), single(SDD), int32(noViews),
          double(betas), single(couchZ), int32(flatPanel), single(data),
          logical(map))

Array conventions used throughout this package (C order, numpy/torch):

* image  ``float32[nz, ny, nx]``  == MATLAB ``single[nx ny nz]`` (x fastest)
* sino   ``float32[noViews, nu, nv]`` == MATLAB ``single[nv nu noViews]`` (v fastest)
* map    ``bool[ny, nx]``          == MATLAB ``logical[nx ny]``

Units follow the reference: lengths in mm, attenuation in 1/cm inside the
projectors (they divide the in-plane path length by 10,
``geom/cbct/cbct_proj.c:300``).
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import Optional

import numpy as np


@dataclass
class CTGeometry:
    reconSize: tuple            # (nx, ny, nz)
    reconSpacing: tuple         # (dx, dy, dz) mm
    reconOffset: tuple          # (ox, oy, oz) in voxels
    detSize: tuple              # (nu, nv)
    detSpacing: tuple           # (du, dv) mm
    detOffset: tuple            # (ou, ov) in pixels
    SAD: float
    ADD: float
    SDD: float
    betas: np.ndarray           # float64[noViews], radians
    couchZ: Optional[np.ndarray] = None   # float32[noViews], mm
    flatPanel: int = 1          # 1 flat, 0 curved (equiangular)
    map: Optional[np.ndarray] = None      # bool[ny, nx]
    shortScan: bool = False

    def __post_init__(self):
        self.reconSize = tuple(int(v) for v in self.reconSize)
        self.reconSpacing = tuple(float(np.float32(v)) for v in self.reconSpacing)
        self.reconOffset = tuple(float(np.float32(v)) for v in self.reconOffset)
        self.detSize = tuple(int(v) for v in self.detSize)
        self.detSpacing = tuple(float(np.float32(v)) for v in self.detSpacing)
        self.detOffset = tuple(float(np.float32(v)) for v in self.detOffset)
        self.betas = np.ascontiguousarray(np.asarray(self.betas, dtype=np.float64).reshape(-1))
        if self.couchZ is None:
            self.couchZ = np.zeros(self.betas.size, dtype=np.float32)
        self.couchZ = np.ascontiguousarray(np.asarray(self.couchZ, dtype=np.float32).reshape(-1))
        if self.map is None:
            self.map = np.ones((self.ny, self.nx), dtype=bool)
        self.map = np.ascontiguousarray(np.asarray(self.map, dtype=bool))
        if self.map.shape != (self.ny, self.nx):
            raise ValueError("map must have shape (ny, nx)")
        if self.couchZ.size != self.betas.size:
            raise ValueError("couchZ must have one entry per view")

    # convenience accessors -------------------------------------------------
    nx = property(lambda s: s.reconSize[0])
    ny = property(lambda s: s.reconSize[1])
    nz = property(lambda s: s.reconSize[2])
    nu = property(lambda s: s.detSize[0])
    nv = property(lambda s: s.detSize[1])
    noViews = property(lambda s: int(s.betas.size))

    @property
    def image_shape(self):
        return (self.nz, self.ny, self.nx)

    @property
    def sino_shape(self):
        return (self.noViews, self.nu, self.nv)

    @property
    def voxel_views(self) -> int:
        return self.nx * self.ny * self.nz * self.noViews

    def subset(self, M: int, isub: int) -> "CTGeometry":
        """Views ``1+mod(isub,M):M:end`` (geom/shell/forwardProjectMex.m:36-38)."""
        if M == 1:
            return self
        sel = slice(isub % M, None, M)
        return replace(self, betas=self.betas[sel].copy(), couchZ=self.couchZ[sel].copy())

    def scalars(self):
        """The scalar MEX arguments in reference order (after ``type``)."""
        return (self.nx, self.ny, self.nz,
                self.reconSpacing[0], self.reconSpacing[1], self.reconSpacing[2],
                self.reconOffset[0], self.reconOffset[1], self.reconOffset[2],
                self.nu, self.nv, self.detSpacing[0], self.detSpacing[1],
                self.detOffset[0], self.detOffset[1],
                float(np.float32(self.SAD)), float(np.float32(self.ADD)), float(np.float32(self.SDD)),
                self.noViews)


def circular_betas(n_views: int, arc: float = 2 * np.pi) -> np.ndarray:
    """Evenly spaced view angles ``(0:N-1) * arc / N`` (geom/test_projectors_3d.m:59)."""
    return np.arange(n_views, dtype=np.float64) * (arc / n_views)


def helical_geometry(reconSize, reconSpacing, reconOffset, detSize, detSpacing, detOffset, SAD: float, ADD: float,
                     noViewsTurn: int, noTurns: int, pitch: float, flatPanel: int = 1) -> CTGeometry:
    """Helical scan (parameters/loadProjectionGeometryHelicalCT.m:16-57): noViewsTurn *
    noTurns + 1 views centred on beta = pi, the couch advancing pitch * (detector height)
    per turn (couchZ in mm, centred on 0), and the FOV map of the fan."""
    SDD = SAD + ADD
    n_views = int(noViewsTurn) * int(noTurns) + 1
    k = np.arange(1, n_views + 1, dtype=np.float64) - (n_views + 1) / 2.0
    couch_spacing = pitch * detSize[1] * detSpacing[1] / noViewsTurn
    betas = k * 2.0 * np.pi / noViewsTurn + np.pi
    couch = (k * couch_spacing).astype(np.float32)
    half_fan = detSize[0] * detSpacing[0] / 2.0 / SDD
    if flatPanel:
        half_fan = np.arctan(half_fan)
    fov = 2.0 * np.sin(half_fan) * SAD
    nx, ny = int(reconSize[0]), int(reconSize[1])
    x = np.arange(nx) - (nx - 1) / 2.0
    y = np.arange(ny) - (ny - 1) / 2.0
    radius = max(max(reconSize), fov / reconSpacing[0]) / 2.0
    mask = np.sqrt(x[None, :] ** 2 + y[:, None] ** 2) < radius      # [ny, nx]
    return CTGeometry(reconSize, reconSpacing, reconOffset, detSize, detSpacing, detOffset, SAD, ADD, SDD, betas,
                      couchZ=couch, flatPanel=flatPanel, map=mask, shortScan=True)


@dataclass
class FanGeometry:
    """2-D fan-beam geometry, the arguments of geom/fbct/fbct_geom_mex.c:66-84:
    image ``[ny, nx]`` (MATLAB ``[nx ny]``), sinogram ``[noViews, nu]`` (MATLAB ``[nu noViews]``)."""
    reconSize: tuple            # (nx, ny)
    reconSpacing: tuple         # (dx, dy) mm
    reconOffset: tuple          # (ox, oy) voxels
    nu: int
    du: float
    detOffset: float            # pixels
    SAD: float
    ADD: float
    SDD: float
    betas: np.ndarray
    flatPanel: int = 1

    def __post_init__(self):
        self.reconSize = tuple(int(v) for v in self.reconSize)
        self.reconSpacing = tuple(float(np.float32(v)) for v in self.reconSpacing)
        self.reconOffset = tuple(float(np.float32(v)) for v in self.reconOffset)
        self.nu = int(self.nu)
        self.du = float(np.float32(self.du))
        self.detOffset = float(np.float32(self.detOffset))
        self.betas = np.ascontiguousarray(np.asarray(self.betas, dtype=np.float64).reshape(-1))

    nx = property(lambda s: s.reconSize[0])
    ny = property(lambda s: s.reconSize[1])
    noViews = property(lambda s: int(s.betas.size))

    @property
    def image_shape(self):
        return (self.ny, self.nx)

    @property
    def sino_shape(self):
        return (self.noViews, self.nu)

    def scalars(self):
        """nx, ny, dx, dy, ox, oy, nu, du, ou, sad, add, sdd, noviews (fbct_geom_mex.c order)."""
        return (self.nx, self.ny, self.reconSpacing[0], self.reconSpacing[1], self.reconOffset[0],
                self.reconOffset[1], self.nu, self.du, self.detOffset, float(np.float32(self.SAD)),
                float(np.float32(self.ADD)), float(np.float32(self.SDD)), self.noViews)
