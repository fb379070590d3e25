"""Seeded synthetic phantoms and scan geometries for the benchmark configurations.

No dataset is involved: the reference's own demos read XCAT/CTData volumes
that are not part of this project.  These generators stand in with seeded
ellipsoid phantoms of the configurations' shapes, sizes and attenuation ranges.

Units: phantoms are generated in 1/mm.  The reference projectors expect 1/cm
(they divide the in-plane path length by 10, geom/cbct/cbct_proj.c:300), so
``to_projector_units`` multiplies by 10 before projecting.
"""
from __future__ import annotations

import numpy as np

from .geometry import CTGeometry, circular_betas


def _voxel_centres(geom: CTGeometry):
    nx, ny, nz = geom.reconSize
    dx, dy, dz = geom.reconSpacing
    ox, oy, oz = geom.reconOffset
    x = (np.arange(nx) - (nx - 1) / 2.0 + ox) * dx
    y = (np.arange(ny) - (ny - 1) / 2.0 + oy) * dy
    z = (np.arange(nz) - (nz - 1) / 2.0 + oz) * dz
    return x, y, z


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def ellipsoid_phantom(geom: CTGeometry, n_ellipsoids: int, mu_range, water_mu: float, water_radius: float,
                      centre_radius: float, centre_halfz: float, axis_range, seed: int) -> np.ndarray:
    """Water cylinder (full height) plus seeded rotated ellipsoids; float32[nz, ny, nx] in 1/mm.

    Voxelised by centre sampling; each ellipsoid's value replaces what lies below it.
    """
    rng = np.random.default_rng(seed)
    x, y, z = _voxel_centres(geom)
    img = np.zeros(geom.image_shape, dtype=np.float32)
    r2 = x[None, :] ** 2 + y[:, None] ** 2
    img[:, r2 <= water_radius ** 2] = np.float32(water_mu)
    for _ in range(n_ellipsoids):
        rad = centre_radius * np.sqrt(rng.random())
        ang = rng.uniform(0, 2 * np.pi)
        c = np.array([rad * np.cos(ang), rad * np.sin(ang), rng.uniform(-centre_halfz, centre_halfz)])
        ax = rng.uniform(axis_range[0], axis_range[1], 3)
        R = _random_rotation(rng)
        mu = np.float32(rng.uniform(mu_range[0], mu_range[1]))
        ext = ax.max()
        sx = np.nonzero(np.abs(x - c[0]) <= ext)[0]
        sy = np.nonzero(np.abs(y - c[1]) <= ext)[0]
        sz = np.nonzero(np.abs(z - c[2]) <= ext)[0]
        if sx.size == 0 or sy.size == 0 or sz.size == 0:
            continue
        Z, Y, X = np.meshgrid(z[sz] - c[2], y[sy] - c[1], x[sx] - c[0], indexing="ij")
        P = np.stack([X, Y, Z], axis=-1) @ R  # coordinates in the ellipsoid frame
        inside = ((P / ax) ** 2).sum(-1) <= 1.0
        sub = img[sz[0]:sz[-1] + 1, sy[0]:sy[-1] + 1, sx[0]:sx[-1] + 1]
        sub[inside] = mu
    return img


def to_projector_units(img_per_mm: np.ndarray) -> np.ndarray:
    return (img_per_mm * np.float32(10.0)).astype(np.float32)


def config1(n_views: int = 360, seed: int = 1):
    """Config 1: 128x128x64 at 1 mm, 12 ellipsoids (mu 0.015-0.035 /mm) in a water cylinder
    (0.02 /mm, r 55 mm); 360 views over 2 pi, flat 256x96 detector at 1.6 mm, SAD 1000, SDD 1500."""
    g = CTGeometry((128, 128, 64), (1.0, 1.0, 1.0), (0, 0, 0), (256, 96), (1.6, 1.6), (0, 0), 1000.0, 500.0, 1500.0,
                   circular_betas(n_views))
    x = ellipsoid_phantom(g, 12, (0.015, 0.035), 0.02, 55.0, 45.0, 24.0, (3.0, 15.0), seed)
    return g, x


def config2(n_views: int = 720, seed: int = 2):
    """Config 2: 512x512x256 at 0.5 mm, 20 ellipsoids (mu 0.01-0.05 /mm) in a 150 mm-radius water
    cylinder (wider than the 128 mm half-width grid, so clipped by the volume); 720 views over 2 pi,
    flat 1024x384 detector at 0.8 mm, SAD 1000, SDD 1500."""
    g = CTGeometry((512, 512, 256), (0.5, 0.5, 0.5), (0, 0, 0), (1024, 384), (0.8, 0.8), (0, 0), 1000.0, 500.0,
                   1500.0, circular_betas(n_views))
    x = ellipsoid_phantom(g, 20, (0.01, 0.05), 0.02, 150.0, 100.0, 50.0, (5.0, 30.0), seed)
    return g, x
