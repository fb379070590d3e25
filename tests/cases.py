"""Geometry cases shared by the parity tests and the golden-fixture generator.

Small enough for the single-threaded oracle to finish in well under a second
each; chosen to reach the edge behaviour of the reference projectors.  Every
case keeps distance-driven u footprints at 10 detector columns or fewer (the
reference writes wider footprints past its 10-entry weight array).
"""
from __future__ import annotations

import numpy as np

from ctsim_b200.geometry import CTGeometry, circular_betas


def _geom(size, spacing, offset, det, dspacing, doffset, nviews, flat=1, sad=1000.0, sdd=1500.0, betas=None,
          couch=None, mask=None):
    if betas is None:
        betas = circular_betas(nviews)
    return CTGeometry(size, spacing, offset, det, dspacing, doffset, sad, sdd - sad, sdd, betas,
                      couchZ=couch, flatPanel=flat, map=mask)


def make_cases():
    rng = np.random.default_rng(20261203)
    cases = {}
    cases["basic"] = _geom((24, 20, 10), (1.0, 1.0, 1.0), (0, 0, 0), (48, 16), (1.6, 1.6), (0, 0), 11)
    cases["offsets_curved"] = _geom((20, 22, 9), (1.0, 1.0, 1.0), (0.3, -0.2, 0.7), (40, 14), (1.6, 1.6),
                                    (1.5, -0.5), 13, flat=0,
                                    betas=np.sort(rng.uniform(0, 2 * np.pi, 13)))
    mask = rng.random((18, 16)) > 0.25
    cases["couch_map"] = _geom((16, 18, 12), (1.0, 1.0, 1.0), (0, 0, 0), (36, 20), (1.5, 1.5), (0, 0), 9,
                               couch=np.linspace(-6.0, 6.0, 9).astype(np.float32), mask=mask)
    cases["truncated"] = _geom((24, 24, 8), (1.0, 1.0, 1.0), (0, 0, 0), (20, 6), (1.6, 1.6), (2.0, 0.5), 10)
    cases["thick_slices"] = _geom((14, 14, 6), (1.0, 1.0, 2.5), (0, 0, 0), (30, 40), (1.6, 0.8), (0, 0), 8)
    cases["fine_voxels"] = _geom((30, 30, 12), (0.3, 0.3, 0.3), (0, 0, 0), (24, 12), (1.6, 1.6), (0, 0), 7)
    cases["ragged"] = _geom((13, 11, 37), (1.0, 1.0, 0.5), (0.5, 0, -1.0), (30, 34), (1.4, 1.2), (0, 0), 5)
    cases["wide_u"] = _geom((10, 12, 6), (2.0, 2.0, 1.0), (0, 0, 0), (80, 12), (0.4, 1.6), (0, 0), 6)
    cases["short_scan"] = _geom((18, 18, 8), (1.0, 1.0, 1.0), (0, 0, 0), (40, 12), (1.6, 1.6), (0, 0), 12,
                                betas=np.linspace(0.1, np.pi + 0.6, 12))
    cases["tall_curved"] = _geom((12, 12, 70), (1.0, 1.0, 0.4), (0, 0, 0), (30, 60), (1.6, 1.0), (0, 0), 5, flat=0)
    return cases


def make_arc_cases():
    """Arc-detector geometries (detector_type 2: an arc of radius ADD about the rotation
    axis, geom/cbct/cbct_proj3.c), for the distance-driven pair only."""
    rng = np.random.default_rng(20261204)
    cases = {}
    cases["arc_basic"] = _geom((24, 20, 10), (1.0, 1.0, 1.0), (0, 0, 0), (48, 16), (1.2, 1.6), (0, 0), 11, flat=2)
    cases["arc_offsets_couch"] = _geom((20, 22, 9), (1.0, 1.0, 1.0), (0.3, -0.2, 0.7), (44, 14), (1.3, 1.6),
                                       (1.5, -0.5), 13, flat=2, betas=np.sort(rng.uniform(0, 2 * np.pi, 13)),
                                       couch=np.linspace(-4.0, 4.0, 13).astype(np.float32),
                                       mask=rng.random((22, 20)) > 0.2)
    return cases


ARC_KINDS = ("proj,dd", "back,dd")


def make_fan_cases():
    """2-D fan-beam geometries (geom/fbct): flat and curved detectors, offsets, a truncated
    detector and footprints several bins wide (the 2-D code has no footprint-width limit)."""
    from ctsim_b200.geometry import FanGeometry
    rng = np.random.default_rng(20261205)
    return {
        "fan_basic": FanGeometry((32, 28), (1.0, 1.0), (0, 0), 64, 1.2, 0.0, 1000.0, 500.0, 1500.0,
                                 circular_betas(17)),
        "fan_offsets_curved": FanGeometry((30, 34), (0.7, 0.9), (0.4, -0.3), 50, 1.6, 2.5, 900.0, 600.0, 1500.0,
                                          np.sort(rng.uniform(0, 2 * np.pi, 13)), 0),
        "fan_wide": FanGeometry((16, 16), (2.0, 2.0), (0, 0), 90, 0.5, -3.0, 1000.0, 500.0, 1500.0,
                                circular_betas(9)),
        "fan_truncated": FanGeometry((40, 40), (1.0, 1.0), (0, 0), 24, 1.6, 4.0, 1000.0, 500.0, 1500.0,
                                     circular_betas(10)),
    }


FAN_KINDS = ("proj,dd", "proj,tf", "back,dd", "back,tf")


def case_inputs(geom, seed=0):
    """Seeded non-negative image (with exact zeros) and sinogram for a case."""
    rng = np.random.default_rng(seed)
    x = rng.random(geom.image_shape, dtype=np.float32)
    x[x < 0.1] = 0.0
    y = rng.random(geom.sino_shape, dtype=np.float32)
    return x, y


KINDS = ("proj,dd", "proj,tf", "back,dd", "back,tf", "back,pd", "back,hpd", "back,var")
