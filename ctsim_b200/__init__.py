"""ctsim_b200: B200 (sm_100a) cone-beam projectors behind the CTSim MEX interface.

The product is the CUDA library ``_lib/libctsim_b200.so`` (C ABI in
include/ctsim_b200.h); this package is its Python host side.
"""
from .geometry import CTGeometry, circular_betas
from .projector import (Plan, plan_for, cbct_geom_mex, forwardProjectMex, backProjectMex, orderedSubset,
                        loadPojectors)

__all__ = ["CTGeometry", "circular_betas", "Plan", "plan_for", "cbct_geom_mex", "forwardProjectMex",
           "backProjectMex", "orderedSubset", "loadPojectors"]
