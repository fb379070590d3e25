"""Generate the golden fixtures from the reference's own compiled C.

Runs every case of tests/cases.py through the reference's geom/cbct projectors
(built unmodified by oracle/Makefile into oracle/_ref/libcbct_ref.so; the arc-detector
cases through cbct_proj3.c / cbct_back3.c in oracle/_ref/libcbct_ref3.so) and saves
inputs and outputs as tests/golden/<case>.npz.  Needs the reference checkout
only when the library has to be built.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from cases import (ARC_KINDS, FAN_KINDS, KINDS, case_inputs, make_arc_cases, make_cases,  # noqa: E402
                   make_fan_cases)
from oracle.bindings import build, ref3_cbct, ref_available, ref_cbct, ref_fbct  # noqa: E402


def main():
    if not ref_available():
        build()
    for name, g in make_cases().items():
        x, y = case_inputs(g)
        out = {"image_in": x, "sino_in": y, "betas": g.betas, "couchZ": g.couchZ, "map": g.map}
        for k in KINDS:
            src = x if k.startswith("proj") else y
            out[k.replace(",", "_")] = ref_cbct(k, g, src)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))
    # the arc detector: the reference's geom/cbct/cbct_proj3.c / cbct_back3.c pair
    for name, g in make_arc_cases().items():
        x, y = case_inputs(g)
        out = {"image_in": x, "sino_in": y, "betas": g.betas, "couchZ": g.couchZ, "map": g.map}
        for k in ARC_KINDS:
            out[k.replace(",", "_")] = ref3_cbct(k, g, x if k.startswith("proj") else y)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


def fan_main():
    """The 2-D fan-beam pair (geom/fbct/fbct_proj.c, fbct_back.c through ref_shim_fbct.c)."""
    for name, g in make_fan_cases().items():
        x, y = case_inputs(g)
        out = {"image_in": x, "sino_in": y, "betas": g.betas}
        for k in FAN_KINDS:
            out[k.replace(",", "_")] = ref_fbct(k, g, x if k.startswith("proj") else y)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
    fan_main()
