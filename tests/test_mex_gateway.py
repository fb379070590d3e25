"""The MEX gateway sources (ctsim_b200/mex/: cone beam and 2-D fan beam) compile against
a stand-in mex.h and the C ABI header (MATLAB itself is not available here)."""
import os
import subprocess

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


import pytest


@pytest.mark.parametrize("name", ["cbct_geom_mex_b200.c", "fbct_geom_mex_b200.c"])
def test_mex_gateway_compiles(name):
    src = os.path.join(ROOT, "ctsim_b200", "mex", name)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only",
                        "-I", os.path.join(ROOT, "tests", "mex_stub"), "-I", os.path.join(ROOT, "include"), src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_header_is_plain_c():
    hdr = os.path.join(ROOT, "include", "ctsim_b200.h")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-x", "c", hdr],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
