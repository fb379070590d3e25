"""Build the sm_100a projector library in-tree: ctsim_b200/_lib/libctsim_b200.so.

    python -m ctsim_b200.build            # compile (nvcc cross-compiles without a GPU)
    python -m ctsim_b200.build --ptxas    # also print ptxas register/spill/smem usage
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libctsim_b200.so")
SOURCES = ["kernels.cu", "capi.cu", "noalloc.cu", "fdk.cu", "pwls.cu", "sino.cu", "fan.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--shared", "-Xcompiler", "-fPIC,-ffp-contract=off",
    "-cudart", "static",
]


def needs_rebuild() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "ctsim_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    if not force and not verbose_ptxas and not needs_rebuild():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else [])
    cmd += [os.path.join(CSRC, s) for s in SOURCES] + ["-o", LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libctsim_b200.so")
    if verbose_ptxas:
        sys.stdout.write(r.stderr)
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="--ptxas" in sys.argv, force=True)
    print(LIB)
