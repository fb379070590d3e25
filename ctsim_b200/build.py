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
    """Compile every source to an object (in parallel), then link the shared library."""
    if not force and not verbose_ptxas and not needs_rebuild():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OUT_DIR, exist_ok=True)
    compile_flags = [f for f in FLAGS if f not in ("--shared", "-cudart", "static")]

    def compile_one(src):
        obj = os.path.join(OUT_DIR, os.path.splitext(src)[0] + ".o")
        cmd = [NVCC] + compile_flags + (["-Xptxas", "-v"] if verbose_ptxas else [])
        cmd += ["-c", os.path.join(CSRC, src), "-o", obj]
        return obj, subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    for obj, r in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed compiling {os.path.basename(obj)}")
        if verbose_ptxas:
            sys.stdout.write(r.stderr)
    r = subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "--shared", "-cudart", "static"] +
                       [o for o, _ in results] + ["-o", LIB], capture_output=True, text=True)
    for o, _ in results:
        os.remove(o)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libctsim_b200.so")
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="--ptxas" in sys.argv, force=True)
    print(LIB)
