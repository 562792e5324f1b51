"""Compile the CUDA library in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
SOURCES = [os.path.join(_HERE, "csrc", "dgm_capi.cu"), os.path.join(_HERE, "csrc", "dgm_noalloc.cu"),
           os.path.join(_HERE, "csrc", "dgm_mesh.cpp"), os.path.join(_HERE, "csrc", "dgm_output.cpp")]
DEPS = SOURCES + [os.path.join(_HERE, "csrc", "dgm_device.cuh"), os.path.join(_HERE, "csrc", "dgm_tc.cuh"),
                  os.path.join(_ROOT, "include", "dgm_b200.h")]
OUT = os.path.join(_HERE, "_lib", "libdgm_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-shared",
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(p) <= t for p in DEPS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [nvcc(), *NVCC_FLAGS, "-I", os.path.join(_ROOT, "include"), "-o", OUT + ".tmp", *SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
