"""Builds the product library zhijian_b200/libzj_fr.so in-tree with nvcc.

sm_100a only: ``-gencode arch=compute_100a,code=sm_100a``.  Host sources are
compiled with ``-ffp-contract=off`` so the one-time metric terms and normals
round like the reference host code; device code keeps FMA contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libzj_fr.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["host_setup.cpp", "compat_fp64.cu", "phys_fp64.cu", "ns_fp64.cu", "capi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "zj_fr.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    """Compile the library if any source is newer than it; returns its path."""
    if not force and not _stale():
        return LIB
    cmd = [NVCC, "-shared", "-O3", "-std=c++17", "-lineinfo", *ARCH,
           "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           "-o", LIB + ".tmp"]
    if ptxas_v:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose or ptxas_v:
        sys.stdout.write(r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    build_driver()
    return LIB


DRIVER = os.path.join(HERE, "zj_run")


def build_driver() -> str:
    """The C++ driver (cpp/zj_run.cpp) over the FRSolver facade, linked to the
    in-tree library."""
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "cpp", "zj_run.cpp"), "-L", HERE, "-lzj_fr",
           "-Wl,-rpath,$ORIGIN", "-o", DRIVER]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("driver build failed:\n" + r.stderr)
    return DRIVER


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="--ptxas-v" in sys.argv)
