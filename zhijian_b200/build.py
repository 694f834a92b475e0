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

SOURCES = ["host_setup.cpp", "tri_setup.cpp", "gmsh.cpp", "partition.cpp", "compat_fp64.cu", "phys_fp64.cu", "phys_fp32.cu", "ns_fp64.cu",
           "ns_fp32.cu", "ns_tc.cu", "tri_fp64.cu", "tri_fp32.cu", "jvp.cu", "adjoint.cu", "capi.cu"]
OBJDIR = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "zj_fr.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    """Compile the library if any source is newer than it; returns its path.
    Each translation unit compiles in its own nvcc process (in parallel),
    then one nvcc links the shared library."""
    if not force and not _stale():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    flags = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
             "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if ptxas_v:
        flags += ["-Xptxas", "-v"]
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
        cmd = [NVCC, "-c", *flags, "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                            text=True)))
        objs.append(obj)
    errors = []
    for src, pr in procs:
        out, _ = pr.communicate()
        if pr.returncode != 0:
            errors.append(f"{src}:\n{out}")
        elif verbose or ptxas_v:
            sys.stdout.write(out)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    cmd = [NVCC, "-shared", *ARCH, "-o", LIB + ".tmp", *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
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
