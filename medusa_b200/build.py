"""Build the medusa_b200 CUDA library in-tree for sm_100a.

    python -m medusa_b200.build [--force] [--verbose]

Produces medusa_b200/_lib/libmedusa_b200.so (exports exactly the mdg_* entry points of
include/medusa_b200.h).  The FP64 sweep translation units are compiled with
-fmad=false and the host code with -ffp-contract=off: no multiply-add contraction, so
every product and sum rounds as in the reference's CPU build.  The mixed-precision
sweep (mdg_sweep1d_mixed.cu) is compiled with -use_fast_math instead.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libmedusa_b200.so")
INCLUDE = os.path.join(ROOT, "include")

SOURCES = ["mdg_capi.cu", "mdg_sweep1d.cu", "mdg_sweep1d_mixed.cu", "mdg_sweep2d.cu", "mdg_misc.cu",
           "mdg_geometry.cpp", "mdg_noalloc.cu", "mdg_server.cu", "mdg_tables.cu", "mdg_sweep3d.cu", "mdg_tma.cu"]
HEADERS = ["mdg_internal.h", "mdg_hydro.cuh", "mdg_kernels.cuh", "mdg_load1d.cuh", "mdg_tables.cuh",
           "mdg_grid3d.cuh", "mdg_mixed.cuh", "mdg_tma.cuh",
           "mdg_timeloop.cuh"]
# The mixed-precision sweep: fast FP32 division/square root and multiply-add contraction
# (its FP64 parts are not required to round like the reference's).
MIXED_FLAGS = ["-use_fast_math"]
FLAGS = {"mdg_sweep1d_mixed.cu": MIXED_FLAGS}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "medusa_b200.h")]
    objs = []
    for src in SOURCES:
        sp = os.path.join(CSRC, src)
        obj = os.path.join(objdir, src + ".o")
        objs.append(obj)
        if not force and _newer(obj, [sp] + hdrs + [os.path.abspath(__file__)]):
            continue
        fp = FLAGS.get(src, ["-fmad=false"])
        cmd = [nvcc(), "-c", sp, "-o", obj, "-std=c++17", "-O3", "-lineinfo"] + fp + [
               "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", "-I", INCLUDE] + ARCH
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed on %s" % src)
    mapfile = os.path.join(objdir, "exports.map")
    with open(mapfile, "w") as f:
        f.write("{ global: mdg_*; local: *; };\n")
    if force or not _newer(LIB, objs + [mapfile]):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + [
            "-Xlinker", "--version-script=" + mapfile, "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            raise RuntimeError("link of libmedusa_b200.so failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
