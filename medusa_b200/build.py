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
import time
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libmedusa_b200.so")
INCLUDE = os.path.join(ROOT, "include")

SOURCES = ["mdg_capi.cu", "mdg_sweep1d.cu", "mdg_sweep1d_mixed.cu", "mdg_sweep2d.cu", "mdg_misc.cu",
           "mdg_geometry.cpp", "mdg_noalloc.cu", "mdg_server.cu", "mdg_tables.cu", "mdg_sweep3d.cu", "mdg_tma.cu",
           "mdg_eos_table.cu"]
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


def build(force: bool = False, verbose: bool = False, report: bool = False) -> str:
    """Compile the translation units that are out of date (all with force), in parallel,
    and link the library; with report, one line on stderr says what was compiled."""
    t0 = time.time()
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "medusa_b200.h")]
    objs, jobs = [], []
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
        jobs.append((src, cmd))

    def compile_one(job):
        return job, subprocess.run(job[1], capture_output=True, text=True)

    failed = []
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for (src, cmd), r in ex.map(compile_one, jobs):
            if verbose or r.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed on %s" % ", ".join(failed))
    mapfile = os.path.join(objdir, "exports.map")
    if not (os.path.exists(mapfile) and open(mapfile).read() == "{ global: mdg_*; local: *; };\n"):
        with open(mapfile, "w") as f:
            f.write("{ global: mdg_*; local: *; };\n")
    linked = False
    if force or not _newer(LIB, objs + [mapfile]):
        linked = True
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + [
            "-Xlinker", "--version-script=" + mapfile, "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            raise RuntimeError("link of libmedusa_b200.so failed")
    if report:
        sys.stderr.write("medusa_b200: compiled %d of %d translation units for sm_100a%s, %s libmedusa_b200.so "
                         "(%.0f s)\n" % (len(jobs), len(SOURCES), " (forced)" if force else "",
                                         "linked" if linked else "kept", time.time() - t0))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose, report=True))
