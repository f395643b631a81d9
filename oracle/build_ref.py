"""Build recipe for oracle/_ref: the reference's own hydro sweep, compiled UNMODIFIED
from the reference tree, around the glue in oracle/refshim/.

TEST INFRASTRUCTURE ONLY.  Nothing under medusa_b200/ imports, links or runs what
this script builds.  The reference's Makefile is not used: this recipe writes the
build.h that Makefile:157-212 would write (same DEFS list) for each configuration
and compiles the hot-path sources directly with gcc.  Outputs go only into
oracle/_ref/ (git-ignored; it travels with the working tree to a GPU host).

Two binaries per configuration:
  ref_<cfg>        parity build, -O2 -fno-fast-math -ffp-contract=off
  reffast_<cfg>    the reference's own flags (Makefile:14), used as the timed CPU baseline

Usage: python oracle/build_ref.py [--ref-root DIR] [--force]
The reference tree defaults to $MDG_REFERENCE_ROOT, else /root/reference.
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "refshim")
DEFAULT_REF_ROOT = os.environ.get("MDG_REFERENCE_ROOT", "/root/reference")

# hot-path sources compiled unmodified (the link set of the hydro executable minus main.c/io.c,
# whose HDF5 I/O is replaced by the glue)
REF_SOURCES = ["array.c", "mpi.c", "utils.c", "step.c", "geometry.c", "rad_fluid.c",
               "fluid.c", "riemann.c", "reconstruct.c", "bc.c", "eos.c", "timer.c",
               "quadrupole.c", "tracer.c"]

BASE_DEFS = dict(USE_MPI="FALSE", USE_OMP="FALSE", USE_GPU="FALSE", EOS="GAMMA_LAW",
                 GRAV="NO_GRAV", GR_MONOPOLE="FALSE", PN_POTENTIAL="FALSE",
                 USE_EXT_SRC="FALSE", USE_AUX_SRC="FALSE", DO_HYDRO="TRUE",
                 PRINT_OPAC_DATA="FALSE", DO_RADIATION="FALSE", PHOTON="FALSE",
                 NEUTRINO="FALSE", PERTURB="NONE", DO_ROTATION="FALSE",
                 ENFORCE_FLOORS="FALSE", OUTPUT_PRECISION="DOUBLE", DO_TIMING="FALSE",
                 DEBUG="FALSE", POLAR_AVG="FALSE", USE_FORTRAN_CODE="FALSE",
                 USE_EXP_INTERP="FALSE", RAD_CLOSURE="M1", USE_LARGER_STEP="FALSE",
                 USE_LINEAR_ALLOCATION="TRUE", INEL_DT_CONTROL="FALSE")
DEF_ORDER = ["NDIM", "USE_MPI", "USE_OMP", "USE_GPU", "GEOM", "EOS", "GRAV", "GR_MONOPOLE",
             "PN_POTENTIAL", "USE_EXT_SRC", "USE_AUX_SRC", "DO_HYDRO", "PRINT_OPAC_DATA",
             "DO_RADIATION", "PHOTON", "NEUTRINO", "PERTURB", "DO_ROTATION",
             "ENFORCE_FLOORS", "DENDRITIC_GRID", "OUTPUT_PRECISION", "DO_TIMING", "DEBUG",
             "POLAR_AVG", "USE_FORTRAN_CODE", "USE_EXP_INTERP", "RAD_CLOSURE",
             "USE_LARGER_STEP", "USE_LINEAR_ALLOCATION", "INEL_DT_CONTROL", "RCOORD",
             "THCOORD"]

CONFIGS = {
    # 1-D Cartesian (Sod shock tube)
    "cart1d": dict(NDIM="1", GEOM="CARTESIAN", DENDRITIC_GRID="FALSE",
                   RCOORD="UNIFORM", THCOORD="UNIFORM"),
    # 2-D Cartesian (Kelvin-Helmholtz)
    "cart2d": dict(NDIM="2", GEOM="CARTESIAN", DENDRITIC_GRID="FALSE",
                   RCOORD="UNIFORM", THCOORD="UNIFORM"),
    # 1-D spherical, uniform radius (ensemble members: Sod/Noh/Sedov type)
    "sph1d": dict(NDIM="1", GEOM="SPHERICAL", DENDRITIC_GRID="FALSE",
                  RCOORD="UNIFORM", THCOORD="UNIFORM"),
    # the same with the ENFORCE_FLOORS switch on (problems that set rho_floor/e_floor:
    # Noh, double rarefaction)
    "cart1d_floors": dict(NDIM="1", GEOM="CARTESIAN", DENDRITIC_GRID="FALSE",
                          RCOORD="UNIFORM", THCOORD="UNIFORM", ENFORCE_FLOORS="TRUE"),
    "sph1d_floors": dict(NDIM="1", GEOM="SPHERICAL", DENDRITIC_GRID="FALSE",
                         RCOORD="UNIFORM", THCOORD="UNIFORM", ENFORCE_FLOORS="TRUE"),
    # 2-D Cartesian with the fixed gravitational acceleration of GRAV=FIXED_GRAV
    # (Rayleigh-Taylor, problems/init_rt.c; setups/rt_2d.mk)
    "cart2d_grav": dict(NDIM="2", GEOM="CARTESIAN", DENDRITIC_GRID="FALSE",
                        RCOORD="UNIFORM", THCOORD="UNIFORM", GRAV="FIXED_GRAV"),
    # the same acceleration on 1-D Cartesian and spherical grids
    "cart1d_grav": dict(NDIM="1", GEOM="CARTESIAN", DENDRITIC_GRID="FALSE",
                        RCOORD="UNIFORM", THCOORD="UNIFORM", GRAV="FIXED_GRAV"),
    "sph1d_grav": dict(NDIM="1", GEOM="SPHERICAL", DENDRITIC_GRID="FALSE",
                       RCOORD="UNIFORM", THCOORD="UNIFORM", GRAV="FIXED_GRAV"),
    # 3-D spherical on the dendritic grid (Sedov blast), uniform radius and theta
    "sph3d": dict(NDIM="3", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                  RCOORD="UNIFORM", THCOORD="UNIFORM"),
    # 2-D (r, theta) spherical on the dendritic grid
    "sph2d": dict(NDIM="2", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                  RCOORD="UNIFORM", THCOORD="UNIFORM"),
    # the spherical grids with the SINH radial map (r = rtrans sinh(x/rtrans))
    "sph1d_sinh": dict(NDIM="1", GEOM="SPHERICAL", DENDRITIC_GRID="FALSE",
                       RCOORD="SINH", THCOORD="UNIFORM"),
    "sph2d_sinh": dict(NDIM="2", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                       RCOORD="SINH", THCOORD="UNIFORM"),
    "sph3d_sinh": dict(NDIM="3", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                       RCOORD="SINH", THCOORD="UNIFORM"),
    # the reference's default coordinate maps (Makefile:26-27: RCOORD=SINH_MODIFIED,
    # THCOORD=POLYTH), which every setup that does not override them runs with
    "sph1d_default": dict(NDIM="1", GEOM="SPHERICAL", DENDRITIC_GRID="FALSE",
                          RCOORD="SINH_MODIFIED", THCOORD="POLYTH"),
    "sph2d_default": dict(NDIM="2", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                          RCOORD="SINH_MODIFIED", THCOORD="POLYTH"),
    "sph3d_default": dict(NDIM="3", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                          RCOORD="SINH_MODIFIED", THCOORD="POLYTH"),
    # self-gravity in the monopole approximation (GRAV=SPHERICAL_MONOPOLE_GRAV,
    # GR_MONOPOLE=FALSE; setups/dustcollapse_1d.mk): 1-D on the SINH radius with floors,
    # and the dendritic grids
    "sph1d_sinh_mono_floors": dict(NDIM="1", GEOM="SPHERICAL", DENDRITIC_GRID="FALSE",
                                   RCOORD="SINH", THCOORD="UNIFORM", GRAV="SPHERICAL_MONOPOLE_GRAV",
                                   ENFORCE_FLOORS="TRUE"),
    "sph1d_mono": dict(NDIM="1", GEOM="SPHERICAL", DENDRITIC_GRID="FALSE",
                       RCOORD="UNIFORM", THCOORD="UNIFORM", GRAV="SPHERICAL_MONOPOLE_GRAV"),
    "sph2d_mono": dict(NDIM="2", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                       RCOORD="UNIFORM", THCOORD="UNIFORM", GRAV="SPHERICAL_MONOPOLE_GRAV"),
    "sph3d_mono": dict(NDIM="3", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                       RCOORD="UNIFORM", THCOORD="UNIFORM", GRAV="SPHERICAL_MONOPOLE_GRAV"),
    # the fixed acceleration of GRAV=FIXED_GRAV on the dendritic grids
    "sph2d_grav": dict(NDIM="2", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                       RCOORD="UNIFORM", THCOORD="UNIFORM", GRAV="FIXED_GRAV"),
    "sph3d_grav": dict(NDIM="3", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                       RCOORD="UNIFORM", THCOORD="UNIFORM", GRAV="FIXED_GRAV"),
    "sph3d_sinh_grav": dict(NDIM="3", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                            RCOORD="SINH", THCOORD="UNIFORM", GRAV="FIXED_GRAV"),
    # a radius log-spaced outwards from rtrans (RCOORD=LOG, r = rtrans exp(|x|/rtrans)): not
    # one of the reference's maps, added to a generated copy of its spherical metric (see
    # log_metric_source below) for grids that start away from the origin
    "sph1d_log": dict(NDIM="1", GEOM="SPHERICAL", DENDRITIC_GRID="FALSE",
                      RCOORD="LOG", THCOORD="UNIFORM"),
    "sph2d_log": dict(NDIM="2", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                      RCOORD="LOG", THCOORD="UNIFORM"),
    "sph3d_log": dict(NDIM="3", GEOM="SPHERICAL", DENDRITIC_GRID="TRUE",
                      RCOORD="LOG", THCOORD="UNIFORM"),
}

# Value of the LOG enumerator in the generated build.h (enumerators.h:5-11 uses 0-6).
LOG_ENUM = 7

# The three branches added to r_of_x, dr_dx and d2r_dx2 of the generated metric copy
# (metrics/metric_spherical_general.c:149-219), in the form of their SINH branches.
LOG_BRANCHES = {
    "double r_of_x(r_of_x_struct_t rx_info,double x)\n{":
        "  #if (RCOORD==LOG)\n  return rx_info.rtrans*exp(fabs(x)/rx_info.rtrans);\n  #endif\n",
    "double dr_dx(double x)\n{":
        "  #if (RCOORD==LOG)\n  return exp(fabs(x)/rx_info.rtrans);\n  #endif\n",
    "double d2r_dx2(double x)\n{":
        "  #if (RCOORD==LOG)\n  return exp(fabs(x)/rx_info.rtrans)/rx_info.rtrans;\n  #endif\n",
}


def log_metric_source(ref_root, cdir):
    """Write <cdir>/metric_spherical_general_log.c: the reference's spherical metric with a
    LOG branch inserted at the top of r_of_x, dr_dx and d2r_dx2 (nothing else changed),
    and return its path.  The copy is a build product under oracle/_ref/ only."""
    src = open(os.path.join(ref_root, "metrics", "metric_spherical_general.c")).read()
    for anchor, branch in LOG_BRANCHES.items():
        if src.count(anchor) != 1:
            raise RuntimeError("metric_spherical_general.c: cannot place the LOG branch after %r" % anchor)
        src = src.replace(anchor, anchor + "\n" + branch)
    out = os.path.join(cdir, "metric_spherical_general_log.c")
    if not (os.path.exists(out) and open(out).read() == src):
        with open(out, "w") as f:
            f.write(src)
    return out

# configurations also built with the reference's timers on (DO_TIMING=TRUE, its Makefile
# flags): reftime_<cfg> writes timing.csv for the phase split of the CPU baseline
TIMING_CONFIGS = ("cart1d", "cart2d", "sph1d", "sph3d_sinh")

PARITY_FLAGS = ["-O2", "-fno-fast-math", "-ffp-contract=off"]
FAST_FLAGS = ["-O3", "-ffast-math", "-ftree-vectorize", "-fpeel-loops"]


def write_build_h(path, defs):
    lines = ["#ifndef BUILD_H_", "#define BUILD_H_", "", '#include "enumerators.h"', ""]
    if defs.get("RCOORD") == "LOG":
        lines.append("#define LOG %d" % LOG_ENUM)
    for k in DEF_ORDER:
        lines.append("#define %s %s" % (k, defs[k]))
    lines.append("")
    lines.append('#define BUILD_STRING "medusa_b200 oracle/_ref build\\n"')
    lines.append("#endif // BUILD_H_")
    lines.append("")
    text = "\n".join(lines)
    if os.path.exists(path) and open(path).read() == text:
        return
    with open(path, "w") as f:
        f.write(text)


def build_config(name, cfg, ref_root, force=False, timing=False):
    defs = dict(BASE_DEFS)
    defs.update(cfg)
    if timing:
        defs["DO_TIMING"] = "TRUE"
    cdir = os.path.join(OUT, name + ("_timing" if timing else ""))
    os.makedirs(cdir, exist_ok=True)
    write_build_h(os.path.join(cdir, "build.h"), defs)
    srcs = [os.path.join(ref_root, s) for s in REF_SOURCES]
    if defs["GRAV"] != "NO_GRAV":
        srcs.append(os.path.join(ref_root, "gravity.c"))
    if defs["GEOM"] == "SPHERICAL" and defs["RCOORD"] == "LOG":
        srcs.append(log_metric_source(ref_root, cdir))
    elif defs["GEOM"] == "SPHERICAL":
        srcs.append(os.path.join(ref_root, "metrics", "metric_spherical_general.c"))
    else:
        srcs.append(os.path.join(SHIM, "metric_cartesian_current.c"))
    srcs += [os.path.join(SHIM, "ref_harness.c"), os.path.join(SHIM, "ref_main.c")]
    deps = srcs + [os.path.join(cdir, "build.h"), os.path.abspath(__file__)]
    built = []
    exes = (("reftime_" + name, FAST_FLAGS),) if timing else (("ref_" + name, PARITY_FLAGS),
                                                               ("reffast_" + name, FAST_FLAGS))
    for exe, flags in exes:
        target = os.path.join(OUT, exe)
        if (not force and os.path.exists(target)
                and os.path.getmtime(target) >= max(os.path.getmtime(d) for d in deps)):
            built.append(target)
            continue
        # the generated LOG copy includes "../decs.h" as its original does from metrics/
        inc = ["-I" + os.path.join(ref_root, "metrics")] if defs["RCOORD"] == "LOG" else []
        cmd = (["gcc", "-std=gnu99", "-w"] + flags +
               ["-I" + cdir, "-I" + ref_root] + inc + ["-include", "limits.h", "-o", target] + srcs + ["-lm"])
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            raise RuntimeError("oracle/_ref build failed for %s" % exe)
        built.append(target)
    return built


# The reference's own main.c driving a problem end to end (oracle/refshim/dropin_glue.c):
# dropin_cpu_<prob> links the reference's step.c, dropin_gpu_<prob> links
# medusa_b200/host/fornax_binding.c and libmedusa_b200 instead.  name -> (config,
# DROPIN_PROB, MDG_BINDING_PROB_KIND)
DROPIN = {
    "sod": ("cart1d", 1, "MDG_PROB_NONE"),
    "dust": ("sph1d_sinh_mono_floors", 2, "MDG_PROB_DUST"),
    "sedov3d": ("sph3d_default", 3, "MDG_PROB_NONE"),
}
ROOT = os.path.dirname(HERE)
LIBDIR = os.path.join(ROOT, "medusa_b200", "_lib")
BINDING = os.path.join(ROOT, "medusa_b200", "host", "fornax_binding.c")


def build_dropin(name, ref_root, force=False):
    cfgname, prob, kind = DROPIN[name]
    defs = dict(BASE_DEFS)
    defs.update(CONFIGS[cfgname])
    cdir = os.path.join(OUT, cfgname)
    os.makedirs(cdir, exist_ok=True)
    write_build_h(os.path.join(cdir, "build.h"), defs)
    srcs = [os.path.join(ref_root, "main.c")] + [os.path.join(ref_root, s) for s in REF_SOURCES]
    if defs["GRAV"] != "NO_GRAV":
        srcs.append(os.path.join(ref_root, "gravity.c"))
    if defs["GEOM"] == "SPHERICAL":
        srcs.append(os.path.join(ref_root, "metrics", "metric_spherical_general.c"))
    else:
        srcs.append(os.path.join(SHIM, "metric_cartesian_current.c"))
    srcs.append(os.path.join(SHIM, "dropin_glue.c"))
    built = []
    lib = os.path.join(LIBDIR, "libmedusa_b200.so")
    for kind_name in ("cpu", "gpu"):
        target = os.path.join(OUT, "dropin_%s_%s" % (kind_name, name))
        s = list(srcs)
        extra = []
        if kind_name == "gpu":
            s = [x for x in s if os.path.basename(x) != "step.c"] + [BINDING]
            extra = ["-I" + os.path.join(ROOT, "include"), "-DMDG_BINDING_PROB_KIND=" + kind,
                     "-L" + LIBDIR, "-lmedusa_b200", "-Wl,-rpath,$ORIGIN/../../medusa_b200/_lib"]
            if not os.path.exists(lib):
                raise FileNotFoundError("build libmedusa_b200.so first (python -m medusa_b200.build)")
        deps = s + [os.path.join(cdir, "build.h"), os.path.abspath(__file__)] + ([lib] if kind_name == "gpu" else [])
        if (not force and os.path.exists(target)
                and os.path.getmtime(target) >= max(os.path.getmtime(d) for d in deps)):
            built.append(target)
            continue
        cmd = (["gcc", "-std=gnu99", "-w"] + PARITY_FLAGS + ["-DDROPIN_PROB=%d" % prob] +
               ["-I" + cdir, "-I" + ref_root, "-include", "limits.h", "-o", target] + s + extra + ["-lm"])
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            raise RuntimeError("oracle/_ref build failed for %s" % target)
        built.append(target)
    return built


def build_eos(ref_root, force=False):
    """oracle/_ref/refeos: the reference's tabulated-EOS zone update
    (eos/burrows/eos_stuff.c, unmodified) driven by oracle/refshim/eos_ref_harness.c, with
    the parity flags and the build switches of the 1-D spherical configuration."""
    defs = dict(BASE_DEFS)
    defs.update(CONFIGS["sph1d"])
    cdir = os.path.join(OUT, "eos")
    os.makedirs(cdir, exist_ok=True)
    write_build_h(os.path.join(cdir, "build.h"), defs)
    srcs = [os.path.join(ref_root, "eos", "burrows", "eos_stuff.c"), os.path.join(SHIM, "eos_ref_harness.c")]
    target = os.path.join(OUT, "refeos")
    deps = srcs + [os.path.join(cdir, "build.h"), os.path.abspath(__file__)]
    if (not force and os.path.exists(target)
            and os.path.getmtime(target) >= max(os.path.getmtime(d) for d in deps)):
        return [target]
    cmd = (["gcc", "-std=gnu99", "-w"] + PARITY_FLAGS + ["-I" + cdir, "-I" + ref_root, "-include", "limits.h",
                                                        "-o", target] + srcs + ["-lm"])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("oracle/_ref build failed for refeos")
    return [target]


def build(ref_root=DEFAULT_REF_ROOT, force=False, dropin=True):
    """Build every configuration (and, when libmedusa_b200.so is built, the drop-in
    runs); returns the list of binaries.  Needs the reference tree."""
    if not os.path.isdir(ref_root):
        raise FileNotFoundError("reference tree not found at %s" % ref_root)
    os.makedirs(OUT, exist_ok=True)
    out = []
    for name, cfg in CONFIGS.items():
        out += build_config(name, cfg, ref_root, force)
    for name in TIMING_CONFIGS:
        out += build_config(name, CONFIGS[name], ref_root, force, timing=True)
    out += build_eos(ref_root, force)
    if dropin and os.path.exists(os.path.join(LIBDIR, "libmedusa_b200.so")):
        for name in DROPIN:
            out += build_dropin(name, ref_root, force)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=DEFAULT_REF_ROOT)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    for p in build(a.ref_root, a.force):
        print(p)
