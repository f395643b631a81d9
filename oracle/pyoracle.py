"""Python access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

- :func:`build_oracle` compiles oracle/hydro_oracle.c (the plain-C restatement of the
  reference sweep) into oracle/_build/liboracle.so with -O2 -fno-fast-math
  -ffp-contract=off, the flags under which it reproduces the reference bit for bit.
- :class:`Oracle` drives that library through ctypes.
- :func:`run_reference` runs the reference itself (built unmodified by
  oracle/build_ref.py into oracle/_ref/) on the same problem in a subprocess.

Only tests/, __graft_entry__.smoke(), bench.py's CPU-baseline leg and
oracle/reference_phases.py (the timer split of that baseline) use this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
SRC = os.path.join(HERE, "hydro_oracle.c")
EOS_SRC = os.path.join(HERE, "eos_table_oracle.c")
ORACLE_FLAGS = ["-O2", "-fno-fast-math", "-ffp-contract=off"]


class Params(ctypes.Structure):
    """Field order of ref_params (oracle/refshim/ref_harness.c) and orc_params."""
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("n3", ctypes.c_int),
                ("startx", ctypes.c_double * 3), ("dx", ctypes.c_double * 3),
                ("gam", ctypes.c_double), ("Kpoly", ctypes.c_double),
                ("eos_kind", ctypes.c_int),
                ("bc_lo", ctypes.c_int * 3), ("bc_hi", ctypes.c_int * 3),
                ("prob_kind", ctypes.c_int),
                ("cfl", ctypes.c_double),
                ("dt_init_safety", ctypes.c_double), ("dt_grow_safety", ctypes.c_double),
                ("initial_dt", ctypes.c_double), ("dtmax", ctypes.c_double),
                ("dtmin", ctypes.c_double), ("tmax", ctypes.c_double),
                ("rtrans", ctypes.c_double), ("hydro_interp_order", ctypes.c_int),
                ("enforce_floors", ctypes.c_int), ("rho_floor", ctypes.c_double),
                ("e_floor", ctypes.c_double), ("grav", ctypes.c_double * 3), ("rcoord", ctypes.c_int),
                ("rfact", ctypes.c_double * 3), ("thcoord", ctypes.c_int), ("poly_xt", ctypes.c_double),
                ("poly_alpha", ctypes.c_double)]


def params_of(pb) -> Params:
    p = Params()
    p.n1, p.n2, p.n3 = pb.n
    for d in range(3):
        p.startx[d] = pb.startx[d]
        p.dx[d] = pb.dx[d]
        p.bc_lo[d] = pb.bc_lo[d]
        p.bc_hi[d] = pb.bc_hi[d]
    p.gam, p.Kpoly, p.eos_kind, p.prob_kind = pb.gam, pb.Kpoly, pb.eos, pb.prob_kind
    p.cfl = pb.cfl
    p.dt_init_safety, p.dt_grow_safety = pb.dt_init_safety, pb.dt_grow_safety
    p.initial_dt, p.dtmax, p.dtmin, p.tmax = pb.initial_dt, pb.dtmax, pb.dtmin, pb.tmax
    p.rtrans = pb.rtrans
    p.hydro_interp_order = pb.hydro_interp_order
    p.enforce_floors = int(getattr(pb, "enforce_floors", 0))
    p.rho_floor = getattr(pb, "rho_floor", -1.0)
    p.e_floor = getattr(pb, "e_floor", -1.0)
    for d in range(3):
        p.grav[d] = getattr(pb, "grav", (0.0, 0.0, 0.0))[d]
    p.rcoord = int(getattr(pb, "rcoord", 0))
    for d in range(3):
        p.rfact[d] = getattr(pb, "rfact", (1.0e6, 1.5e6, 5.0e5))[d]
    p.thcoord = int(getattr(pb, "thcoord", 0))
    p.poly_xt = getattr(pb, "poly_xt", 1.2)
    p.poly_alpha = getattr(pb, "poly_alpha", 4.0)
    return p


def build_oracle(force: bool = False) -> str:
    os.makedirs(BUILD_DIR, exist_ok=True)
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= max(os.path.getmtime(SRC), os.path.getmtime(EOS_SRC))):
        return LIB_PATH
    cmd = ["gcc", "-std=gnu99", "-shared", "-fPIC"] + ORACLE_FLAGS + ["-o", LIB_PATH, SRC, EOS_SRC, "-lm"]
    subprocess.run(cmd, check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_oracle()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(Params), ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_advance_one.restype = ctypes.c_double
        L.orc_advance_one.argtypes = [ctypes.c_void_p]
        L.orc_estimate_dt.restype = ctypes.c_double
        L.orc_estimate_dt.argtypes = [ctypes.c_void_p]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.orc_get_t.restype = ctypes.c_double
        L.orc_get_t.argtypes = [ctypes.c_void_p]
        L.orc_get_min_dt.restype = ctypes.c_double
        L.orc_get_min_dt.argtypes = [ctypes.c_void_p]
        L.orc_get_istep.argtypes = [ctypes.c_void_p]
        L.orc_get_interior.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_set_interior.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_restart.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.orc_get_moments0.argtypes = [ctypes.c_void_p] * 4
        L.orc_get_geom.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.orc_eos_given_rex_n.argtypes = [ctypes.c_void_p, ctypes.POINTER(EosGrid), ctypes.c_int] + [ctypes.c_void_p] * 5
        _lib = L
    return _lib


class EosGrid(ctypes.Structure):
    """orc_eos_grid of oracle/eos_table_oracle.c: table sizes and grid bounds."""
    _fields_ = [("nrec", ctypes.c_int), ("ny", ctypes.c_int), ("nr", ctypes.c_int), ("nt", ctypes.c_int),
                ("r1", ctypes.c_double), ("r2", ctypes.c_double), ("t1", ctypes.c_double),
                ("t2", ctypes.c_double), ("y1", ctypes.c_double), ("y2", ctypes.c_double),
                ("const_hack", ctypes.c_double)]


def eos_given_rex(table, grid: EosGrid, rho, u, ye, temp_guess):
    """The tabulated EOS update of eos_given_rex_per_zone (eos/burrows/eos_stuff.c:768-902)
    for every zone: returns [n][5] = pressure, sound speed, temperature, entropy, Gamma_1."""
    table = np.ascontiguousarray(table, dtype=np.float64)
    cols = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, ye, temp_guess)]
    n = cols[0].size
    out = np.zeros((n, 5))
    lib().orc_eos_given_rex_n(table.ctypes.data, ctypes.byref(grid), n, *[c.ctypes.data for c in cols],
                              out.ctypes.data)
    return out


class Oracle:
    """One problem advanced by the CPU restatement."""

    def __init__(self, pb):
        self.pb = pb
        self._prm = params_of(pb)
        ic = np.ascontiguousarray(pb.ic, dtype=np.float64)
        self._h = lib().orc_create(ctypes.byref(self._prm), pb.ndim, pb.geom, ic.ctypes.data)
        if not self._h:
            raise ValueError("the oracle does not restate this problem's coordinate maps "
                             "(rcoord %d, thcoord %d)" % (self._prm.rcoord, self._prm.thcoord))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def advance(self, nsteps: int = 1):
        """Run nsteps passes of the reference time loop; returns the list of dt used."""
        return [lib().orc_advance_one(self._h) for _ in range(nsteps)]

    def estimate_dt(self) -> float:
        return lib().orc_estimate_dt(self._h)

    def step(self, dt: float):
        lib().orc_step(self._h, dt)

    @property
    def t(self) -> float:
        return lib().orc_get_t(self._h)

    @property
    def min_dt(self) -> float:
        return lib().orc_get_min_dt(self._h)

    def state(self):
        prim = np.zeros((self.pb.ncell, 5))
        eos = np.zeros((self.pb.ncell, 5))
        lib().orc_get_interior(self._h, prim.ctypes.data, eos.ctypes.data)
        return prim, eos

    def set_state(self, prim):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        lib().orc_set_interior(self._h, prim.ctypes.data)

    def restart(self, prim, t: float, istep: int):
        """Resume from a restart (state, time, step) as a new reference process does:
        EOS of the state, dtold = 1e100, estimate_dt's first-call reset."""
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        lib().orc_restart(self._h, prim.ctypes.data, float(t), int(istep))

    def moments0(self):
        n = self.pb.n[0] + 4
        a, b, g = np.zeros(n), np.zeros(n), np.zeros(n)
        lib().orc_get_moments0(self._h, a.ctypes.data, b.ctypes.data, g.ctypes.data)
        return a, b, g

    def geom(self, i: int, j: int = 0):
        out = np.zeros(64)
        lib().orc_get_geom(self._h, i, j, out.ctypes.data)
        return out


# ----------------------------------------------------------------------------- reference
def ref_config(pb) -> str:
    """The oracle/_ref build of a problem: its geometry and dimension, its radial map,
    its gravity (FIXED_GRAV, SPHERICAL_MONOPOLE_GRAV) and whether ENFORCE_FLOORS is
    compiled in."""
    name = ("cart%dd" if pb.geom == 0 else "sph%dd") % pb.ndim
    if getattr(pb, "rcoord", 0) == 1:
        name += "_sinh"
    elif getattr(pb, "rcoord", 0) == 3:
        name += "_log"
    elif getattr(pb, "rcoord", 0) == 2 and getattr(pb, "thcoord", 0) == 1:
        name += "_default"
    if any(g != 0.0 for g in getattr(pb, "grav", (0.0, 0.0, 0.0))):
        name += "_grav"
    if getattr(pb, "monopole", 0):
        name += "_mono"
    return name + ("_floors" if getattr(pb, "enforce_floors", 0) else "")


def ref_available(pb, fast: bool = False) -> bool:
    exe = os.path.join(REF_DIR, ("reffast_" if fast else "ref_") + ref_config(pb))
    return os.path.exists(exe)


def _write_input(pb, path):
    prm = params_of(pb)
    with open(path, "wb") as f:
        f.write(bytes(prm))
        f.write(np.ascontiguousarray(pb.ic, dtype=np.float64).tobytes())


def run_reference(pb, nsteps: int, every: int = 1):
    """Run the unmodified reference for nsteps; returns a list of snapshots
    (istep, t, dt_used, min_dt, prim[ncell,5]) including the initial state."""
    exe = os.path.join(REF_DIR, "ref_" + ref_config(pb))
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        _write_input(pb, fin)
        subprocess.run([exe, "run", fin, fout, str(nsteps), str(every)], check=True, cwd=td,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        raw = np.fromfile(fout, dtype=np.float64)
    rec = 4 + 5 * pb.ncell
    raw = raw.reshape(-1, rec)
    return [(int(r[0]), r[1], r[2], r[3], r[4:].reshape(pb.ncell, 5).copy()) for r in raw]


def _ref_dump(pb, what: str) -> bytes:
    exe = os.path.join(REF_DIR, "ref_" + ref_config(pb))
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        _write_input(pb, fin)
        subprocess.run([exe, what, fin, fout], check=True, cwd=td, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL)
        with open(fout, "rb") as f:
            return f.read()


def reference_grid(pb):
    """The reference's dendritic zone counts: nj[i] for i in [-NG, n1+NG) and, per row
    (i, j) with j in [-NG, nj[i]+NG), nk[i][j] (lists of lists, ghost rows included)."""
    raw = np.frombuffer(_ref_dump(pb, "grid"), dtype=np.int32)
    n1 = pb.n[0]
    nj = raw[:n1 + 4].tolist()
    nk, c = [], n1 + 4
    for i in range(n1 + 4):
        nk.append(raw[c:c + nj[i] + 4].tolist())
        c += nj[i] + 4
    return nj, nk


def reference_geometry(pb):
    """ref_get_geom records (64 doubles: volume, area[NDIM], gcov[0..NDIM][3], gcon[3],
    scale[0..NDIM][3], conn[27]) of zone (i, j, 0) for every row of reference_grid, in
    the same order."""
    return np.frombuffer(_ref_dump(pb, "geom"), dtype=np.float64).reshape(-1, 64).copy()


def time_reference_phases(pb, warmup: int, steps: int) -> dict:
    """The reference's own timers (TIMER_START/TIMER_STOP around step, estimate_dt,
    prim_to_fluxes1/2/3, push, reset_boundaries, ...) over `steps` steps after `warmup`,
    from the reftime_<cfg> build (its Makefile flags with DO_TIMING=TRUE) and the
    timing.csv it writes (io.c:51-108 columns).  Returns {"zone_updates_per_s", "seconds",
    "steps", "cells", "timers": {name: (total seconds, cycles)}}."""
    exe = os.path.join(REF_DIR, "reftime_" + ref_config(pb))
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        _write_input(pb, fin)
        r = subprocess.run([exe, "time", fin, str(warmup), str(steps)], check=True, cwd=td,
                           capture_output=True, text=True)
        rows = open(os.path.join(td, "timing.csv")).read().strip().splitlines()
    out = {}
    for tok in r.stdout.split():
        k, v = tok.split("=")
        out[k] = float(v)
    if rows[0].split(",") != ["timer", "time", "step", "ncycle", "max", "min", "avg"]:
        raise RuntimeError("unexpected timing.csv header: %r" % rows[0])
    out["timers"] = {}
    for row in rows[1:]:
        f = row.split(",")
        out["timers"][f[0]] = (float(f[4]), int(f[3]))
    return out


def time_reference(pb, warmup: int, steps: int, fast: bool = True) -> dict:
    """Time the reference's own build (its Makefile flags when fast=True) in a
    subprocess; returns zone_updates_per_s, seconds, steps, cells."""
    exe = os.path.join(REF_DIR, ("reffast_" if fast else "ref_") + ref_config(pb))
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        _write_input(pb, fin)
        r = subprocess.run([exe, "time", fin, str(warmup), str(steps)], check=True, cwd=td,
                           capture_output=True, text=True)
    out = {}
    for tok in r.stdout.split():
        k, v = tok.split("=")
        out[k] = float(v)
    return out
