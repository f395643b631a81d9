"""Host-side mirror of the reference's hot-path interface over the C ABI.

The reference drives its sweep with three global-state calls from main.c
(estimate_dt(), step(), update_cpu(); decs.h:754-757).  :class:`Solver` holds one or more
problems resident on the GPU and exposes the same operations:

=====================  ===================================================
reference              medusa_b200
=====================  ===================================================
main.c:129-165 upload  ``Solver(problems)`` + ``upload()`` (mdg_create/mdg_upload_state)
estimate_dt()          ``estimate_dt()``  (mdg_estimate_dt)
step(); t += dt        ``step(n)``        (mdg_step)
update_cpu()           ``update_cpu(m)``  (mdg_download_state)
=====================  ===================================================

Every call goes through libmedusa_b200.so; there is no CPU fallback.  If the library is
missing or the GPU is unavailable the constructor raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

from . import problems as _pb

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libmedusa_b200.so")

PREC_FP64 = 0
PREC_MIXED = 1


class MdgError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, code: int, where: str, msg: str):
        super().__init__("%s failed with status %d: %s" % (where, code, msg))
        self.code = code


class LaunchConfig(ctypes.Structure):
    """mdg_launch_config of include/medusa_b200.h."""
    _fields_ = [("threads", ctypes.c_int), ("ctas_per_sm", ctypes.c_int), ("steps_per_graph", ctypes.c_int),
                ("run_length", ctypes.c_int), ("lanes", ctypes.c_int), ("resident", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {"threads": self.threads, "ctas_per_sm": self.ctas_per_sm, "steps_per_graph": self.steps_per_graph,
                "run_length": self.run_length, "lanes": self.lanes, "resident": self.resident}


class ServerConfig(ctypes.Structure):
    """mdg_server_config of include/medusa_b200.h."""
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int), ("hbm_bytes", ctypes.c_longlong),
                ("max_problems", ctypes.c_int), ("max_zones", ctypes.c_int), ("steps_per_round", ctypes.c_int),
                ("threads", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("hbm_bytes_2d", ctypes.c_longlong), ("max_cells_2d", ctypes.c_int),
                ("hbm_bytes_3d", ctypes.c_longlong)]


class ServerStats(ctypes.Structure):
    """mdg_server_stats of include/medusa_b200.h."""
    _fields_ = [(n, ctypes.c_longlong) for n in ("submitted", "completed", "failed", "queued", "running", "rounds")] + \
               [(n, ctypes.c_double) for n in ("zone_updates", "device_seconds", "latency_p50", "latency_p99",
                                                "wait_p50", "wait_p99", "hbm_capacity", "hbm_in_use")] + \
               [("kernel_launches", ctypes.c_longlong)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class ProblemDesc(ctypes.Structure):
    """mdg_problem_desc of include/medusa_b200.h."""
    _fields_ = [("ndim", ctypes.c_int), ("geom", ctypes.c_int), ("eos", ctypes.c_int),
                ("n1", ctypes.c_int), ("n2", ctypes.c_int), ("n3", ctypes.c_int),
                ("startx", ctypes.c_double * 3), ("dx", ctypes.c_double * 3),
                ("gam", ctypes.c_double), ("Kpoly", ctypes.c_double),
                ("bc_lo", ctypes.c_int * 3), ("bc_hi", ctypes.c_int * 3),
                ("prob_kind", ctypes.c_int),
                ("cfl", ctypes.c_double), ("dt_init_safety", ctypes.c_double),
                ("dt_grow_safety", ctypes.c_double), ("initial_dt", ctypes.c_double),
                ("dtmax", ctypes.c_double), ("dtmin", ctypes.c_double), ("tmax", ctypes.c_double),
                ("hydro_interp_order", ctypes.c_int),
                ("enforce_floors", ctypes.c_int), ("rho_floor", ctypes.c_double), ("e_floor", ctypes.c_double),
                ("grav", ctypes.c_double * 3), ("rcoord", ctypes.c_int), ("rtrans", ctypes.c_double),
                ("rfact", ctypes.c_double * 3), ("thcoord", ctypes.c_int), ("poly_xt", ctypes.c_double),
                ("poly_alpha", ctypes.c_double), ("monopole", ctypes.c_int)]


def desc_of(pb: "_pb.Problem") -> ProblemDesc:
    d = ProblemDesc()
    d.ndim, d.geom, d.eos = pb.ndim, pb.geom, pb.eos
    d.n1, d.n2, d.n3 = pb.n
    for k in range(3):
        d.startx[k] = pb.startx[k]
        d.dx[k] = pb.dx[k]
        d.bc_lo[k] = pb.bc_lo[k]
        d.bc_hi[k] = pb.bc_hi[k]
    d.gam, d.Kpoly, d.prob_kind = pb.gam, pb.Kpoly, pb.prob_kind
    d.cfl, d.dt_init_safety, d.dt_grow_safety = pb.cfl, pb.dt_init_safety, pb.dt_grow_safety
    d.initial_dt, d.dtmax, d.dtmin, d.tmax = pb.initial_dt, pb.dtmax, pb.dtmin, pb.tmax
    d.hydro_interp_order = pb.hydro_interp_order
    d.enforce_floors, d.rho_floor, d.e_floor = int(pb.enforce_floors), pb.rho_floor, pb.e_floor
    for k in range(3):
        d.grav[k] = pb.grav[k]
    d.rcoord, d.rtrans = pb.rcoord, pb.rtrans
    for k in range(3):
        d.rfact[k] = pb.rfact[k]
    d.thcoord, d.poly_xt, d.poly_alpha = pb.thcoord, pb.poly_xt, pb.poly_alpha
    d.monopole = int(pb.monopole)
    return d


_lib = None


def library(path: str = _LIB_PATH) -> ctypes.CDLL:
    """Load libmedusa_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError("libmedusa_b200.so not built (run python -m medusa_b200.build): %s" % path)
    L = ctypes.CDLL(path)
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.mdg_create.argtypes = [ctypes.POINTER(ProblemDesc), i, i, i, ctypes.POINTER(vp)]
    L.mdg_upload_state.argtypes = [vp, i, vp]
    L.mdg_estimate_dt.argtypes = [vp, vp]
    L.mdg_step.argtypes = [vp, i]
    L.mdg_run_host.argtypes = [vp, i, vp, vp, i, ctypes.POINTER(ctypes.c_float)]
    L.mdg_estimate_dt_raw.argtypes = [vp, vp]
    L.mdg_step_dt.argtypes = [vp, vp]
    L.mdg_download_state.argtypes = [vp, i, vp, vp]
    L.mdg_get_time.argtypes = [vp, i, ctypes.POINTER(d), ctypes.POINTER(d), ctypes.POINTER(i)]
    L.mdg_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.mdg_set_time.argtypes = [vp, i, d, i]
    L.mdg_write_timers.argtypes = [vp, i, ctypes.c_char_p]
    L.mdg_restart_write.argtypes = [vp, i, ctypes.c_char_p]
    L.mdg_restart_read.argtypes = [vp, i, ctypes.c_char_p]
    L.mdg_synchronize.argtypes = [vp]
    L.mdg_destroy.argtypes = [vp]
    L.mdg_error_string.restype = ctypes.c_char_p
    L.mdg_error_string.argtypes = [i]
    L.mdg_last_error_message.restype = ctypes.c_char_p
    L.mdg_version.restype = i
    L.mdg_set_timing.argtypes = [vp, i]
    L.mdg_get_timers.argtypes = [vp, vp, vp]
    L.mdg_get_launch_config.argtypes = [vp, ctypes.POINTER(LaunchConfig)]
    L.mdg_set_launch_config.argtypes = [vp, ctypes.POINTER(LaunchConfig)]
    L.mdg_resident_cluster.argtypes = [vp, ctypes.POINTER(i)]
    L.mdg_autotune.argtypes = [vp, i, ctypes.POINTER(LaunchConfig), ctypes.POINTER(d)]
    L.mdg_conserved_totals.argtypes = [vp, vp, vp]
    L.mdg_upload_all.argtypes = [vp, vp]
    L.mdg_download_all.argtypes = [vp, vp]
    ll = ctypes.c_longlong
    L.mdg_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
    L.mdg_server_submit.argtypes = [vp, ctypes.POINTER(ProblemDesc), vp, ctypes.POINTER(ll)]
    L.mdg_server_run.argtypes = [vp, i, ctypes.POINTER(i)]
    L.mdg_server_start.argtypes = [vp]
    L.mdg_server_stop.argtypes = [vp]
    L.mdg_server_poll.argtypes = [vp, ll, ctypes.POINTER(i)]
    L.mdg_server_wait.argtypes = [vp, ll, d, ctypes.POINTER(i)]
    L.mdg_server_result.argtypes = [vp, ll, vp, ctypes.POINTER(d), ctypes.POINTER(i), ctypes.POINTER(d)]
    L.mdg_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
    L.mdg_server_destroy.argtypes = [vp]
    L.mdg_snapshot.argtypes = [vp, i]
    L.mdg_snapshot_read.argtypes = [vp, vp, vp, vp]
    L.mdg_snapshot_write_ascii1.argtypes = [vp, ctypes.c_char_p]
    L.mdg_dump_ascii1.argtypes = [vp, i, ctypes.c_char_p]
    L.mdg_grid3d_counts.argtypes = [ctypes.POINTER(ProblemDesc), vp, vp, ctypes.POINTER(ll)]
    L.mdg_grid3d_geometry.argtypes = [ctypes.POINTER(ProblemDesc), vp, ctypes.POINTER(ll)]
    for name in ("mdg_create", "mdg_upload_state", "mdg_estimate_dt", "mdg_step", "mdg_download_state",
                 "mdg_get_time", "mdg_get_stream", "mdg_synchronize", "mdg_destroy", "mdg_set_timing",
                 "mdg_get_timers", "mdg_get_launch_config", "mdg_set_launch_config", "mdg_autotune",
                 "mdg_conserved_totals", "mdg_upload_all", "mdg_download_all", "mdg_server_create", "mdg_server_submit", "mdg_server_run",
                 "mdg_server_start", "mdg_server_stop", "mdg_server_poll", "mdg_server_wait", "mdg_server_result",
                 "mdg_server_get_stats", "mdg_server_destroy", "mdg_grid3d_counts", "mdg_grid3d_geometry",
                 "mdg_snapshot", "mdg_snapshot_read", "mdg_snapshot_write_ascii1", "mdg_dump_ascii1"):
        getattr(L, name).restype = i
    _lib = L
    return L


GEO3_FIELDS = 42


def grid3d_counts(pb: "_pb.Problem"):
    """(nj[i] for the n1 radial rows, nk of every interior row (i, j) in zone order, zone
    count) of a dendritic spherical problem, 3-D or 2-D (mdg_grid3d_counts)."""
    d = desc_of(pb)
    n = ctypes.c_longlong()
    nj = np.zeros(pb.n[0], dtype=np.int32)
    _check(library().mdg_grid3d_counts(ctypes.byref(d), nj.ctypes.data, None, ctypes.byref(n)), "mdg_grid3d_counts")
    nk = np.zeros(int(nj.sum()), dtype=np.int32)
    _check(library().mdg_grid3d_counts(ctypes.byref(d), None, nk.ctypes.data, ctypes.byref(n)), "mdg_grid3d_counts")
    return nj, nk, n.value


def grid3d_geometry(pb: "_pb.Problem") -> np.ndarray:
    """Per-row zone geometry [rows, 42] of a dendritic spherical problem (3-D or 2-D), rows i in
    [-2, n1+2), j in [-2, nj[i]+2) (mdg_grid3d_geometry)."""
    d = desc_of(pb)
    n = ctypes.c_longlong()
    _check(library().mdg_grid3d_geometry(ctypes.byref(d), None, ctypes.byref(n)), "mdg_grid3d_geometry")
    out = np.zeros((n.value, GEO3_FIELDS))
    _check(library().mdg_grid3d_geometry(ctypes.byref(d), out.ctypes.data, ctypes.byref(n)), "mdg_grid3d_geometry")
    return out


def grid3d_zone_volumes(pb: "_pb.Problem") -> np.ndarray:
    """Volume of every interior zone of a dendritic (3-D or 2-D spherical) problem, in zone order."""
    nj, nk, n = grid3d_counts(pb)
    geo = grid3d_geometry(pb)
    n1 = pb.n[0]
    njx = [int(nj[1]), int(nj[0])] + [int(x) for x in nj] + [int(nj[-1])] * 2   # rows i = -2 .. n1+1
    vol = np.empty(n)
    r = c = q = 0
    for i in range(-2, n1 + 2):
        for j in range(-2, njx[i + 2] + 2):
            if 0 <= i < n1 and 0 <= j < nj[i]:
                vol[c:c + nk[q]] = geo[r, 0]
                c += int(nk[q])
                q += 1
            r += 1
    return vol


def grid3d_zone_gcov(pb: "_pb.Problem") -> np.ndarray:
    """Zone-centred metric diagonal gcov[0][0..2] of every interior zone of a dendritic
    (3-D or 2-D spherical) problem, in zone order, shape [zones, 3]."""
    nj, nk, n = grid3d_counts(pb)
    geo = grid3d_geometry(pb)
    n1 = pb.n[0]
    njx = [int(nj[1]), int(nj[0])] + [int(x) for x in nj] + [int(nj[-1])] * 2   # rows i = -2 .. n1+1
    out = np.empty((n, 3))
    r = c = q = 0
    for i in range(-2, n1 + 2):
        for j in range(-2, njx[i + 2] + 2):
            if 0 <= i < n1 and 0 <= j < nj[i]:
                out[c:c + nk[q], :] = geo[r, 4:7]
                c += int(nk[q])
                q += 1
            r += 1
    return out


def grid3d_radial_mean(pb: "_pb.Problem", field: np.ndarray) -> np.ndarray:
    """Volume-weighted mean of a zone field over each radial row of a dendritic problem."""
    nj, nk, n = grid3d_counts(pb)
    vol = grid3d_zone_volumes(pb)
    out = np.zeros(pb.n[0])
    c = q = 0
    for i in range(pb.n[0]):
        cnt = int(nk[q:q + nj[i]].sum())
        w = vol[c:c + cnt]
        out[i] = float(np.sum(field[c:c + cnt] * w) / np.sum(w))
        c += cnt
        q += int(nj[i])
    return out


def run_host(solvers, h_in, h_out, nsteps: int) -> float:
    """mdg_run_host: every solver uploads its host buffer h_in[i] (address of [zone][5]
    doubles of all its problems, page-locked for overlap), takes nsteps steps and downloads
    into h_out[i], the transfers of each overlapping the others' steps; returns the device
    milliseconds from the first upload to the last download."""
    n = len(solvers)
    L = library()
    arr = (ctypes.c_void_p * n)(*[s._h for s in solvers])
    ins = (ctypes.c_void_p * n)(*h_in)
    outs = (ctypes.c_void_p * n)(*h_out)
    ms = ctypes.c_float(0.0)
    _check(L.mdg_run_host(arr, n, ins, outs, nsteps, ctypes.byref(ms)), "mdg_run_host")
    return float(ms.value)


def _check(rc: int, where: str):
    if rc != 0:
        L = library()
        raise MdgError(rc, where, (L.mdg_last_error_message() or b"").decode())


class Solver:
    """Problems resident on one GPU, advanced together."""

    def __init__(self, problems: Sequence["_pb.Problem"], precision: int = PREC_FP64, device: int = 0,
                 upload: bool = True):
        if isinstance(problems, _pb.Problem):
            problems = [problems]
        self.problems = list(problems)
        L = library()
        arr = (ProblemDesc * len(self.problems))(*[desc_of(p) for p in self.problems])
        h = ctypes.c_void_p()
        _check(L.mdg_create(arr, len(self.problems), precision, device, ctypes.byref(h)), "mdg_create")
        self._h = h
        if upload:
            for m, p in enumerate(self.problems):
                self.upload(m, p.ic)

    def close(self):
        if getattr(self, "_h", None):
            library().mdg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- the reference's operations
    def upload(self, m: int, prim: np.ndarray):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        if prim.shape != (self.problems[m].ncell, 5):
            raise ValueError("state of problem %d must have shape (%d, 5)" % (m, self.problems[m].ncell))
        _check(library().mdg_upload_state(self._h, m, prim.ctypes.data), "mdg_upload_state")

    def upload_ptr(self, m: int, host_ptr: int):
        """Upload from a raw host pointer (e.g. pinned memory) laid out [zone][5]."""
        _check(library().mdg_upload_state(self._h, m, ctypes.c_void_p(host_ptr)), "mdg_upload_state")

    def upload_all_ptr(self, host_ptr: int):
        """Upload every problem's state from one host buffer (problems back to back, each
        [zone][5], e.g. pinned memory)."""
        _check(library().mdg_upload_all(self._h, ctypes.c_void_p(host_ptr)), "mdg_upload_all")

    def download_all_ptr(self, host_ptr: int):
        _check(library().mdg_download_all(self._h, ctypes.c_void_p(host_ptr)), "mdg_download_all")

    def download_all(self) -> list:
        """Every problem's state as a list of [zone][5] arrays."""
        n = [p.ncell for p in self.problems]
        buf = np.empty((sum(n), 5))
        self.download_all_ptr(buf.ctypes.data)
        out, o = [], 0
        for k in n:
            out.append(buf[o:o + k])
            o += k
        return out

    def estimate_dt(self) -> np.ndarray:
        out = np.zeros(len(self.problems))
        _check(library().mdg_estimate_dt(self._h, out.ctypes.data), "mdg_estimate_dt")
        return out

    def step(self, nsteps: int = 1):
        _check(library().mdg_step(self._h, int(nsteps)), "mdg_step")

    # --- for a host that runs the main.c time loop itself
    def estimate_dt_raw(self) -> np.ndarray:
        """What estimate_dt() leaves in the reference's dt, per problem (before main.c's
        safety, growth and clipping)."""
        out = np.zeros(len(self.problems))
        _check(library().mdg_estimate_dt_raw(self._h, out.ctypes.data), "mdg_estimate_dt_raw")
        return out

    def step_dt(self, dt):
        """One step() of every problem with the host's dt (scalar or one per problem)."""
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (len(self.problems),)))
        _check(library().mdg_step_dt(self._h, d.ctypes.data), "mdg_step_dt")

    def update_cpu(self, m: int = 0, with_eos: bool = False):
        n = self.problems[m].ncell
        prim = np.empty((n, 5))
        eos = np.empty((n, 5)) if with_eos else None
        _check(library().mdg_download_state(self._h, m, prim.ctypes.data,
                                            eos.ctypes.data if with_eos else None), "mdg_download_state")
        return (prim, eos) if with_eos else prim

    def download_ptr(self, m: int, host_ptr: int):
        _check(library().mdg_download_state(self._h, m, ctypes.c_void_p(host_ptr), None), "mdg_download_state")

    # --- output path
    def snapshot(self, m: int = 0):
        """Queue a copy of problem m's state, EOS records and time; returns at once."""
        self._snap_n = self.problems[m].ncell
        _check(library().mdg_snapshot(self._h, m), "mdg_snapshot")

    def snapshot_read(self):
        """(prim [zone][5], eos [zone][5], t) of the last snapshot (waits for it)."""
        n = getattr(self, "_snap_n", self.problems[0].ncell)
        prim, eos, t = np.empty((n, 5)), np.empty((n, 5)), ctypes.c_double()
        _check(library().mdg_snapshot_read(self._h, prim.ctypes.data, eos.ctypes.data, ctypes.byref(t)),
               "mdg_snapshot_read")
        return prim, eos, t.value

    def snapshot_write_ascii1(self, path: str):
        _check(library().mdg_snapshot_write_ascii1(self._h, str(path).encode()), "mdg_snapshot_write_ascii1")

    def dump_ascii1(self, path: str, m: int = 0):
        """Write problem m as the reference's dump_ascii1 (io.c:111-220) does."""
        self._snap_n = self.problems[m].ncell
        _check(library().mdg_dump_ascii1(self._h, m, str(path).encode()), "mdg_dump_ascii1")

    def time(self, m: int = 0):
        t, dt = ctypes.c_double(), ctypes.c_double()
        ist = ctypes.c_int()
        _check(library().mdg_get_time(self._h, m, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(ist)),
               "mdg_get_time")
        return t.value, dt.value, ist.value

    def synchronize(self):
        _check(library().mdg_synchronize(self._h), "mdg_synchronize")

    TIMER_NAMES = ("estimate_dt", "stage0", "stage1", "finish")

    def set_timing(self, enable: bool = True):
        _check(library().mdg_set_timing(self._h, int(bool(enable))), "mdg_set_timing")

    def timers(self) -> dict:
        ms = np.zeros(4)
        calls = np.zeros(4, dtype=np.int64)
        _check(library().mdg_get_timers(self._h, ms.ctypes.data, calls.ctypes.data), "mdg_get_timers")
        return {n: (float(ms[k]), int(calls[k])) for k, n in enumerate(self.TIMER_NAMES)}

    def write_timers(self, path: str, m: int = 0):
        """Append the timers to a CSV file in the reference's timing.csv columns."""
        _check(library().mdg_write_timers(self._h, int(m), os.fsencode(path)), "mdg_write_timers")

    # --- launch shape, autotuning and conservation diagnostics
    def launch_config(self) -> dict:
        c = LaunchConfig()
        _check(library().mdg_get_launch_config(self._h, ctypes.byref(c)), "mdg_get_launch_config")
        return c.as_dict()

    def set_launch_config(self, threads: int = None, ctas_per_sm: int = None, steps_per_graph: int = None,
                          run_length: int = None, lanes: int = None, resident: int = None):
        cur = self.launch_config()
        c = LaunchConfig(cur["threads"] if threads is None else threads,
                         cur["ctas_per_sm"] if ctas_per_sm is None else ctas_per_sm,
                         cur["steps_per_graph"] if steps_per_graph is None else steps_per_graph,
                         cur["run_length"] if run_length is None else run_length,
                         cur["lanes"] if lanes is None else lanes,
                         cur["resident"] if resident is None else resident)
        _check(library().mdg_set_launch_config(self._h, ctypes.byref(c)), "mdg_set_launch_config")

    def resident_cluster(self) -> int:
        """CTAs per problem of the resident stepper, 0 when mdg_step cannot use it."""
        n = ctypes.c_int()
        _check(library().mdg_resident_cluster(self._h, ctypes.byref(n)), "mdg_resident_cluster")
        return n.value

    def autotune(self, trial_steps: int = 5):
        """Pick the fastest launch shape (the mixed 1-D sweep's threads, persistent CTAs and
        lanes, a dendritic sweep's run length); returns (config, ms per step)."""
        c = LaunchConfig()
        ms = ctypes.c_double()
        _check(library().mdg_autotune(self._h, int(trial_steps), ctypes.byref(c), ctypes.byref(ms)), "mdg_autotune")
        return c.as_dict(), ms.value

    def set_time(self, m: int, t: float, istep: int):
        """The time record of a run resumed from a restart (mdg_set_time)."""
        _check(library().mdg_set_time(self._h, int(m), float(t), int(istep)), "mdg_set_time")

    def restart_write(self, path: str, m: int = 0):
        """Write problem m's restart file (state, t, step count)."""
        _check(library().mdg_restart_write(self._h, int(m), os.fsencode(path)), "mdg_restart_write")

    def restart_read(self, path: str, m: int = 0):
        """Resume problem m from a restart file."""
        _check(library().mdg_restart_read(self._h, int(m), os.fsencode(path)), "mdg_restart_read")

    def conserved_totals(self):
        """(mass, energy) arrays over the problems, compensated FP64 sums on the device."""
        n = len(self.problems)
        mass, energy = np.zeros(n), np.zeros(n)
        _check(library().mdg_conserved_totals(self._h, mass.ctypes.data, energy.ctypes.data),
               "mdg_conserved_totals")
        return mass, energy

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(library().mdg_get_stream(self._h, ctypes.byref(s)), "mdg_get_stream")
        return s.value or 0


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3


class Server:
    """Solve server (mdg_server_*): 1-D, 2-D and 3-D problems resident on one GPU, admitted
    by their device-memory footprint and advanced together; each request runs to its end
    time (the problem's tmax).  2-D requests need hbm_bytes_2d > 0, 3-D requests
    hbm_bytes_3d > 0."""

    def __init__(self, precision: int = PREC_MIXED, device: int = 0, hbm_bytes: int = 2 << 30,
                 max_problems: int = 4096, max_zones: int = 16384, steps_per_round: int = 20,
                 threads: int = 64, ctas_per_sm: int = 0, hbm_bytes_2d: int = 0, max_cells_2d: int = 1 << 20,
                 hbm_bytes_3d: int = 0):
        L = library()
        c = ServerConfig(device, precision, int(hbm_bytes), max_problems, max_zones, steps_per_round, threads,
                         ctas_per_sm, int(hbm_bytes_2d), int(max_cells_2d), int(hbm_bytes_3d))
        h = ctypes.c_void_p()
        _check(L.mdg_server_create(ctypes.byref(c), ctypes.byref(h)), "mdg_server_create")
        self._h = h
        self._n = {}

    def close(self):
        if getattr(self, "_h", None):
            library().mdg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, pb: "_pb.Problem") -> int:
        ic = np.ascontiguousarray(pb.ic, dtype=np.float64)
        d = desc_of(pb)
        rid = ctypes.c_longlong()
        _check(library().mdg_server_submit(self._h, ctypes.byref(d), ic.ctypes.data, ctypes.byref(rid)),
               "mdg_server_submit")
        self._n[rid.value] = pb.ncell
        return rid.value

    def run(self, rounds: int = 0) -> int:
        act = ctypes.c_int()
        _check(library().mdg_server_run(self._h, int(rounds), ctypes.byref(act)), "mdg_server_run")
        return act.value

    def start(self):
        _check(library().mdg_server_start(self._h), "mdg_server_start")

    def stop(self):
        _check(library().mdg_server_stop(self._h), "mdg_server_stop")

    def poll(self, rid: int) -> int:
        st = ctypes.c_int()
        _check(library().mdg_server_poll(self._h, rid, ctypes.byref(st)), "mdg_server_poll")
        return st.value

    def wait(self, rid: int, timeout: float = 60.0) -> int:
        st = ctypes.c_int()
        _check(library().mdg_server_wait(self._h, rid, float(timeout), ctypes.byref(st)), "mdg_server_wait")
        return st.value

    def result(self, rid: int):
        """(final state [zone][5], t, steps, seconds from submission to completion)."""
        prim = np.empty((self._n[rid], 5))
        t, lat = ctypes.c_double(), ctypes.c_double()
        ist = ctypes.c_int()
        _check(library().mdg_server_result(self._h, rid, prim.ctypes.data, ctypes.byref(t), ctypes.byref(ist),
                                           ctypes.byref(lat)), "mdg_server_result")
        del self._n[rid]
        return prim, t.value, ist.value, lat.value

    def stats(self) -> dict:
        st = ServerStats()
        _check(library().mdg_server_get_stats(self._h, ctypes.byref(st)), "mdg_server_get_stats")
        return st.as_dict()

