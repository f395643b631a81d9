"""Benchmark of the hydro sweep: zone-updates/s, batched mixed precision vs plain FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ensemble|kh2048|server|sedov3d|sod1d|eos] [--no-cpu-baseline]

A step is one full RK2 step of the reference time loop (estimate_dt + both stages +
t += dt) of every problem of the workload; the metric is zone-updates/s (zones x steps /
seconds), whole job over all ranks.

Workload "ensemble" (default): 2048 independent 1-D spherical problems, zone counts
log-uniform in [128, 8192] (4.0 M zones), Sod/Noh/Sedov initial states with seeded
density and pressure ratios and gamma in {4/3, 1.4, 5/3}
(medusa_b200.problems.ensemble_1d, seed 7 + rank).  The headline runs them all in one
solver with the mixed-precision sweep (FP32 reconstruction/Riemann, FP64 state, fluxes,
sources, update and dt), launch shape chosen by the autotuner, each step's launches
replayed from a CUDA graph.  Beside it, measured in the same run:
  - the same ensemble batched through the plain FP64 sweep;
  - the plain FP64 sweep run one problem at a time (a sample of 64 problems, each in its
    own solver, back to back), the baseline of the >= 3x target;
  - accuracy of the mixed result against the plain FP64 result at the same physical time:
    volume-weighted relative L1 of density and internal energy, mass and total-energy
    differences (compensated sums), per problem kind; beside it the FP64 result's own
    sensitivity floor (the same FP64 run with its CFL number scaled by 1 + 1e-7) and, for
    the Noh problems, the FP64 path's L1 error against the analytic solution.
Workload "kh2048": 2-D Kelvin-Helmholtz 2048 x 2048, plain FP64, gamma 5/3, CFL 0.8.
Workloads "server" (the solve server under seeded request streams), "sedov3d" (3-D Sedov
on the dendritic grid), "sod1d" (the 1024-zone Sod job, timed whole) and "eos" (the
tabulated nuclear EOS zone update over 8 M zones of a synthetic table of the reference's
sizes; metric zone EOS updates/s) are described at their functions.

- value:  device time of K steps with the state resident in HBM, CUDA events on the
          solver's stream, barrier + synchronize on both sides, max over ranks.  The
          ensemble state (2 x 160 MB) and the KH state (2 x 168 MB) exceed the 126 MB L2,
          so no L2 flush is needed.
- e2e:    the same metric through the public API with host buffers: upload of every
          initial state from pinned memory, K steps, download of every final state to
          pinned memory, all inside the timed region.
- roofline: the dominant kernel (second RK stage) against the measured HBM copy
          bandwidth; algorithmic bytes per zone-update B_alg = 240 NDIM - 40
          (1-D 200 B, 2-D 440 B), of which the second stage accounts for 120 B (1-D) /
          240 B (2-D).
- cpu_baseline: the reference's own CPU build (its Makefile flags) on a bounded sample
          of the same workload (ensemble: problem-parallel over the host's cores).
With --gpus N > 1 (torchrun) every rank runs its own workload (ensemble: seed 7 + rank;
KH: a replica); there is no collective on the data path.
--impl reference times the reference's CPU implementation instead (rank 0 only).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = 2048
ENSEMBLE_COUNT = 2048
ENSEMBLE_SEED = 7
# geometry-table bytes the plain FP64 1-D stage kernel reads per zone: 19 of the 22
# reconstruction coefficients (the linear-reconstruction ones are not read) and 22 face and
# zone geometry fields (area, scale, 3 face gcov, 3 zone gcov, 3 gcon, volume, scale[0][0],
# 9 connection coefficients)
FP64_1D_TABLE_BYTES = 8 * (19 + 22)
FALLBACK_HBM_GBS = 6650.0


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def read_profile_value(name, key):
    """A number recorded as '<key> <value>' in a committed ncu summary under profiles/."""
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            if line.startswith(key + " "):
                return float(line.split()[1])
    except Exception:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(backend=None):
    """(world, rank, local rank, torch.distributed or None) from the torchrun environment;
    NCCL by default (MDG_DIST_BACKEND=gloo runs the same rank logic on CPU)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = backend or os.environ.get("MDG_DIST_BACKEND", "nccl")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        return world, rank, local, dist
    return 1, 0, 0, None


class Ctx:
    """Rank bookkeeping: barrier, max over ranks of a device time and sums of the units
    each rank processed (every rank calls these in the same order)."""

    def __init__(self, world, rank, local, dist):
        self.world, self.rank, self.local, self.dist = world, rank, local, dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def _reduce(self, x, op):
        import torch
        dev = "cuda" if self.dist.get_backend() == "nccl" else "cpu"
        tt = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(tt, op=op)
        return float(tt.item())

    def max_ms(self, ms):
        if self.dist is None:
            return ms
        return self._reduce(ms, self.dist.ReduceOp.MAX)

    def total(self, x):
        """Sum over ranks (the whole job's units: zones, zone-updates/s of independent servers)."""
        if self.dist is None:
            return x
        return self._reduce(x, self.dist.ReduceOp.SUM)


def warm_up(solver, W):
    """W untimed steps, then one CUDA graph's worth more, so that the graph the timed
    steps replay is captured and instantiated before the timed region."""
    solver.step(W)
    g = solver.launch_config().get("steps_per_graph", 0)
    if g > 0:
        solver.step(g)


def timed_steps(ctx, solver, K, sample_clocks=False):
    """Device time (ms, max over ranks) of K steps on the solver's stream."""
    import torch
    stream = torch.cuda.ExternalStream(solver.stream, device=ctx.local)
    sampler = ClockSampler(ctx.local) if sample_clocks else None
    if sampler:
        sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ctx.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    solver.step(K)
    e1.record(stream)
    e1.synchronize()
    solver.synchronize()
    ctx.barrier()
    clocks = sampler.stop() if sampler else None
    return ctx.max_ms(e0.elapsed_time(e1)), clocks


def stage_times(solver, nsteps):
    """Per-step device time of each RK stage from the library's event timers, each stage
    one launch over all problems (lanes set to 1 for the measurement: the roofline is the
    kernel's, whatever the scheduling of the timed run)."""
    cfg = solver.launch_config()
    if cfg.get("lanes", 1) != 1:
        solver.set_launch_config(lanes=1)
    solver.set_timing(True)
    solver.step(nsteps)
    solver.synchronize()
    tm = solver.timers()
    solver.set_timing(False)
    if cfg.get("lanes", 1) != 1:
        solver.set_launch_config(lanes=cfg["lanes"])
    return ({k: tm[k][0] / max(1, tm[k][1]) for k in ("stage0", "stage1", "estimate_dt", "finish")})


def run_to_times(ctx, problems, t_end, precision, nsteps, cfg):
    """A solver over `problems` whose end times are t_end, stepped until every problem
    has reached its end time (a problem that reaches it stays there: dt = dtmin);
    returns (solver, steps beyond nsteps, largest relative time mismatch)."""
    from medusa_b200.solver import Solver
    s = Solver([pb.copy(tmax=te) for pb, te in zip(problems, t_end)], precision=precision, device=ctx.local)
    if cfg:
        s.set_launch_config(**cfg)
    s.step(nsteps)
    extra = 0
    while True:
        t_now = [s.time(m)[0] for m in range(len(problems))]
        if all(tn >= te * (1.0 - 1.0e-12) for tn, te in zip(t_now, t_end)) or extra >= 20 * nsteps:
            break
        s.step(20)
        extra += 20
    return s, extra, max(abs(tn - te) / te for tn, te in zip(t_now, t_end))


def e2e_run(ctx, make_solver, problems, K, W):
    """Upload every state from pinned host memory, K steps, download every state, all in
    the timed region; returns (ms, h2d bytes, d2h bytes)."""
    import numpy as np
    import torch
    offs = np.cumsum([0] + [p.ncell for p in problems])
    host = np.concatenate([np.ascontiguousarray(p.ic, dtype=np.float64) for p in problems])
    h_in = torch.from_numpy(host).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    s = make_solver(upload=False)
    stream = torch.cuda.ExternalStream(s.stream, device=ctx.local)
    row = 5 * 8
    s.upload_all_ptr(h_in.data_ptr())
    warm_up(s, W)
    s.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    ctx.barrier()
    torch.cuda.synchronize()
    f0.record(stream)
    s.upload_all_ptr(h_in.data_ptr())     # every problem's state in one copy
    s.step(K)
    s.download_all_ptr(h_out.data_ptr())
    f1.record(stream)
    f1.synchronize()
    ctx.barrier()
    ms = ctx.max_ms(f0.elapsed_time(f1))
    s.close()
    nbytes = int(offs[-1]) * row
    return ms, nbytes, nbytes


def e2e_run_overlapped(ctx, make_solver, problems, K, W, groups=4):
    """The public API's overlapped host path (mdg_run_host): the problems split into
    `groups` solvers of about equal zone count, each uploading its states from pinned host
    memory, taking K steps and downloading its final states on its own stream, the copies
    of each overlapping the others' steps.  Device time from the first upload to the last
    download (CUDA events inside mdg_run_host), max over ranks; (ms, h2d bytes, d2h bytes,
    solvers)."""
    import numpy as np
    import torch
    from medusa_b200.solver import run_host
    sizes = np.array([p.ncell for p in problems], dtype=np.int64)
    cut = np.searchsorted(np.cumsum(sizes), np.arange(1, groups) * sizes.sum() / groups)
    bounds = [0] + [int(c) + 1 for c in cut] + [len(problems)]
    parts = [problems[a:b] for a, b in zip(bounds[:-1], bounds[1:]) if b > a]
    solvers, h_in, h_out = [], [], []
    for part in parts:
        host = np.concatenate([np.ascontiguousarray(p.ic, dtype=np.float64) for p in part])
        h_in.append(torch.from_numpy(host).pin_memory())
        h_out.append(torch.empty_like(h_in[-1]).pin_memory())
        s = make_solver(part, upload=False)
        s.upload_all_ptr(h_in[-1].data_ptr())
        warm_up(s, W)
        solvers.append(s)
    for s in solvers:
        s.synchronize()
    ctx.barrier()
    torch.cuda.synchronize()
    ms = run_host(solvers, [t.data_ptr() for t in h_in], [t.data_ptr() for t in h_out], K)
    ctx.barrier()
    ms = ctx.max_ms(ms)
    for s in solvers:
        s.close()
    nbytes = int(sizes.sum()) * 5 * 8
    return ms, nbytes, nbytes, len(parts)


# ----------------------------------------------------------------------------- CPU side
def cpu_baseline_kh(pb_full, steps=2):
    """Reference CPU build (Makefile flags) on a bounded sample: `steps` RK2 steps of the
    full grid, single core (the reference's hot path has no host threading)."""
    from oracle import pyoracle
    if pyoracle.ref_available(pb_full, fast=True):
        r = pyoracle.time_reference(pb_full, 0, steps, fast=True)
        return {"value": r["zone_updates_per_s"], "unit": "zone-updates/s", "cores": 1,
                "kind": "reference",
                "sample": "%d RK2 steps of the %dx%d grid, reference build with its own flags "
                          "(-O3 -ffast-math), 1 core, %.1f s" % (steps, NX, NX, r["seconds"])}
    o = pyoracle.Oracle(pb_full)
    t0 = time.perf_counter()
    o.advance(1)
    el = time.perf_counter() - t0
    return {"value": pb_full.ncell / el, "unit": "zone-updates/s", "cores": 1, "kind": "port",
            "sample": "1 RK2 step of the %dx%d grid, CPU oracle, 1 core, %.1f s" % (NX, NX, el)}


def cpu_baseline_ensemble(problems, steps=20, warm=2, min_wall=10.0, zu_round=1.5e8):
    """The reference CPU build on the ensemble's problems as independent single-threaded
    processes over all host cores (the reference has no host threading on this path;
    problem-parallel is its best use of the host): every problem (or every n-th, so that
    one round is about zu_round zone-updates) runs `steps` timed RK2 steps (the GPU arm's
    step count, at most 200) after `warm` untimed ones; rounds repeat until at least
    min_wall seconds of wall time have passed.  Rate = timed zone-updates / (summed timed
    seconds / processes), i.e. perfect packing of the processes (the reference's best
    case).  Both the GPU arm's cpu_baseline and the --impl reference line use this."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import pyoracle
    steps = max(2, min(int(steps), 200))
    total = sum(p.ncell for p in problems) * steps
    every = max(1, int(math.ceil(total / zu_round)))
    sample = problems[::every]
    procs = os.cpu_count() or 1
    if pyoracle.ref_available(sample[0], fast=True):
        kind = "reference"

        def job(pb):
            r = pyoracle.time_reference(pb, warm, steps, fast=True)
            return r["cells"] * r["steps"], r["seconds"]
    else:
        kind = "port"

        def job(pb):
            o = pyoracle.Oracle(pb)
            o.advance(warm)
            t0 = time.perf_counter()
            o.advance(steps)
            return pb.ncell * steps, time.perf_counter() - t0
    t0 = time.perf_counter()
    zu = busy = 0.0
    rounds = 0
    with ThreadPoolExecutor(max_workers=procs) as ex:
        while rounds == 0 or time.perf_counter() - t0 < min_wall:
            res = list(ex.map(job, sample))
            zu += sum(r[0] for r in res)
            busy += sum(r[1] for r in res)
            rounds += 1
    wall = time.perf_counter() - t0
    return {"value": zu / (busy / procs), "unit": "zone-updates/s", "cores": procs, "kind": kind,
            "sample": "%d of the %d problems (every %dth), %d timed RK2 steps each after %d warm-up, %d round(s), "
                      "%d concurrent single-threaded processes, %s build%s; %.1f s wall, %.3g zone-updates"
                      % (len(sample), len(problems), every, steps, warm, rounds, procs, kind,
                         " with its own flags (-O3 -ffast-math)" if kind == "reference" else "", wall, zu)}


def run_reference_arm(args, ctx):
    from medusa_b200 import problems as P
    if ctx.rank != 0:
        return
    if args.workload == "sod1d":
        # the whole C1 job: its step count from the CPU restatement (bit-identical to the
        # reference), then the reference build timed over exactly those steps
        from oracle import pyoracle
        pb = P.sod(1024).copy(cfl=0.8, tmax=0.2)
        o = pyoracle.Oracle(pb)
        nsteps = 0
        while o.t < pb.tmax and nsteps < 10000:
            o.advance(1)
            nsteps += 1
        r = pyoracle.time_reference(pb, 0, nsteps, fast=True)
        cb = {"value": r["zone_updates_per_s"], "unit": "zone-updates/s", "cores": 1, "kind": "reference",
              "sample": "the whole job (%d RK2 steps to t = 0.2), reference build with its own flags "
                        "(-O3 -ffast-math), 1 core, %.3f s" % (nsteps, r["seconds"])}
        config = {"workload": "sod_1d_cartesian_1024_to_t0.2_fp64", "global_batch": 1, "seq_len": 1024,
                  "parallelism": "replicas", "l2": "resident in L2 (80 KB state)"}
        dtype = "f64"
    elif args.workload == "sedov3d":
        cb = cpu_baseline_sedov3d(steps=max(1, min(args.steps, 2)), radius=args.sedov3d_radius)
        config = {"workload": sedov3d_workload_name(SEDOV3D, args.sedov3d_radius), "global_batch": 1,
                  "seq_len": sedov3d_problem(SEDOV3D, args.sedov3d_radius).ncell, "parallelism": "replicas",
                  "l2": "inputs larger than L2"}
        dtype = "f64"
    elif args.workload == "kh2048":
        pb = P.kelvin_helmholtz(NX)
        cb = cpu_baseline_kh(pb, steps=max(1, min(args.steps, 2)))
        config = {"workload": "kelvin_helmholtz_2d_%dx%d_fp64" % (NX, NX), "global_batch": 1,
                  "seq_len": NX * NX, "parallelism": "replicas", "l2": "inputs larger than L2"}
        dtype = "f64"
    elif args.workload == "server":
        from medusa_b200 import loadgen
        probs = loadgen.request_stream(args.server_requests, seed=11, frac_2d=args.server_frac_2d,
                                       frac_3d=args.server_frac_3d)
        cb = cpu_baseline_ensemble(probs, steps=args.steps)
        config = {"workload": server_workload_name(args), "requests": len(probs)}
        dtype = "f64"
    elif args.workload == "eos":
        cb = cpu_baseline_eos()
        config = {"workload": "tabulated_eos_given_rex_%dM_zones_table_16x50x300x300" % (EOS_ZONES >> 20),
                  "global_batch": 1, "seq_len": EOS_ZONES, "parallelism": "replicas"}
        line = {"metric": "zone EOS updates/s", "value": cb["value"], "unit": "zone EOS updates/s",
                "n_gpus": ctx.world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": config, "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "zone EOS updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    else:
        probs = P.ensemble_1d(args.ensemble_count, seed=ENSEMBLE_SEED)
        cb = cpu_baseline_ensemble(probs, steps=args.steps)
        config = ensemble_config(probs, 1)
        dtype = "f64"
    line = {"metric": "zone-updates/s", "value": cb["value"], "unit": "zone-updates/s", "n_gpus": ctx.world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic", "impl": "reference",
            "config": config, "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- workloads
def ensemble_config(problems, world):
    ncell = sum(p.ncell for p in problems)
    return {"workload": "ensemble_1d_spherical_%d_problems_128_8192_zones" % len(problems),
            "global_batch": world * len(problems), "seq_len": ncell,
            "parallelism": "problem-parallel, no collective" if world > 1 else "single",
            "kinds": "Sod/Noh/Sedov, rho ratio 2-100, p ratio 2-1e4, gamma 4/3|1.4|5/3",
            "l2": "inputs larger than L2 (state 2 x %.0f MB)" % (ncell * 40 / 1e6)}


def run_ensemble(args, ctx):
    import numpy as np
    from medusa_b200 import analytic as A
    from medusa_b200 import problems as P
    from medusa_b200.solver import PREC_FP64, PREC_MIXED, Solver

    K, W = args.steps, args.warmup
    probs = P.ensemble_1d(args.ensemble_count, seed=ENSEMBLE_SEED + ctx.rank)
    ncell = sum(p.ncell for p in probs)
    ncell_all = ctx.total(ncell)   # each rank advances its own ensemble
    NT = 10   # timer-instrumented steps (roofline)

    # ---- headline: batched mixed precision, autotuned, CUDA graphs
    mix = Solver(probs, precision=PREC_MIXED, device=ctx.local)
    if args.launch:
        th, cps = (int(x) for x in args.launch.split(","))
        mix.set_launch_config(threads=th, ctas_per_sm=cps)
        tuned, tune_ms = mix.launch_config(), None
    else:
        tuned, tune_ms = mix.autotune(trial_steps=10)
    warm_up(mix, W)
    mix.synchronize()
    ms_mix, clocks = timed_steps(ctx, mix, K, sample_clocks=True)
    value = ncell_all * K / (ms_mix / 1e3)
    st_mix = stage_times(mix, NT)

    # ---- the same ensemble batched through the plain FP64 sweep (same step count)
    f64 = Solver(probs, precision=PREC_FP64, device=ctx.local)
    warm_up(f64, W)
    f64.synchronize()
    ms_f64, _ = timed_steps(ctx, f64, K)
    st_f64 = stage_times(f64, NT)

    mix.close()

    # ---- accuracy at equal physical time: each problem's time after W + K + NT plain FP64
    # steps is its end time for a fresh mixed run (whose last step lands on it) and for a
    # plain FP64 run with the CFL number scaled by 1 + 1e-7, the FP64 result's own
    # sensitivity to a perturbation at FP32 resolution
    t_end = [f64.time(m)[0] for m in range(len(probs))]
    acc, extra, t_mis = run_to_times(ctx, probs, t_end, PREC_MIXED, W + K + NT, tuned)
    ref2, _, _ = run_to_times(ctx, [pb.copy(cfl=pb.cfl * (1.0 + 1.0e-7)) for pb in probs], t_end, PREC_FP64,
                              W + K + NT, None)
    kinds = ("sod", "noh", "sedov")
    st = {k: {"l1_rho": [], "l1_u": [], "floor_rho": [], "mass": [], "energy": [], "trunc": []} for k in kinds}
    mm, em = acc.conserved_totals()
    mf, ef = f64.conserved_totals()
    for m, pb in enumerate(probs):
        a = acc.update_cpu(m)
        b = f64.update_cpu(m)
        c = ref2.update_cpu(m)
        w = A.spherical_volumes(pb.n[0])
        d = st[[k for k in kinds if "_" + k + "_" in pb.name][0]]
        d["l1_rho"].append(A.l1_rel(a[:, 0], b[:, 0], w))
        d["l1_u"].append(A.l1_rel(a[:, 1], b[:, 1], w))
        d["floor_rho"].append(A.l1_rel(c[:, 0], b[:, 0], w))
        d["mass"].append(abs(mm[m] - mf[m]) / abs(mf[m]))
        d["energy"].append(abs(em[m] - ef[m]) / abs(ef[m]))
        if "noh" in pb.name:
            r = (np.arange(pb.n[0]) + 0.5) * pb.dx[0]
            d["trunc"].append(A.l1_rel(b[:, 0], A.noh_spherical(r, t_end[m], pb.gam)[:, 0], w))
    acc.close()
    ref2.close()
    f64.close()

    def mm_(v):
        v = np.asarray(v, dtype=np.float64)
        return {"median": float(np.median(v)), "max": float(np.max(v))} if v.size else None

    accuracy = {"compared_at": "equal physical time: each problem's time after %d plain FP64 steps "
                               "(mixed: %d + %d steps, last step landing on that time; max relative time "
                               "mismatch %.1e)" % (W + K + NT, W + K + NT, extra, t_mis),
                "fp64_floor": "plain FP64 with CFL x (1 + 1e-7), same end times"}
    for k in kinds:
        d = st[k]
        e = {"count": len(d["l1_rho"]), "l1_rho_mixed_vs_fp64": mm_(d["l1_rho"]),
             "l1_u_mixed_vs_fp64": mm_(d["l1_u"]), "l1_rho_fp64_floor": mm_(d["floor_rho"]),
             "mass_drift_vs_fp64": mm_(d["mass"]), "energy_drift_vs_fp64": mm_(d["energy"])}
        if d["trunc"]:
            e["l1_rho_fp64_vs_analytic"] = mm_(d["trunc"])
            e["mixed_over_truncation"] = mm_(np.asarray(d["l1_rho"]) / np.asarray(d["trunc"]))
            e["fp64_floor_over_truncation"] = mm_(np.asarray(d["floor_rho"]) / np.asarray(d["trunc"]))
        accuracy[k] = e

    # ---- one problem at a time through the plain FP64 sweep (every 32nd problem)
    import torch
    sample = probs[::32]
    K1 = min(K, 100)
    ms_one, zu_one = 0.0, 0
    for pb in sample:
        s = Solver(pb, precision=PREC_FP64, device=ctx.local)
        warm_up(s, W)
        s.synchronize()
        stream = torch.cuda.ExternalStream(s.stream, device=ctx.local)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step(K1)
        e1.record(stream)
        e1.synchronize()
        ms_one += e0.elapsed_time(e1)
        zu_one += pb.ncell * K1
        s.close()
    one_rate = zu_one / (ms_one / 1e3)

    # ---- e2e through the public API with host buffers: the overlapped host path
    # (mdg_run_host, the ensemble in four solvers), and beside it one solver whose upload,
    # steps and download run back to back
    def make_part(part, upload):
        s = Solver(part, precision=PREC_MIXED, device=ctx.local, upload=upload)
        s.set_launch_config(**tuned)
        return s
    ms_e2e, h2d, d2h, ngroups = e2e_run_overlapped(ctx, make_part, probs, K, W)
    e2e = ncell_all * K / (ms_e2e / 1e3)
    ms_e2e1, _, _ = e2e_run(ctx, lambda upload: make_part(probs, upload), probs, K, W)

    if ctx.rank != 0:
        return
    peak, peak_kind = read_peaks()
    b_stage1 = 120.0   # 1-D second stage: read stage state + base state, write new state
    achieved = b_stage1 * ncell / (st_mix["stage1"] / 1e3) / 1e9
    traffic = read_profile_value("stage1d_mixed_ensemble_ncu.md", "TRAFFIC_PER_LAUNCH_STAGE1_BYTES")
    line = {
        "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s",
        "n_gpus": ctx.world, "steps": K, "warmup": W, "ms_per_step": ms_mix / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": ensemble_config(probs, ctx.world),
        "precision": "mixed: FP32 reconstruction/limiting/Riemann, FP64 state/fluxes/sources/update/dt",
        "launch": dict(tuned, autotune_ms_per_step=tune_ms),
        # per step and lane: dt, the two stage kernels, the time update
        "gpu_launches": 4 * K * tuned.get("lanes", 1),
        "e2e": {"value": e2e, "unit": "zone-updates/s", "h2d_bytes_per_step": h2d / K,
                "d2h_bytes_per_step": d2h / K,
                "timed": "mdg_run_host: upload of all %d initial states (pinned H2D) + %d steps + download of "
                         "all final states (pinned D2H), the ensemble in %d solvers whose copies overlap each "
                         "other's steps" % (len(probs), K, ngroups),
                "ms": ms_e2e,
                "one_solver": {"value": ncell_all * K / (ms_e2e1 / 1e3), "ms": ms_e2e1,
                               "timed": "one solver: upload, %d steps, download back to back" % K}},
        "comparison": {
            "fp64_batched": {"value": ncell_all * K / (ms_f64 / 1e3), "ms_per_step": ms_f64 / K,
                             "stage_ms": st_f64},
            "fp64_one_at_a_time": {"value": one_rate, "sample": "%d problems (every 32nd), %d steps "
                                                                "each, one solver at a time" % (len(sample), K1)},
            "mixed_over_fp64_one_at_a_time": value / (ctx.world * one_rate),
            "mixed_over_fp64_batched": ms_f64 / ms_mix,
        },
        "accuracy": accuracy,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "stage1d_mixed_kernel<%d,1> (second RK stage)" % tuned["threads"],
                     "kernel_ms": st_mix["stage1"], "stage0_ms": st_mix["stage0"],
                     "algorithmic_bytes_per_zone": b_stage1,
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"},
        "clocks": clocks,
    }
    # the batched plain FP64 sweep against the same roofline: its second-stage kernel, the
    # 120 B/zone of the state accounting, and beside it the bytes it really needs per zone
    # with the geometry tables the reference's Romberg geometry requires (19 reconstruction
    # coefficients and 22 face/zone geometry fields of 8 B, read once per zone)
    fp64_ms = st_f64["stage1"]
    fp64_ach = b_stage1 * ncell / (fp64_ms / 1e3) / 1e9
    line["roofline_fp64"] = {
        "bound": "hbm", "achieved": fp64_ach, "peak": peak, "unit": "GB/s", "frac": fp64_ach / peak,
        "kernel": "stage1d_kernel<1> (plain FP64 second RK stage)", "kernel_ms": fp64_ms,
        "stage0_ms": st_f64["stage0"], "algorithmic_bytes_per_zone": b_stage1,
        "table_bytes_per_zone": FP64_1D_TABLE_BYTES,
        "achieved_with_tables": (b_stage1 + FP64_1D_TABLE_BYTES) * ncell / (fp64_ms / 1e3) / 1e9,
        "traffic": read_profile_value("stage1d_fp64_ensemble_ncu.md", "TRAFFIC_PER_LAUNCH_STAGE1_BYTES"),
        "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"}
    if not args.no_cpu_baseline:
        cb = cpu_baseline_ensemble(probs, steps=K)
        line["cpu_baseline"] = cb
        fp64_rate = ncell_all * K / (ms_f64 / 1e3)
        line["comparison"]["fp64_batched_over_cpu_reference"] = fp64_rate / cb["value"]
        line["comparison"]["mixed_over_cpu_reference"] = value / cb["value"]
    print(json.dumps(line), flush=True)


def run_kh(args, ctx):
    import medusa_b200
    from medusa_b200 import problems as P

    K, W = args.steps, args.warmup
    pb = P.kelvin_helmholtz(NX)
    ncell = pb.ncell
    s = medusa_b200.Solver(pb, device=ctx.local)
    warm_up(s, W)
    s.synchronize()
    ms, clocks = timed_steps(ctx, s, K, sample_clocks=True)
    value = ctx.world * ncell * K / (ms / 1e3)
    st = stage_times(s, min(K, 20))
    s.close()
    ms_e2e, h2d, d2h = e2e_run(ctx, lambda upload: medusa_b200.Solver(pb, device=ctx.local, upload=upload),
                               [pb], K, W)
    e2e = ctx.world * ncell * K / (ms_e2e / 1e3)
    # the mixed-precision split sweep on the same grid, and its accuracy at equal time
    from medusa_b200 import analytic as A
    from medusa_b200.solver import PREC_MIXED
    sm = medusa_b200.Solver(pb, precision=PREC_MIXED, device=ctx.local)
    warm_up(sm, W)
    sm.synchronize()
    ms_mix, _ = timed_steps(ctx, sm, K)
    sm.close()
    nacc = min(K, 50)
    with medusa_b200.Solver(pb, device=ctx.local) as sf:
        sf.step(nacc)
        ref = sf.update_cpu(0)
        t_end = sf.time(0)[0]
        m0, e0 = sf.conserved_totals()
    with medusa_b200.Solver(pb.copy(tmax=t_end), precision=PREC_MIXED, device=ctx.local) as sa:
        n_mix = 0
        while sa.time(0)[0] < t_end * (1.0 - 1.0e-12) and n_mix < 4 * nacc:
            sa.step(10)
            n_mix += 10
        mix = sa.update_cpu(0)
        m1, e1 = sa.conserved_totals()
    accuracy = {"steps": nacc, "t": t_end, "l1_rho": A.l1_rel(mix[:, 0], ref[:, 0]),
                "l1_u": A.l1_rel(mix[:, 1], ref[:, 1]),
                "mass_drift_vs_fp64": abs(m1[0] - m0[0]) / m0[0], "energy_drift_vs_fp64": abs(e1[0] - e0[0]) / e0[0]}
    if ctx.rank != 0:
        return
    peak, peak_kind = read_peaks()
    b_stage1 = 240.0
    achieved = b_stage1 * ncell / (st["stage1"] / 1e3) / 1e9
    traffic = read_profile_value("sweep2d_kh2048_ncu.md", "TRAFFIC_PER_LAUNCH_STAGE1_BYTES")
    line = {
        "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s",
        "n_gpus": ctx.world, "steps": K, "warmup": W, "ms_per_step": ms / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "kelvin_helmholtz_2d_%dx%d_fp64" % (NX, NX), "global_batch": ctx.world,
                   "seq_len": ncell, "parallelism": "replicas" if ctx.world > 1 else "single",
                   "precision": "plain FP64 (reference operation order)",
                   "l2": "inputs larger than L2 (state 2 x 168 MB)"},
        "gpu_launches": 6 * K,
        "e2e": {"value": e2e, "unit": "zone-updates/s", "h2d_bytes_per_step": h2d / K,
                "d2h_bytes_per_step": d2h / K,
                "timed": "upload initial state (pinned H2D) + %d steps + download state (pinned D2H)" % K,
                "ms": ms_e2e},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "second RK stage (xsweep2d_kernel<1> + ysweep2d_kernel<1>)",
                     "kernel_ms": st["stage1"], "stage0_ms": st["stage0"],
                     "algorithmic_bytes_per_zone": b_stage1,
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"},
        "clocks": clocks,
        "mixed": {"value": ctx.world * ncell * K / (ms_mix / 1e3), "unit": "zone-updates/s", "ms_per_step": ms_mix / K,
                  "precision": "FP32 reconstruction and HLLC wave speeds, FP64 fluxes, accumulation, update, dt",
                  "accuracy_vs_fp64": accuracy},
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_kh(pb)
    print(json.dumps(line), flush=True)


SEDOV3D = (384, 128, 256)
SEDOV3D_SAMPLE = (96, 64, 128)
SEDOV3D_DR_MIN = 1.0e-3     # innermost zone width of the "sinh" radial map; r spans [0, 1]
SEDOV3D_R_LOG = 1.0e-3      # the "sinh-r1e-3" map: log-spaced zones from r = 1e-3 to 1


def sedov3d_problem(dims, radius="sinh-r1e-3"):
    """The 3-D Sedov workload: E = 1 deposited inside r < 0.02, on
      - "sinh-r1e-3" (default): the SINH radial map with rtrans = 1e-3, i.e. zones
        log-spaced from r = 1e-3 to 1 (about 2e-5 wide inside r = 1e-3).  A purely
        log-spaced radius starting at r = 1e-3 (RCOORD=LOG) is rejected on the 3-D
        dendritic grid by the reference's own init_dendritic (4-to-1 phi refinement) and
        by the library alike;
      - "sinh": the SINH map with zones SEDOV3D_DR_MIN x 384/n1 wide at the centre;
      - "uniform": the uniform radius."""
    from medusa_b200 import problems as P
    if radius == "uniform":
        return P.sedov_3d(*dims)
    if radius == "sinh-r1e-3":
        return P.sedov_3d(*dims, r_dep=0.02, coords="sinh_rt", r_in=SEDOV3D_R_LOG)
    return P.sedov_3d(*dims, r_dep=0.02, dr_min=SEDOV3D_DR_MIN * SEDOV3D[0] / dims[0])


def sedov3d_workload_name(dims, radius="sinh-r1e-3"):
    tag = {"sinh": "sinh_r_", "uniform": "", "sinh-r1e-3": "log_r_1e-3_to_1_sinh_"}[radius]
    return "sedov_3d_dendritic_spherical_%s%dx%dx%d_fp64" % (tag, *dims)


def sedov3d_grid_text(pb, radius):
    from medusa_b200 import problems as P
    e = P.radial_edges(pb)
    if radius == "uniform":
        return "uniform radius"
    if radius == "sinh-r1e-3":
        return ("SINH radial map with rtrans %.1e (RCOORD=SINH): zones log-spaced from r = 1e-3 to 1 "
                "(d ln r = %.4f at r = 1), %.2e wide inside r = 1e-3" % (pb.rtrans, math.log(e[-1] / e[-2]), e[1]))
    return ("SINH radial map (RCOORD=SINH, rtrans %.4f): zones %.1e wide at the centre, %.1e at r = 1"
            % (pb.rtrans, e[1], 1.0 - e[-2]))


def cpu_baseline_sedov3d(steps=2, radius="sinh-r1e-3"):
    """Reference CPU build (its Makefile flags), one core, `steps` RK2 steps of the same
    Sedov blast on a smaller dendritic grid (96 x 64 x 128 before coarsening, the same
    radial map scaled to 96 zones): the full grid needs several GB of host memory for the
    reference's per-zone geometry records."""
    from oracle import pyoracle
    pb = sedov3d_problem(SEDOV3D_SAMPLE, radius)
    if pyoracle.ref_available(pb, fast=True):
        r = pyoracle.time_reference(pb, 1, steps, fast=True)
        return {"value": r["zone_updates_per_s"], "unit": "zone-updates/s", "cores": 1, "kind": "reference",
                "sample": "%d RK2 steps of the Sedov blast on the %dx%dx%d dendritic grid (%d zones, %s radius), "
                          "reference build with its own flags (-O3 -ffast-math), 1 core, %.1f s"
                          % (steps, *SEDOV3D_SAMPLE, pb.ncell, radius, r["seconds"])}
    return {"value": None, "unit": "zone-updates/s", "cores": 1, "kind": "reference",
            "sample": "unavailable: the 3-D reference build is absent"}


def run_sedov3d(args, ctx):
    import numpy as np
    import medusa_b200
    from medusa_b200 import problems as P

    K, W = args.steps, args.warmup
    dims = tuple(int(x) for x in args.sedov3d_dims.split(",")) if args.sedov3d_dims else SEDOV3D
    pb = sedov3d_problem(dims, args.sedov3d_radius)
    ncell = pb.ncell
    s = medusa_b200.Solver(pb, device=ctx.local)
    warm_up(s, W)
    s.synchronize()
    ms, clocks = timed_steps(ctx, s, K, sample_clocks=True)
    value = ctx.world * ncell * K / (ms / 1e3)
    st = stage_times(s, min(K, 10))
    s.close()
    ms_e2e, h2d, d2h = e2e_run(ctx, lambda upload: medusa_b200.Solver(pb, device=ctx.local, upload=upload),
                               [pb], K, W)
    e2e = ctx.world * ncell * K / (ms_e2e / 1e3)
    # the mixed-precision sweep on the same grid, and its accuracy at equal physical time
    from medusa_b200 import analytic as A
    from medusa_b200.solver import PREC_MIXED, grid3d_radial_mean, grid3d_zone_volumes
    sm = medusa_b200.Solver(pb, precision=PREC_MIXED, device=ctx.local)
    warm_up(sm, W)
    sm.synchronize()
    ms_mix, _ = timed_steps(ctx, sm, K)
    sm.close()
    nacc = args.sedov3d_accuracy_steps
    with medusa_b200.Solver(pb, device=ctx.local) as sf:
        sf.step(nacc)
        ref = sf.update_cpu(0)
        t_end = sf.time(0)[0]
        m0, e0 = sf.conserved_totals()
    with medusa_b200.Solver(pb.copy(tmax=t_end), precision=PREC_MIXED, device=ctx.local) as sa:
        n_mix = 0
        while sa.time(0)[0] < t_end * (1.0 - 1.0e-12) and n_mix < 4 * nacc:
            sa.step(10)
            n_mix += 10
        mix = sa.update_cpu(0)
        m1, e1 = sa.conserved_totals()
    vol = grid3d_zone_volumes(pb)
    rc = P.radial_centers(pb)
    r_of = lambda prim: float(rc[int(np.argmax(grid3d_radial_mean(pb, prim[:, 0])))])
    accuracy = {"steps": nacc, "t": t_end, "l1_rho": A.l1_rel(mix[:, 0], ref[:, 0], vol),
                "l1_u": A.l1_rel(mix[:, 1], ref[:, 1], vol),
                "mass_drift_vs_fp64": abs(m1[0] - m0[0]) / m0[0], "energy_drift_vs_fp64": abs(e1[0] - e0[0]) / e0[0],
                "shock_radius_fp64": r_of(ref), "shock_radius_mixed": r_of(mix),
                "shock_radius_sedov": A.sedov_shock_radius(1.0, t_end, 1.0, pb.gam),
                "dr_at_shock": float(np.interp(r_of(ref), rc, np.diff(P.radial_edges(pb))))}
    full = sedov3d_full_run(ctx, pb, args.sedov3d_t_end) if args.sedov3d_t_end > 0.0 else None
    if ctx.rank != 0:
        return
    peak, peak_kind = read_peaks()
    b_stage1 = 360.0
    achieved = b_stage1 * ncell / (st["stage1"] / 1e3) / 1e9
    traffic = read_profile_value({"sinh": "sweep3d_sedov_sinh_ncu.md", "uniform": "sweep3d_sedov_ncu.md",
                                  "sinh-r1e-3": "sweep3d_sedov_log_r1e-3_ncu.md"}[args.sedov3d_radius],
                                 "TRAFFIC_PER_LAUNCH_STAGE1_BYTES")
    line = {
        "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s",
        "n_gpus": ctx.world, "steps": K, "warmup": W, "ms_per_step": ms / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": sedov3d_workload_name(dims, args.sedov3d_radius), "global_batch": ctx.world,
                   "seq_len": ncell, "parallelism": "replicas" if ctx.world > 1 else "single",
                   "precision": "plain FP64 (reference operation order)",
                   "grid": sedov3d_grid_text(pb, args.sedov3d_radius),
                   "l2": "inputs larger than L2 (state 2 x %.0f MB)" % (ncell * 40 / 1e6)},
        "gpu_launches": 10 * K,
        "e2e": {"value": e2e, "unit": "zone-updates/s", "h2d_bytes_per_step": h2d / K,
                "d2h_bytes_per_step": d2h / K,
                "timed": "upload initial state (pinned H2D) + %d steps + download state (pinned D2H)" % K,
                "ms": ms_e2e},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "second RK stage (face0/face1/face2/push3 kernels <1>)",
                     "kernel_ms": st["stage1"], "stage0_ms": st["stage0"],
                     "algorithmic_bytes_per_zone": b_stage1,
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"},
        "clocks": clocks,
        "mixed": {"value": ctx.world * ncell * K / (ms_mix / 1e3), "unit": "zone-updates/s", "ms_per_step": ms_mix / K,
                  "precision": "FP32 reconstruction and HLLC wave speeds, FP64 state, fluxes, sources, dt",
                  "accuracy_vs_fp64": accuracy},
    }
    if full is not None:
        line["full_run"] = full
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sedov3d(radius=args.sedov3d_radius)
    print(json.dumps(line), flush=True)


def sedov3d_full_run(ctx, pb, t_end, chunk=2000):
    """The Sedov blast run from t = 0 to t_end in plain FP64 and in mixed precision (each
    step the main.c loop, the last one clipped onto t_end); device time with CUDA events;
    L1 of density and total energy density against the Sedov-Taylor solution (shell
    averages of the analytic state per radial row, volume-weighted over the zones), the
    mixed result against the FP64 one, and mass and energy drift over the run."""
    import numpy as np
    import torch
    import medusa_b200
    from medusa_b200 import analytic as A
    from medusa_b200 import problems as P
    from medusa_b200.solver import PREC_FP64, PREC_MIXED, grid3d_counts, grid3d_zone_gcov, grid3d_zone_volumes

    vol = grid3d_zone_volumes(pb)
    gcov = grid3d_zone_gcov(pb)
    nj, nk, _ = grid3d_counts(pb)
    per_row = np.add.reduceat(nk, np.concatenate([[0], np.cumsum(nj)[:-1]]))
    edges = P.radial_edges(pb)

    def etot(prim):
        return 0.5 * prim[:, 0] * np.sum(gcov * prim[:, 2:5] ** 2, axis=1) + prim[:, 1]

    def run(precision):
        with medusa_b200.Solver(pb.copy(tmax=t_end), precision=precision, device=ctx.local) as s:
            m0, e0 = s.conserved_totals()
            stream = torch.cuda.ExternalStream(s.stream, device=ctx.local)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            w0 = time.time()
            ev0.record(stream)
            while True:
                s.step(chunk)
                t, _, istep = s.time(0)
                sys.stderr.write("sedov3d %s: step %d, t %.6e of %.3e, %.1f s\n"
                                 % ("fp64" if precision == PREC_FP64 else "mixed", istep, t, t_end,
                                    time.time() - w0))
                sys.stderr.flush()
                if t >= t_end * (1.0 - 1.0e-12):
                    break
            ev1.record(stream)
            ev1.synchronize()
            s.synchronize()
            wall = time.time() - w0
            m1, e1 = s.conserved_totals()
            prim = s.update_cpu(0)
            return {"prim": prim, "t": t, "steps": istep, "device_ms": ev0.elapsed_time(ev1), "wall_s": wall,
                    "mass_drift": float((m1[0] - m0[0]) / m0[0]), "energy_drift": float((e1[0] - e0[0]) / e0[0])}

    out = {"t_end": t_end}
    res = {}
    S = A.SedovTaylor(pb.gam)
    # zones of the blast: radial rows whose inner edge lies inside 1.25 shock radii (the
    # ambient gas outside is at rest in both and would dilute the norm)
    row_in = np.repeat(edges[:-1] < 1.25 * S.shock_radius(1.0, t_end), per_row)
    w = vol * row_in
    for name, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        r = run(prec)
        ana = A.sedov_row_averages(edges, r["t"], pb.gam, energy=1.0, rho0=1.0, p_amb=1.0e-5)
        rho_a = np.repeat(ana[:, 0], per_row)
        e_a = np.repeat(ana[:, 3], per_row)
        res[name] = r
        out[name] = {"steps": r["steps"], "t": r["t"], "device_ms": r["device_ms"], "wall_s": r["wall_s"],
                     "zone_updates_per_s": pb.ncell * r["steps"] / (r["device_ms"] / 1e3),
                     "l1_rho_vs_sedov": A.l1_rel(r["prim"][:, 0], rho_a, w),
                     "l1_etot_vs_sedov": A.l1_rel(etot(r["prim"]), e_a, w),
                     "mass_drift": r["mass_drift"], "energy_drift": r["energy_drift"]}
    a, b = res["mixed"]["prim"], res["fp64"]["prim"]
    out["mixed_vs_fp64"] = {"l1_rho": A.l1_rel(a[:, 0], b[:, 0], w), "l1_u": A.l1_rel(a[:, 1], b[:, 1], w),
                            "l1_etot": A.l1_rel(etot(a), etot(b), w),
                            "l1_rho_over_fp64_truncation": A.l1_rel(a[:, 0], b[:, 0], w) /
                            out["fp64"]["l1_rho_vs_sedov"]}
    out["sedov"] = {"xi0": S.xi0, "shock_radius": S.shock_radius(1.0, res["fp64"]["t"]),
                    "reference": "Sedov-Taylor point blast, closed form (Sedov 1959; Kamm & Timmes 2007), "
                                 "shell averages per radial row; L1 over the zones of the rows inside 1.25 "
                                 "shock radii (%d zones)" % int(row_in.sum())}
    return out


EOS_ZONES = 8 * 1024 * 1024
EOS_BYTES_PER_ZONE = 72      # rho, u, Ye, T read; T, p, cs, s, Gamma_1 written (FP64)


def cpu_baseline_eos(n=1 << 20):
    """The reference's own tabulated-EOS zone update (eos/burrows/eos_stuff.c:768-902,
    oracle/_ref/refeos) on one core over n seeded zones of the synthetic table at the
    reference's sizes, from the temperatures of a first pass (the warm start that the GPU
    leg's timed launches have too); the second pass's loop alone is timed."""
    import subprocess
    import tempfile
    import numpy as np
    from medusa_b200 import eos_table as ET
    from oracle import pyoracle
    exe = os.path.join(pyoracle.REF_DIR, "refeos")
    if not os.path.exists(exe):
        return {"value": None, "unit": "zone EOS updates/s", "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref/refeos was not built"}
    g = ET.REFERENCE_GRID
    tab = ET.synthetic_table(g)
    rho, u, ye, tg = ET.synthetic_zones(g, n, seed=32, table=tab)
    with tempfile.TemporaryDirectory() as td:
        ft, fz, fo = (os.path.join(td, x) for x in ("table.bin", "zones.bin", "out.bin"))
        tab.tofile(ft)
        for _ in range(2):
            with open(fz, "wb") as f:
                f.write(np.int64(n).tobytes())
                f.write(np.ascontiguousarray(np.stack([rho, u, ye, tg], axis=1)).tobytes())
            r = subprocess.run([exe, ft, fz, fo], check=True, capture_output=True, text=True)
            tg = np.fromfile(fo, dtype=np.float64).reshape(-1, 5)[:, 2].copy()
    kv = dict(tok.split("=") for tok in r.stdout.split())
    sec = float(kv["seconds"])
    return {"value": n / sec, "unit": "zone EOS updates/s", "cores": 1, "kind": "reference",
            "sample": "%d zones, temperature guesses from a first pass, the reference's eos_given_rex_per_zone "
                      "built with -O2 -fno-fast-math, 1 core, %.3f s" % (n, sec)}


def run_eos(args, ctx):
    """The tabulated nuclear EOS zone update (eos_given_rex_per_zone) over EOS_ZONES zones
    of the synthetic table at the reference's sizes (16 x 50 x 300 x 300); each launch
    starts from the previous launch's temperatures, as successive calls of the reference
    do (eos[TEMP] is the guess)."""
    import numpy as np
    import torch
    from medusa_b200 import eos_table as ET
    g = ET.REFERENCE_GRID
    tab = ET.synthetic_table(g)
    n = EOS_ZONES
    rho, u, ye, tg = ET.synthetic_zones(g, n, seed=31, table=tab)
    dev = ctx.local
    with ET.EosTable(tab, g, device=dev) as t:
        ins = [torch.tensor(a, dtype=torch.float64, device="cuda:%d" % dev) for a in (rho, u, ye, tg)]
        outs = [torch.empty(n, dtype=torch.float64, device="cuda:%d" % dev) for _ in range(4)]
        stream = torch.cuda.current_stream(dev)
        ptrs = [x.data_ptr() for x in ins] + [o.data_ptr() for o in outs]

        def launch():
            t.given_rex_device(n, *ptrs, stream=stream.cuda_stream)
        for _ in range(args.warmup):
            launch()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(dev)
        sampler.start()
        ctx.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            launch()
        e1.record(stream)
        e1.synchronize()
        ms = ctx.max_ms(e0.elapsed_time(e1)) / args.steps
        clocks = sampler.stop()
        # end to end through the host entry point: host arrays, copies in and out included
        h0 = time.perf_counter()
        k_e2e = 3
        for _ in range(k_e2e):
            t.given_rex(rho, u, ye, tg)
        e2e_ms = (time.perf_counter() - h0) * 1e3 / k_e2e
    value = ctx.world * n / (ms / 1e3)
    if ctx.rank != 0:
        return
    peak, peak_kind = read_peaks()
    achieved = EOS_BYTES_PER_ZONE * n / (ms / 1e3) / 1e9
    line = {
        "metric": "zone EOS updates/s", "value": value, "unit": "zone EOS updates/s", "n_gpus": ctx.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "tabulated_eos_given_rex_%dM_zones_table_16x50x300x300" % (n >> 20),
                   "global_batch": ctx.world, "seq_len": n,
                   "parallelism": "replicas" if ctx.world > 1 else "single",
                   "l2": "inputs and outputs (600 MB) and table (180 MB on the device) larger than L2"},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "e2e": {"value": ctx.world * n / (e2e_ms / 1e3), "unit": "zone EOS updates/s",
                "h2d_bytes_per_step": 32 * n, "d2h_bytes_per_step": 40 * n,
                "timed": "mdg_eos_given_rex_host: pageable host arrays, copies in and out, wall clock"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "eos_rex_kernel",
                     "algorithmic_bytes_per_zone": EOS_BYTES_PER_ZONE,
                     "note": "streamed zone bytes only; each zone also gathers 4 x 64 B of interpolated "
                             "records and 32 B per energy-scan step from the table",
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"},
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_eos()
    print(json.dumps(line), flush=True)


def run_sod1d(args, ctx):
    """Config C1: the Sod tube of problems/init_sod.c, 1024 zones, CFL 0.8, run to t = 0.2
    in plain FP64, timed as a whole (device time from t = 0 to the end: the resident
    stepper, one launch per 256 steps, where the device allows its 16-CTA cluster, else
    the per-phase launches replayed from CUDA graphs), compared zone by zone with the
    reference's own run of the same job and with the exact Riemann solution."""
    import numpy as np
    import torch
    from medusa_b200 import analytic as A
    from medusa_b200 import problems as P
    from medusa_b200.solver import Solver
    pb = P.sod(1024).copy(cfl=0.8, tmax=0.2)
    nmax = 4000                      # at most; steps past t = 0.2 leave the problem unchanged
    with Solver(pb, device=ctx.local) as s:
        # the job's step count first (untimed), then exactly that many steps timed
        s.step(nmax)
        s.synchronize()
        nmax = s.time(0)[2]
        warm_up(s, args.warmup)
        s.upload(0, pb.ic)
        stream = torch.cuda.ExternalStream(s.stream, device=ctx.local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(ctx.local)
        sampler.start()
        ctx.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        s.step(nmax)
        e1.record(stream)
        e1.synchronize()
        s.synchronize()
        ms = ctx.max_ms(e0.elapsed_time(e1))
        clocks = sampler.stop()
        prim = s.update_cpu(0)
        t, _, istep = s.time(0)
        resident = s.resident_cluster()
    value = ctx.world * pb.ncell * istep / (ms / 1e3)
    l1 = A.l1_rel(prim[:, 0], A.sod_exact_state(1024, t)[:, 0])
    if ctx.rank != 0:
        return
    from oracle import pyoracle
    ref = {}
    if pyoracle.ref_available(pb) and not args.no_cpu_baseline:
        last = pyoracle.run_reference(pb, istep, every=istep)[-1]
        d = np.abs(prim - last[4]) / np.maximum(np.abs(last[4]), 1.0e-300)
        d[prim == last[4]] = 0.0
        ref = {"max_rel_diff_vs_reference": float(d.max()), "bit_identical_fraction": float(np.mean(prim == last[4])),
               "reference_t": last[1], "reference_steps": last[0]}
    peak, peak_kind = read_peaks()
    achieved = 200.0 * pb.ncell * istep / (ms / 1e3) / 1e9
    line = {
        "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s", "n_gpus": ctx.world,
        "steps": istep, "warmup": args.warmup, "ms_per_step": ms / istep, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "sod_1d_cartesian_1024_to_t0.2_fp64", "global_batch": ctx.world, "seq_len": 1024,
                   "parallelism": "replicas" if ctx.world > 1 else "single",
                   "l2": "resident in L2 (80 KB state): a latency-bound job, timed whole"},
        # resident: one launch per 256 steps; else dt, two stages and the time update per step
        "gpu_launches": (nmax + 255) // 256 if resident else 4 * nmax,
        "resident_cluster_ctas": resident,
        "time_to_solution_ms": ms, "t": t, "clocks": clocks,
        "accuracy": dict({"l1_rho_vs_exact_riemann": l1}, **ref),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "note": "1024 zones: bound by the latency of each step's dependent "
                                              "phases, not by HBM",
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"},
    }
    if not args.no_cpu_baseline and pyoracle.ref_available(pb, fast=True):
        r = pyoracle.time_reference(pb, 0, istep, fast=True)
        line["cpu_baseline"] = {"value": r["zone_updates_per_s"], "unit": "zone-updates/s", "cores": 1,
                                "kind": "reference",
                                "sample": "the whole job (%d RK2 steps), reference build with its own flags "
                                          "(-O3 -ffast-math), 1 core, %.3f s" % (istep, r["seconds"])}
    print(json.dumps(line), flush=True)


def server_workload_name(args):
    if args.server_frac_3d > 0.0:
        return "server_stream_%d%%_1d_%d%%_2d_%d%%_3d_sedov_128x64x128" % (
            round(100 * (1 - args.server_frac_2d - args.server_frac_3d)), round(100 * args.server_frac_2d),
            round(100 * args.server_frac_3d))
    if args.server_frac_2d > 0.0:
        return "server_stream_1d_spherical_256_8192_and_%d%%_2d_cartesian_128sq_1024sq" % round(
            100 * args.server_frac_2d)
    return "server_stream_1d_spherical_256_8192_zones"


def run_server(args, ctx):
    """Solve-server stream: seeded 1-D spherical requests (Sod/Noh/Sedov, 256-8192 zones)
    and, with --server-frac-2d, 2-D Cartesian ones (Kelvin-Helmholtz / Rayleigh-Taylor,
    128^2-1024^2 zones), each to its end time, submitted with Poisson arrivals at a swept
    rate to a running server, mixed precision and plain FP64; throughput and p50/p99
    time-to-solution."""
    import math
    from medusa_b200 import loadgen
    from medusa_b200.solver import PREC_FP64, PREC_MIXED, Server

    rates = [float(r) for r in args.server_rates.split(",")]
    reqs = loadgen.request_stream(args.server_requests, seed=11 + ctx.rank, frac_2d=args.server_frac_2d,
                                  frac_3d=args.server_frac_3d)
    spr = 20
    sweep = {}
    best = {}
    two_d = args.server_frac_2d > 0.0
    three_d = args.server_frac_3d > 0.0
    for name, prec in (("mixed", PREC_MIXED), ("fp64", PREC_FP64)):
        sweep[name] = []
        srv = Server(precision=prec, device=ctx.local, hbm_bytes=24 << 30, max_problems=16384, max_zones=8192,
                     steps_per_round=spr, threads=64, ctas_per_sm=12,
                     hbm_bytes_2d=(32 << 30) if two_d else 0, max_cells_2d=(1 << 20) + 4096,
                     hbm_bytes_3d=(24 << 30) if three_d else 0)
        srv.start()
        # warm-up: graph capture and first admissions
        loadgen.drive(srv, reqs[:32], math.inf)
        for rate in rates:
            n = len(reqs) if math.isinf(rate) else int(min(len(reqs), max(200, rate * args.server_seconds)))
            ctx.barrier()
            r = loadgen.drive(srv, reqs[:n], rate)
            sweep[name].append(r)
        st = srv.stats()
        srv.stop()
        srv.close()
        best[name] = max(sweep[name], key=lambda r: r["zone_updates_per_s"])
        best[name]["device_seconds_total"] = st["device_seconds"]
        best[name]["rounds_total"] = st["rounds"]
        best[name]["kernel_launches_total"] = st["kernel_launches"]
    value = ctx.total(best["mixed"]["zone_updates_per_s"])   # independent servers, one per rank
    if ctx.rank != 0:
        return
    peak, peak_kind = read_peaks()
    m = best["mixed"]
    zu_dev = m["zone_updates_per_s"]
    h2d = sum(pb.ncell for pb in reqs[:m["requests"]]) * 40
    line = {
        "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s", "n_gpus": ctx.world,
        "steps": spr, "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": server_workload_name(args),
                   "requests": len(reqs), "rates_req_per_s": args.server_rates,
                   "mix": ("1-D spherical Sod/Noh/Sedov, %d%% 2-D Cartesian KH/RT (FP64 split sweep in both "
                           "server precisions) and %d%% 3-D Sedov on the 128x64x128 dendritic grid (the "
                           "server's precision) to their end times"
                           % (round(100 * args.server_frac_2d), round(100 * args.server_frac_3d))) if two_d else
                          "1-D spherical Sod/Noh/Sedov to their end times (the 1-D part of the request mix)",
                   "steps_per_round": spr, "parallelism": "single" if ctx.world == 1 else "independent servers"},
        "p50_s": m["latency_p50_s"], "p99_s": m["latency_p99_s"],
        "sweep": sweep,
        "fp64_best_zone_updates_per_s": best["fp64"]["zone_updates_per_s"],
        "mixed_over_fp64": m["zone_updates_per_s"] / best["fp64"]["zone_updates_per_s"],
        "gpu_launches": m["kernel_launches_total"],
        "e2e": {"value": value, "unit": "zone-updates/s", "h2d_bytes_per_step": h2d / max(1, m["rounds_total"]),
                "d2h_bytes_per_step": h2d / max(1, m["rounds_total"]),
                "timed": "submission of every request from host memory to the return of every final state"},
        "roofline": {"bound": "hbm", "achieved": 200.0 * zu_dev / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": 200.0 * zu_dev / 1e9 / peak, "traffic": None,
                     "note": "whole-stream rate x 200 B/zone-update (1-D B_alg), wall clock",
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ensemble",
                    choices=["ensemble", "kh2048", "server", "sedov3d", "sod1d", "eos"])
    ap.add_argument("--server-requests", type=int, default=6000)
    ap.add_argument("--server-rates", default="1000,4000,16000,inf",
                    help="server: Poisson arrival rates (requests/s) swept; inf = all at once")
    ap.add_argument("--sedov3d-dims", default="",
                    help="sedov3d: n1,n2,n3 of the grid (default 384,128,256; smaller grids for profiling)")
    ap.add_argument("--sedov3d-radius", default="sinh-r1e-3", choices=["sinh-r1e-3", "sinh", "uniform"],
                    help="sedov3d: radial map; sinh-r1e-3 = zones log-spaced from r = 1e-3 to 1 (RCOORD=SINH "
                         "with rtrans 1e-3), sinh = zones 1e-3 wide at the centre widening geometrically to "
                         "r = 1, uniform = 1/n1 wide")
    ap.add_argument("--sedov3d-t-end", type=float, default=0.0,
                    help="sedov3d: also run the blast to this time in FP64 and in mixed precision and report "
                         "L1 of density and energy against the Sedov-Taylor solution and against each other, "
                         "and the mass and energy drift (0: skip; the configured end time is 0.05)")
    ap.add_argument("--sedov3d-accuracy-steps", type=int, default=60,
                    help="sedov3d: steps of the FP64 run the mixed run is compared with at equal time")
    ap.add_argument("--server-frac-2d", type=float, default=0.0,
                    help="server: fraction of 2-D Cartesian requests (0.263 = the 70:25 share of 1-D and 2-D "
                         "requests of the mixed stream)")
    ap.add_argument("--server-frac-3d", type=float, default=0.0,
                    help="server: fraction of 3-D Sedov requests (0.05 with --server-frac-2d 0.25: the C5 mix)")
    ap.add_argument("--server-seconds", type=float, default=3.0,
                    help="server: length of the arrival window at each finite rate")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ensemble-count", type=int, default=ENSEMBLE_COUNT,
                    help="ensemble: number of problems (a smaller ensemble for profiling runs)")
    ap.add_argument("--launch", default=None,
                    help="ensemble: fixed mixed-sweep launch shape 'threads,ctas_per_sm' instead of the autotuner")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.steps is None:
        args.steps = 1000 if args.workload == "ensemble" else 200

    ctx = Ctx(*dist_setup())
    try:
        if args.impl == "reference":
            run_reference_arm(args, ctx)
            return
        import torch
        torch.cuda.set_device(ctx.local)
        if args.workload == "ensemble":
            run_ensemble(args, ctx)
        elif args.workload == "server":
            run_server(args, ctx)
        elif args.workload == "sedov3d":
            run_sedov3d(args, ctx)
        elif args.workload == "sod1d":
            run_sod1d(args, ctx)
        elif args.workload == "eos":
            run_eos(args, ctx)
        else:
            run_kh(args, ctx)
    finally:
        if ctx.dist is not None:
            ctx.dist.destroy_process_group()


if __name__ == "__main__":
    main()
