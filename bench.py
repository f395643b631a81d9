"""Benchmark: plain FP64 hydro sweep on the 2-D Kelvin-Helmholtz workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: Kelvin-Helmholtz on the periodic unit square, 2048 x 2048 zones, gamma = 5/3,
CFL 0.8 (seeded synthetic initial state, medusa_b200.problems.kelvin_helmholtz).  A step
is one full RK2 step of the reference time loop (estimate_dt + both stages + t += dt);
the metric is zone-updates/s (zones x steps / seconds), whole job over all ranks.

- value:  device time of K steps with the state resident in HBM, CUDA events on the
          solver's stream, barrier + synchronize on both sides, max over ranks.  The
          state (2 x 168 MB) exceeds the 126 MB L2, so no L2 flush is needed.
- e2e:    the same metric through the public API with host buffers: upload of the
          initial state from pinned memory, K steps, download of the final state to
          pinned memory, all inside the timed region.
- roofline: the dominant kernel (second RK stage) against the measured HBM copy
          bandwidth; algorithmic bytes per zone-update B_alg(2-D) = 440 B, of which the
          second stage accounts for 240 B.
- cpu_baseline: the reference's own CPU build (its Makefile flags) on a bounded sample
          of the same workload, rank 0 only.
With --gpus N > 1 (torchrun), every rank runs an independent replica (the single-grid
sweep does not shard: replicas only).
--impl reference times the reference's CPU implementation instead (rank 0 only).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = 2048
B_ALG_STEP = 440.0          # bytes per zone-update, 2-D (240*NDIM - 40)
B_ALG_STAGE1 = 240.0        # second-stage share: read state, accumulators and base state
FALLBACK_HBM_GBS = 6650.0


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def read_profile_traffic():
    """Per-launch DRAM traffic of the second-stage kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "stage2d_kh2048_ncu.md")
    try:
        for line in open(path):
            if line.startswith("TRAFFIC_PER_LAUNCH_STAGE1_BYTES"):
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


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=None)
        return world, rank, local, dist
    return 1, 0, 0, None


def cpu_baseline_reference(pb_full, steps=2):
    """Reference CPU build (Makefile flags) on a bounded sample: `steps` RK2 steps of the
    full grid, single core (the reference's hot path has no host threading)."""
    from oracle import pyoracle
    if pyoracle.ref_available(pb_full, fast=True):
        r = pyoracle.time_reference(pb_full, 0, steps, fast=True)
        return {"value": r["zone_updates_per_s"], "unit": "zone-updates/s", "cores": 1,
                "kind": "reference",
                "sample": "%d RK2 steps of the %dx%d grid, reference build with its own flags "
                          "(-O3 -ffast-math), 1 core, %.1f s" % (steps, NX, NX, r["seconds"])}
    # the oracle restatement when the reference build is not present
    o = pyoracle.Oracle(pb_full)
    t0 = time.perf_counter()
    o.advance(1)
    el = time.perf_counter() - t0
    return {"value": pb_full.ncell / el, "unit": "zone-updates/s", "cores": 1, "kind": "port",
            "sample": "1 RK2 step of the %dx%d grid, CPU oracle, 1 core, %.1f s" % (NX, NX, el)}


def run_reference_arm(args, world, rank):
    from medusa_b200 import problems as P
    if rank != 0:
        return
    pb = P.kelvin_helmholtz(NX)
    cb = cpu_baseline_reference(pb, steps=max(1, min(args.steps, 2)))
    line = {"metric": "zone-updates/s", "value": cb["value"], "unit": "zone-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "kelvin_helmholtz_2d_%dx%d_fp64" % (NX, NX), "global_batch": 1,
                       "seq_len": NX * NX, "parallelism": "replicas", "l2": "inputs larger than L2"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world, rank, local, dist = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        if dist is not None:
            dist.destroy_process_group()
        return

    import numpy as np
    import torch
    import medusa_b200
    from medusa_b200 import problems as P

    torch.cuda.set_device(local)
    pb = P.kelvin_helmholtz(NX)
    ncell = pb.ncell
    K, W = args.steps, args.warmup

    s = medusa_b200.Solver(pb, device=local)
    stream = torch.cuda.ExternalStream(s.stream, device=local)
    s.step(W)
    s.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- value: K steps, state resident in HBM
    sampler = ClockSampler(local)
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    s.step(K)
    e1.record(stream)
    e1.synchronize()
    s.synchronize()
    barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * ncell * K / (ms / 1e3)

    # ---- per-kernel timers (roofline of the dominant kernel)
    s.set_timing(True)
    nt = min(K, 20)
    s.step(nt)
    s.synchronize()
    tm = s.timers()
    s.set_timing(False)
    st0 = tm["stage0"][0] / max(1, tm["stage0"][1])
    st1 = tm["stage1"][0] / max(1, tm["stage1"][1])
    peak, peak_kind = read_peaks()
    achieved = B_ALG_STAGE1 * ncell / (st1 / 1e3) / 1e9
    traffic = read_profile_traffic()

    # ---- e2e: pinned host buffers, upload + K steps + download in the timed region
    h_in = torch.from_numpy(np.ascontiguousarray(pb.ic)).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    s2 = medusa_b200.Solver(pb, device=local, upload=False)
    stream2 = torch.cuda.ExternalStream(s2.stream, device=local)
    s2.upload_ptr(0, h_in.data_ptr())
    s2.step(W)
    s2.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    f0.record(stream2)
    s2.upload_ptr(0, h_in.data_ptr())
    s2.step(K)
    s2.download_ptr(0, h_out.data_ptr())
    f1.record(stream2)
    f1.synchronize()
    barrier()
    ms_e2e = f0.elapsed_time(f1)
    if dist is not None:
        tt = torch.tensor([ms_e2e], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_e2e = float(tt.item())
    e2e = world * ncell * K / (ms_e2e / 1e3)
    nbytes = ncell * 5 * 8
    s2.close()
    s.close()

    if rank == 0:
        line = {
            "metric": "zone-updates/s", "value": value, "unit": "zone-updates/s",
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "kelvin_helmholtz_2d_%dx%d_fp64" % (NX, NX), "global_batch": world,
                       "seq_len": ncell, "parallelism": "replicas" if world > 1 else "single",
                       "precision": "plain FP64 (reference operation order)",
                       "l2": "inputs larger than L2 (state 2 x 168 MB)"},
            "gpu_launches": 4 * K,
            "e2e": {"value": e2e, "unit": "zone-updates/s", "h2d_bytes_per_step": nbytes / K,
                    "d2h_bytes_per_step": nbytes / K,
                    "timed": "upload initial state (pinned H2D) + %d steps + download state (pinned D2H)" % K,
                    "ms": ms_e2e},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "stage2d_kernel<1> (second RK stage)",
                         "kernel_ms": st1, "stage0_ms": st0,
                         "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"},
            "clocks": clocks,
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_reference(pb)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
