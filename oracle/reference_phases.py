"""Where the reference's CPU time goes: the phase split of its hot path from its own
timers (TEST/MEASUREMENT INFRASTRUCTURE ONLY; never part of the product path).

    python -m oracle.reference_phases

Runs the reftime_<cfg> builds of oracle/build_ref.py (the unmodified reference with its
Makefile flags and DO_TIMING=TRUE; timing.csv as io.c:51-108 writes it) on one core for
each workload and prints a Markdown table: per timer, seconds per step and the share of
the time of a step (estimate_dt + step).  The timers nest: step contains
prim_to_fluxes1/2/3, push, reset_boundaries and update_eos(_ghost); riemann_flux_HLLE and
p_to_phys_src_finish sit inside those.
"""
from __future__ import annotations

import os
import sys

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from medusa_b200 import problems as P
from oracle import pyoracle

ORDER = ("estimate_dt", "step", "prim_to_fluxes1", "prim_to_fluxes2", "prim_to_fluxes3", "push",
         "reset_boundaries", "update_eos", "update_eos_ghost", "riemann_flux_HLLE", "p_to_phys_src_finish",
         "avg_poles_3d")


def workloads():
    """(label, problem, warm-up steps, timed steps)."""
    return [
        ("C1 Sod 1024 (whole job)", P.sod(1024).copy(cfl=0.8, tmax=0.2), 0, 572),
        ("C2 Kelvin-Helmholtz 512^2 (C2's per-zone work; 2048^2 takes 12 s a step)",
         P.kelvin_helmholtz(512), 2, 20),
        ("C4 member: spherical Sedov, 4096 zones", P.spherical_1d("sedov", 4096, 1.4, p_ratio=1.0e4, r0=0.05),
         10, 200),
        ("C3 form: 3-D Sedov, dendritic 96 x 32 x 64, SINH radius (145,920 zones)",
         P.sedov_3d(96, 32, 64, r_dep=0.1, dr_min=0.004), 1, 6),
    ]


def main():
    print("| workload | zone-updates/s (1 core) | timer | s per step | share of step time |")
    print("|---|---:|---|---:|---:|")
    for label, pb, warm, steps in workloads():
        if not os.path.exists(os.path.join(pyoracle.REF_DIR, "reftime_" + pyoracle.ref_config(pb))):
            print("| %s | — | reftime_%s not built | | |" % (label, pyoracle.ref_config(pb)))
            continue
        r = pyoracle.time_reference_phases(pb, warm, steps)
        tm = r["timers"]
        total = tm.get("step", (0.0, 0))[0] + tm.get("estimate_dt", (0.0, 0))[0]
        first = True
        for name in ORDER:
            if name not in tm or tm[name][1] == 0:
                continue
            sec = tm[name][0]
            print("| %s | %s | %s | %.3e | %.1f %% |" % (label if first else "", "%.3g" % r["zone_updates_per_s"]
                                                       if first else "", name, sec / steps, 100.0 * sec / total))
            first = False


if __name__ == "__main__":
    main()
