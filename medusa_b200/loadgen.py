"""Synthetic request streams for the solve server.

:func:`request_stream` draws a seeded list of 1-D spherical requests (Sod-, Noh- and
Sedov-type, zone counts log-uniform in a range, density/pressure ratios and gamma as in
:func:`medusa_b200.problems.ensemble_1d`), each with an end time chosen per kind so that
it runs a few hundred steps at the largest sizes; a fraction `frac_2d` of the requests are
2-D Cartesian instead (Kelvin-Helmholtz on the unit square or Rayleigh-Taylor on
[0, 0.5] x [0, 1] with rho 2 over 1, g = -0.1 and velocity noise 0.01, zone counts
log-uniform in [zmin_2d, zmax_2d]) and a fraction `frac_3d` 3-D Sedov blasts on the
dendritic spherical grid (dims_3d before coarsening).  :func:`drive` submits such a stream to a
running :class:`medusa_b200.solver.Server` with Poisson arrivals at a given rate (all at
once for rate=inf), waits for every result and reports throughput and latency
percentiles.
"""
from __future__ import annotations

import math
import threading
import time

import numpy as np

from . import problems as P

# end time per kind: a fixed fraction of the sound-crossing time of the unit sphere
T_END = {"sod": 0.05, "noh": 0.08, "sedov": 0.02, "kh": 0.05, "rt": 0.1, "sedov3d": 0.01}


def _request_2d(m: int, u) -> "P.Problem":
    """2-D request m from four uniforms: kind, zone count (log-uniform in the range given by
    u[0] already scaled to a zone count), noise seed and end-time factor."""
    z, kind_u, t_u = u
    if kind_u < 0.5:
        n = max(16, int(round(math.sqrt(z))))
        pb = P.kelvin_helmholtz(n, n, seed=1000 + m).copy(tmax=T_END["kh"] * (0.5 + t_u))
        pb.name = "req%05d_kh%d" % (m, n)
    else:
        n1 = max(8, int(round(math.sqrt(z / 2.0))))
        pb = P.rayleigh_taylor_2d(n1, 2 * n1, g=-0.1, seed=2000 + m, noise=0.01).copy(tmax=T_END["rt"] * (0.5 + t_u))
        pb.name = "req%05d_rt%dx%d" % (m, n1, 2 * n1)
    return pb


def request_stream(count: int, seed: int = 11, nmin: int = 256, nmax: int = 8192, frac_2d: float = 0.0,
                   zmin_2d: int = 128 * 128, zmax_2d: int = 1024 * 1024, frac_3d: float = 0.0,
                   dims_3d: tuple = (128, 64, 128)) -> list:
    """`count` seeded requests (Problems whose tmax is the end time)."""
    u = P.uniform01(seed, 6 * count).reshape(count, 6)
    # the 2-D draws come from their own stream, so the 1-D requests of a seed stay the same
    u2 = P.uniform01(seed + 7919, 4 * count).reshape(count, 4)
    gams = (4.0 / 3.0, 1.4, 5.0 / 3.0)
    kinds = ("sod", "noh", "sedov")
    out = []
    for m in range(count):
        if u2[m, 0] < frac_2d:
            z = math.exp(math.log(zmin_2d) + u2[m, 1] * (math.log(zmax_2d) - math.log(zmin_2d)))
            out.append(_request_2d(m, (z, u2[m, 2], u2[m, 3])))
            continue
        if u2[m, 0] < frac_2d + frac_3d:
            pb = P.sedov_3d(*dims_3d, r_dep=0.02, noise=0.01, seed=3000 + m)
            pb = pb.copy(tmax=T_END["sedov3d"] * (0.5 + u2[m, 3]))
            pb.name = "req%05d_sedov3d" % m
            out.append(pb)
            continue
        n1 = int(round(math.exp(math.log(nmin) + u[m, 0] * (math.log(nmax) - math.log(nmin)))))
        n1 = max(nmin, min(nmax, n1))
        kind = kinds[min(2, int(u[m, 1] * 3))]
        rr = math.exp(math.log(2.0) + u[m, 2] * (math.log(100.0) - math.log(2.0)))
        pr = math.exp(math.log(2.0) + u[m, 3] * (math.log(1.0e4) - math.log(2.0)))
        gam = gams[min(2, int(u[m, 4] * 3))]
        r0 = 0.5 if kind == "sod" else 0.05
        pb = P.spherical_1d(kind, n1, gam, rho_ratio=rr, p_ratio=pr, r0=r0, cfl=0.8)
        pb = pb.copy(tmax=T_END[kind] * (0.5 + u[m, 5]))
        pb.name = "req%05d_%s" % (m, pb.name)
        out.append(pb)
    return out


def drive(server, reqs: list, rate: float, seed: int = 3, timeout: float = 600.0) -> dict:
    """Submit `reqs` to a started server with Poisson arrivals of `rate` requests per
    second (math.inf: all at once), wait for all of them and collect the results.
    Returns wall seconds from the first submission to the last completion, zone-updates,
    throughput and latency percentiles (seconds from submission to completion)."""
    n = len(reqs)
    if math.isinf(rate):
        arrivals = np.zeros(n)
    else:
        gaps = -np.log(1.0 - P.uniform01(seed, n)) / rate
        arrivals = np.cumsum(gaps) - gaps[0]
    ids = [None] * n
    t_sub = np.zeros(n)
    t0 = time.perf_counter()

    def client():
        for k in range(n):
            delay = arrivals[k] - (time.perf_counter() - t0)
            if delay > 0.0005:
                time.sleep(delay)
            t_sub[k] = time.perf_counter() - t0
            ids[k] = server.submit(reqs[k])

    th = threading.Thread(target=client)
    th.start()
    th.join()
    lat, zu, failed, last = [], 0.0, 0, 0.0
    for k in range(n):
        st = server.wait(ids[k], timeout=timeout)
        if st != 2:
            failed += 1
            continue
        _, t, ist, latency = server.result(ids[k])
        lat.append(latency)
        last = max(last, t_sub[k] + latency)
        zu += reqs[k].ncell * ist
    wall = last
    lat = np.asarray(lat)
    return {"rate_req_per_s": None if math.isinf(rate) else rate, "requests": n, "failed": failed,
            "wall_s": wall, "zone_updates": zu, "zone_updates_per_s": zu / wall,
            "latency_p50_s": float(np.percentile(lat, 50)) if lat.size else None,
            "latency_p99_s": float(np.percentile(lat, 99)) if lat.size else None,
            "offered_zone_updates_per_s": None if math.isinf(rate) else zu / n * rate}
