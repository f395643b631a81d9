"""Shared test cases: the golden fixture set and helpers to compare states."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402

GOLDEN_DIR = os.path.join(HERE, "golden")


def golden_cases():
    return make_golden.cases()


def golden_cases3d():
    return make_golden.cases3d()


def golden_cases_gravity():
    return make_golden.cases_gravity()


def load_golden(name):
    return np.load(os.path.join(GOLDEN_DIR, name + ".npz"))


def max_rel_diff(a, b, floor=1.0e-300):
    """max |a-b| / max(|a|,|b|) over entries, treating +0 and -0 as equal."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    num = np.abs(a - b)
    den = np.maximum(np.maximum(np.abs(a), np.abs(b)), floor)
    r = num / den
    r[num == 0] = 0.0
    return float(r.max()) if r.size else 0.0


def field_rel_err(a, b):
    """Largest per-variable error max|a-b| / max(|a|,|b|) over the whole field: the
    error relative to each primitive variable's scale (velocity components that vanish
    by symmetry carry round-off, where an entrywise ratio is meaningless)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    worst = 0.0
    for v in range(a.shape[1]):
        scale = max(np.abs(a[:, v]).max(), np.abs(b[:, v]).max())
        d = np.abs(a[:, v] - b[:, v]).max()
        worst = max(worst, d / scale if scale > 0 else d)
    return float(worst)


def pointwise_rel_err(a, ref, pb, gcov=None):
    """Largest zone-by-zone relative error of state a against ref (both [zone][5]):
      * density and internal energy: |a - ref| / |ref| at every zone (no field scale; a
        zone of the ambient medium counts as much as one inside the blast);
      * velocities: the error of each physical component, |a_k - ref_k| sqrt(g_kk), over
        the zone's own speed scale max(|v|, c_s) (|v| the physical speed of ref, c_s its
        sound speed sqrt(Gamma P / rho)); a component that is zero by symmetry has no
        scale of its own, so the zone's signal speed stands in for it.
    gcov: zone-centred metric diagonal [zone][3] (dendritic grids); None means unit
    factors (Cartesian grids; the radial component of 1-D spherical ones).  Entries
    equal on both sides (+0 and -0 included) count as zero error."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(ref, dtype=np.float64)
    out = 0.0
    for v in (0, 1):
        num = np.abs(a[:, v] - b[:, v])
        den = np.maximum(np.abs(b[:, v]), 1.0e-300)
        r = np.where(num == 0, 0.0, num / den)
        out = max(out, float(r.max()) if r.size else 0.0)
    g = np.ones((b.shape[0], 3)) if gcov is None else np.asarray(gcov, dtype=np.float64)
    rho = np.maximum(np.abs(b[:, 0]), 1.0e-300)
    if pb.eos == 0:
        press = (pb.gam - 1.0) * b[:, 1]
    else:
        press = pb.Kpoly * np.power(np.abs(b[:, 0]), pb.gam)
    cs = np.sqrt(np.maximum(pb.gam * press / rho, 0.0))
    sq = np.sqrt(np.abs(g))
    vphys = np.sqrt(np.sum((b[:, 2:5] * sq) ** 2, axis=1))
    scale = np.maximum(np.maximum(vphys, cs), 1.0e-300)
    for k in range(3):
        num = np.abs(a[:, 2 + k] - b[:, 2 + k]) * sq[:, k]
        r = np.where(num == 0, 0.0, num / scale)
        out = max(out, float(r.max()) if r.size else 0.0)
    return out


def zone_gcov(pb):
    """The metric diagonal pointwise_rel_err needs: the library's per-zone gcov on the
    dendritic spherical grids (3-D, and 2-D spherical), unit factors otherwise."""
    if pb.ndim == 3 or (pb.ndim == 2 and pb.geom == 1):
        from medusa_b200.solver import grid3d_zone_gcov
        return grid3d_zone_gcov(pb)
    return None


def bit_identical_fraction(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.mean((a == b) | (np.isnan(a) & np.isnan(b))))


def record(name, **kw):
    """Append a measurement to $MDG_PARITY_LOG (JSON lines) when that is set."""
    import json
    import os
    path = os.environ.get("MDG_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(dict(case=name, **kw)) + "\n")
