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
