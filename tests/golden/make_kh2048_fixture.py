"""Regenerate tests/golden/kh2048_200.npz: the Kelvin-Helmholtz 2048 x 2048 workload run
for 200 steps by the UNMODIFIED reference (the parity build of oracle/build_ref.py,
single-threaded; about 20-25 minutes of CPU).

The full final state is 168 MB, so the fixture keeps what a GPU test needs to judge a
run of the same 200 steps without it:
  * the SHA-256 of the initial state (the test checks it starts from the same bits) and
    of the final state ([zone][5] float64, zone order): equal digests mean every value
    of the GPU's final state is bit-identical to the reference's;
  * the final state of the zones (16a, 16b): every 16th zone of every 16th row;
  * per variable, the sum over every row and over every column of the final state, so
    a difference anywhere on the grid shows in one row sum and one column sum;
  * t, dt and min_dt after 50, 100, 150 and 200 steps.

    python tests/golden/make_kh2048_fixture.py
"""
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from medusa_b200 import problems as P  # noqa: E402
from oracle import build_ref, pyoracle  # noqa: E402

N = 2048
STEPS = 200
EVERY = 50
STRIDE = 16
OUT = os.path.join(HERE, "kh2048_200.npz")


def sha256_of(prim) -> str:
    return hashlib.sha256(np.ascontiguousarray(prim, dtype=np.float64).tobytes()).hexdigest()


def reduce_state(prim, n1, n2, stride=STRIDE):
    """(sampled zones [n1/stride, n2/stride, 5], row sums [n1, 5], column sums [n2, 5]) of a
    [zone][5] state in the reference's i-major zone order."""
    g = np.asarray(prim, dtype=np.float64).reshape(n1, n2, 5)
    return g[::stride, ::stride, :].copy(), g.sum(axis=1), g.sum(axis=0)


def main():
    build_ref.build()
    pb = P.kelvin_helmholtz(N)
    t0 = time.time()
    snaps = pyoracle.run_reference(pb, STEPS, every=EVERY)
    wall = time.time() - t0
    first, last = snaps[0], snaps[-1]
    sample, rows, cols = reduce_state(last[4], N, N)
    np.savez_compressed(OUT, ic_sha256=sha256_of(first[4]), final_sha256=sha256_of(last[4]),
                        sample=sample, stride=STRIDE, row_sums=rows, col_sums=cols,
                        steps=np.array([s[0] for s in snaps[1:]]), t=np.array([s[1] for s in snaps[1:]]),
                        dt=np.array([s[2] for s in snaps[1:]]), min_dt=np.array([s[3] for s in snaps[1:]]),
                        reference_wall_s=wall)
    print("kh2048: %d steps, t %.6e, %.0f s of reference CPU time -> %s" % (last[0], last[1], wall,
                                                                          os.path.relpath(OUT, ROOT)))


if __name__ == "__main__":
    main()
