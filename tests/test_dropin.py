"""The reference's own main.c driving a problem end to end (oracle/build_ref.py, DROPIN):
the CPU build (main.c + the reference's step.c + oracle/refshim/dropin_glue.c) against
the harness run of the same problem, so that the glue -- the input-file reader and the
restated problem hooks -- is pinned before the drop-in GPU build
(medusa_b200/host/fornax_binding.c in place of step.c) is compared with it on a GPU
(tests/test_gpu_dropin.py)."""
import os
import struct
import subprocess

import numpy as np
import pytest

from medusa_b200 import problems as P
from oracle import pyoracle

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def run_dropin(kind, prob, inputs, tmp_path, n):
    exe = os.path.join(REF, "dropin_%s_%s" % (kind, prob))
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref drop-in builds absent (need the reference tree)")
    inp = tmp_path / ("input." + prob)
    inp.write_text("".join("%s = %s\n" % kv for kv in inputs.items()) + "# comment line\n")
    out = tmp_path / ("%s_%s.bin" % (kind, prob))
    env = dict(os.environ, DROPIN_OUT=str(out))
    subprocess.run([exe, str(inp)], check=True, cwd=tmp_path, env=env, stdout=subprocess.DEVNULL,
                   stderr=subprocess.DEVNULL, timeout=600)
    b = out.read_bytes()
    istep = struct.unpack("i", b[:4])[0]
    t = struct.unpack("d", b[4:12])[0]
    if n is None:
        n = (len(b) - 12) // 80
    a = np.frombuffer(b[12:], dtype=np.float64).reshape(2, n, 5)
    return istep, t, a[0].copy(), a[1].copy()


def test_reference_main_sod_matches_harness(tmp_path):
    """main.c's loop with the input file n1 = 256, cfl = 0.8, tmax = 0.05 against the
    harness's restatement of the same loop on P.sod(256): the same state, bit for bit."""
    istep, t, prim, _ = run_dropin("cpu", "sod", dict(n1=256, cfl=0.8, tmax=0.05), tmp_path, 256)
    pb = P.sod(256).copy(cfl=0.8, tmax=0.05)
    if not pyoracle.ref_available(pb):
        pytest.skip("oracle/_ref not built")
    last = pyoracle.run_reference(pb, istep, every=istep)[-1]
    assert last[0] == istep
    assert last[1] == t
    assert np.array_equal(last[4], prim)


def test_reference_main_dust_collapse_matches_harness(tmp_path):
    """The dust collapse (monopole gravity, SINH radius, floors, the outer v^r hook) with
    the hook's own rtrans_solve: the harness run with that rtrans gives the same state."""
    istep, t, prim, _ = run_dropin("cpu", "dust", dict(n1=200, cfl=0.9, tmax=0.002), tmp_path, 200)
    pb = P.dust_collapse(200).copy(tmax=0.002)
    if not pyoracle.ref_available(pb):
        pytest.skip("oracle/_ref not built")
    last = pyoracle.run_reference(pb, istep, every=istep)[-1]
    assert last[0] == istep
    # rtrans: the hook's rtrans_solve and problems.sinh_rtrans agree to their 1e-10 bisection
    assert abs(last[1] - t) <= 1.0e-8 * t
    assert np.max(np.abs(last[4] - prim) / np.maximum(np.abs(prim), 1.0e-300)) <= 1.0e-6
