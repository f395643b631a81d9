"""The drop-in boundary end to end: the reference's own main.c (its input-file reader,
time loop with the dt rules of main.c:226-264, problem hooks, EOS fill and analysis
hooks) linked once with the reference's step.c and once with
medusa_b200/host/fornax_binding.c, which calls libmedusa_b200 instead
(oracle/build_ref.py, DROPIN).  Same input file, same binary apart from step.c: the final
states must agree to the FP64 sweep's bars (the drop-in run computes every step on the
GPU; only the host code around it is shared)."""
import numpy as np
import pytest

from tests._cases import record
from tests.test_dropin import run_dropin

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    out = 0.0
    vscale = max(np.abs(b[:, 2:5]).max(), 1.0e-300)
    for v in range(5):
        scale = vscale if v >= 2 else max(np.abs(b[:, v]).max(), 1.0e-300)
        out = max(out, float(np.abs(a[:, v] - b[:, v]).max() / scale))
    return out


@pytest.mark.parametrize("prob,inputs,n", [
    ("sod", dict(n1=1024, cfl=0.8, tmax=0.2), 1024),
    ("dust", dict(n1=200, cfl=0.9, tmax=0.004), 200),
    # problems/init_sedov.c on the 3-D dendritic grid with the default build maps
    # (SINH_MODIFIED radius, POLYTH theta; rtrans from the hook's own rtrans_solve)
    ("sedov3d", dict(n1=24, n2=16, n3=32, cfl=0.8, tmax=0.02), None),
])
def test_dropin_gpu_run_equals_reference_run(prob, inputs, n, tmp_path):
    ic, tc, pc, ec = run_dropin("cpu", prob, inputs, tmp_path, n)
    ig, tg, pg, eg = run_dropin("gpu", prob, inputs, tmp_path, n)
    e = rel_err(pg, pc)
    record("dropin_" + prob, steps=ic, err=e, bit_identical=float(np.mean(pg == pc)))
    assert ig == ic
    assert abs(tg - tc) <= 1.0e-12 * tc
    assert e <= 1.0e-9
    # the EOS records the GPU run hands back through update_cpu: pressure, sound speed, Gamma
    for v in (0, 1, 4):
        assert np.max(np.abs(eg[:, v] - ec[:, v]) / np.abs(ec[:, v])) <= 1.0e-9
