"""The reference's own timers on the CPU (oracle/_ref reftime_<cfg> builds, DO_TIMING=TRUE):
timing.csv in the io.c:51-108 columns, with the cycle counts that step.c's TIMER_START /
TIMER_STOP sites imply for an RK2 step (one step and one estimate_dt per step; two
prim_to_fluxes and push calls, one per stage)."""
import os

import pytest

from medusa_b200 import problems as P
from oracle import pyoracle


def _need(pb):
    if not os.path.exists(os.path.join(pyoracle.REF_DIR, "reftime_" + pyoracle.ref_config(pb))):
        pytest.skip("reftime build absent (python oracle/build_ref.py)")


@pytest.mark.parametrize("pb,sweep", [(P.sod(128), "prim_to_fluxes1"), (P.kelvin_helmholtz(32), "prim_to_fluxes2")],
                         ids=["cart1d", "cart2d"])
def test_reference_timers_count_the_phases_of_the_timed_steps(pb, sweep):
    _need(pb)
    r = pyoracle.time_reference_phases(pb, 3, 10)
    tm = r["timers"]
    assert tm["step"][1] == 10 and tm["estimate_dt"][1] == 10
    assert tm[sweep][1] == 20 and tm["push"][1] == 20
    assert tm["step"][0] >= tm[sweep][0] + tm["push"][0] > 0.0
    assert r["steps"] == 10 and r["cells"] == pb.ncell
