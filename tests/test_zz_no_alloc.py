"""mdg_advance_1d_noalloc: the 1-D advance for callers that cannot allocate device memory
(hosts whose device memory belongs to their own pool allocator, real-time loops that
cannot take cudaMalloc's synchronisation, embeddings with a fixed device footprint).

The caller owns the input and output buffers (here: torch tensors standing in for the
caller's own memory); the entry point keeps all its intermediate data in one static
device array.  Checked through the C ABI against the allocating entry points
(mdg_create + mdg_upload_state + mdg_step + mdg_download_state) and against the CPU
oracle, on several calls in a row with different problem sizes, so stale contents of
the shared array would show: spherical Sedov and Noh problems, a SINH radial map, a
Cartesian Sod tube with periodic and with reflecting boundaries run in place
(prim_in == prim_out), and the error statuses (a NaN in the initial state, a dtmin above
every possible step).

This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from medusa_b200 import problems as P
from medusa_b200 import solver as S
from oracle import pyoracle
from tests._cases import field_rel_err, pointwise_rel_err

pytestmark = pytest.mark.gpu

TOL = 1.0e-12        # the per-step parity bar of the other GPU tests, against the allocating ABI
ORACLE_TOL = 1.0e-9  # the whole-run bar of the other GPU tests, against the oracle
MAX_ZONES = 8192
NONFINITE = 11


def _noalloc_fn():
    L = S.library()
    f = L.mdg_advance_1d_noalloc
    f.argtypes = [ctypes.POINTER(S.ProblemDesc), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    f.restype = ctypes.c_int
    return f


def _with_allocating_abi(pb, nsteps):
    with S.Solver(pb) as s:
        s.step(nsteps)
        s.synchronize()
        prim = s.update_cpu(0)
        t, dt, _ = s.time(0)
    return prim, t, dt


def _call_noalloc(pb, nsteps, in_place=False):
    import torch
    f = _noalloc_fn()
    dev = torch.device("cuda", 0)
    # caller-owned device buffers, [var][zone]
    d_in = torch.from_numpy(np.ascontiguousarray(pb.ic.T)).to(dev)
    d_out = d_in if in_place else torch.full_like(d_in, float("nan"))
    stream = torch.cuda.current_stream(dev)
    t = ctypes.c_double(-1.0)
    dt = ctypes.c_double(-1.0)
    desc = S.desc_of(pb)
    rc = f(ctypes.byref(desc), d_in.data_ptr(), d_out.data_ptr(), nsteps, stream.cuda_stream,
           ctypes.byref(t), ctypes.byref(dt))
    torch.cuda.synchronize(dev)
    return rc, d_out.cpu().numpy().T.copy(), t.value, dt.value


def _with_noalloc_abi(pb, nsteps, in_place=False):
    rc, prim, t, dt = _call_noalloc(pb, nsteps, in_place)
    assert rc == 0, "mdg_advance_1d_noalloc returned %d" % rc
    return prim, t, dt


def _check_against_both(pb, n, in_place=False):
    ref, t_ref, dt_ref = _with_allocating_abi(pb, n)
    got, t_got, dt_got = _with_noalloc_abi(pb, n, in_place)
    assert np.all(np.isfinite(got)), pb.name
    assert field_rel_err(got, ref) <= TOL, pb.name
    assert pointwise_rel_err(got, ref, pb) <= TOL, pb.name
    assert abs(t_got - t_ref) <= TOL * t_ref, pb.name
    assert abs(dt_got - dt_ref) <= TOL * dt_ref, pb.name
    o = pyoracle.Oracle(pb)
    o.advance(n)
    oprim, _ = o.state()
    assert pointwise_rel_err(got, oprim, pb) <= ORACLE_TOL, pb.name
    assert abs(t_got - o.t) <= ORACLE_TOL * o.t, pb.name


def test_noalloc_matches_allocating_entry_points_twice():
    problems = [
        (P.spherical_1d("sedov", 1000, 1.4, p_ratio=1.0e4, r0=0.05), 25),
        (P.spherical_1d("noh", 300, 5.0 / 3.0), 40),
    ]
    for pb, n in problems:
        _check_against_both(pb, n)


def test_noalloc_sinh_radius_and_cartesian_in_place():
    """The SINH radial map, then Cartesian Sod tubes with periodic and with reflecting
    boundaries advanced in place (prim_in == prim_out), one call after the other."""
    sod = P.sod(400)
    cases = [
        (P.spherical_1d("sedov", 192, 1.4, p_ratio=1.0e4, r0=0.05, dr_min=2.0e-3), 30, False),
        (sod.copy(bc_lo=(P.PERIODIC, P.OUTFLOW, P.OUTFLOW), bc_hi=(P.PERIODIC, P.OUTFLOW, P.OUTFLOW),
                  name="sod_periodic"), 30, True),
        (sod.copy(bc_lo=(P.REFLECT, P.OUTFLOW, P.OUTFLOW), bc_hi=(P.REFLECT, P.OUTFLOW, P.OUTFLOW),
                  name="sod_reflect"), 30, True),
    ]
    for pb, n, in_place in cases:
        _check_against_both(pb, n, in_place)


def test_noalloc_reports_nonfinite_state_and_dt_below_dtmin():
    """A NaN in the initial state and a dtmin above every possible step return
    MDG_ERR_NONFINITE (as mdg_synchronize does for the allocating path); a good call
    afterwards succeeds and is unaffected by the failed ones' leftovers."""
    pb = P.spherical_1d("sedov", 200, 1.4, p_ratio=1.0e3, r0=0.1)
    ic = np.array(pb.ic)
    ic[17, 1] = np.nan
    rc, _, _, _ = _call_noalloc(pb.copy(ic=ic, name="sedov_nan"), 5)
    assert rc == NONFINITE
    rc, _, _, _ = _call_noalloc(P.sod(128).copy(dtmin=1.0), 1)
    assert rc == NONFINITE
    _check_against_both(pb, 10)


def test_noalloc_rejects_problems_beyond_the_scratch():
    f = _noalloc_fn()
    pb = P.sod(MAX_ZONES + 1)
    desc = S.desc_of(pb)
    dummy = ctypes.c_double(0.0)
    rc = f(ctypes.byref(desc), ctypes.addressof(dummy), ctypes.addressof(dummy), 1, None, None, None)
    assert rc == 6   # MDG_ERR_OUTOFMEM: does not fit the fixed scratch
