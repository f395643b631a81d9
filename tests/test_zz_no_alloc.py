"""mdg_advance_1d_noalloc: the 1-D advance for callers that cannot allocate device memory
(hosts whose device memory belongs to their own pool allocator, real-time loops that
cannot take cudaMalloc's synchronisation, embeddings with a fixed device footprint).

The caller owns the input and output buffers (here: torch tensors standing in for the
caller's own memory); the entry point keeps all its intermediate data in one static
device array.  Checked through the C ABI against the allocating entry points
(mdg_create + mdg_upload_state + mdg_step + mdg_download_state) on two calls in a row,
with different problem sizes, so stale contents of the shared array would show.

This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from medusa_b200 import problems as P
from medusa_b200 import solver as S
from tests._cases import field_rel_err

pytestmark = pytest.mark.gpu

TOL = 1.0e-12   # the per-step parity bar of the other GPU tests (field-relative)
MAX_ZONES = 8192


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


def _with_noalloc_abi(pb, nsteps):
    import torch
    f = _noalloc_fn()
    dev = torch.device("cuda", 0)
    # caller-owned device buffers, [var][zone]
    d_in = torch.from_numpy(np.ascontiguousarray(pb.ic.T)).to(dev)
    d_out = torch.full_like(d_in, float("nan"))
    stream = torch.cuda.current_stream(dev)
    t = ctypes.c_double(-1.0)
    dt = ctypes.c_double(-1.0)
    desc = S.desc_of(pb)
    rc = f(ctypes.byref(desc), d_in.data_ptr(), d_out.data_ptr(), nsteps, stream.cuda_stream,
           ctypes.byref(t), ctypes.byref(dt))
    assert rc == 0, "mdg_advance_1d_noalloc returned %d" % rc
    torch.cuda.synchronize(dev)
    return d_out.cpu().numpy().T.copy(), t.value, dt.value


def test_noalloc_matches_allocating_entry_points_twice():
    problems = [
        (P.spherical_1d("sedov", 1000, 1.4, p_ratio=1.0e4, r0=0.05), 25),
        (P.spherical_1d("noh", 300, 5.0 / 3.0), 40),
    ]
    for pb, n in problems:
        ref, t_ref, dt_ref = _with_allocating_abi(pb, n)
        got, t_got, dt_got = _with_noalloc_abi(pb, n)
        assert np.all(np.isfinite(got))
        assert field_rel_err(got, ref) <= TOL, pb.name
        assert abs(t_got - t_ref) <= TOL * t_ref
        assert abs(dt_got - dt_ref) <= TOL * dt_ref


def test_noalloc_rejects_problems_beyond_the_scratch():
    f = _noalloc_fn()
    pb = P.sod(MAX_ZONES + 1)
    desc = S.desc_of(pb)
    dummy = ctypes.c_double(0.0)
    rc = f(ctypes.byref(desc), ctypes.addressof(dummy), ctypes.addressof(dummy), 1, None, None, None)
    assert rc == 6   # MDG_ERR_OUTOFMEM: does not fit the fixed scratch
