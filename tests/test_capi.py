"""The C ABI library without a GPU: it loads, exports every entry point that
include/medusa_b200.h declares, and rejects bad input before touching the device."""
import ctypes
import os
import re

import pytest

from medusa_b200 import problems as P
from medusa_b200 import solver as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "medusa_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(mdg_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_abi():
    names = declared_functions()
    for required in ("mdg_create", "mdg_upload_state", "mdg_estimate_dt", "mdg_step",
                     "mdg_download_state", "mdg_destroy"):
        assert required in names


def test_library_exports_every_declared_symbol():
    L = S.library()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_error_strings_and_version():
    L = S.library()
    for code in range(0, 12):
        assert L.mdg_error_string(code)
    assert L.mdg_version() >= 100


@pytest.mark.parametrize("mutate,code", [
    (dict(ndim=4), 1),
    (dict(ndim=3), 5),                                # 3-D grids are spherical (dendritic)
    (dict(hydro_interp_order=4), 1),
    (dict(gam=1.0), 1),
    (dict(bc_lo=(P.SPHERICAL_ORIGIN, 0, 0)), 5),      # spherical origin on a Cartesian grid
    (dict(bc_lo=(P.PERIODIC, 0, 0)), 1),              # unpaired periodic boundary
])
def test_create_rejects_invalid_descriptions(mutate, code):
    """Checked before any device work (runs without a GPU)."""
    pb = P.sod(64).copy(**mutate)
    arr = (S.ProblemDesc * 1)(S.desc_of(pb))
    h = ctypes.c_void_p()
    rc = S.library().mdg_create(arr, 1, 0, 0, ctypes.byref(h))
    assert rc == code
    assert not h.value
    assert S.library().mdg_last_error_message()


def test_null_handles_are_rejected():
    L = S.library()
    assert L.mdg_step(None, 1) == 1
    assert L.mdg_synchronize(None) == 1
    assert L.mdg_destroy(None) == 0


@pytest.mark.parametrize("pb", [P.sod(64).copy(hydro_interp_order=2),
                                P.kelvin_helmholtz(16, 16, nsteps=1).copy(hydro_interp_order=1)],
                         ids=["linear", "2d_pcm"])
def test_mixed_precision_scope_is_checked_before_any_device_work(pb):
    """The mixed sweeps are built for parabolic reconstruction: other problems are
    refused with MDG_ERR_NOTIMPL (validation runs before any CUDA call)."""
    arr = (S.ProblemDesc * 1)(S.desc_of(pb))
    h = ctypes.c_void_p()
    rc = S.library().mdg_create(arr, 1, S.PREC_MIXED, 0, ctypes.byref(h))
    assert rc == 5
    assert not h.value
    assert b"mixed" in S.library().mdg_last_error_message()


def test_unknown_precision_is_rejected():
    arr = (S.ProblemDesc * 1)(S.desc_of(P.sod(64)))
    h = ctypes.c_void_p()
    assert S.library().mdg_create(arr, 1, 7, 0, ctypes.byref(h)) == 1


def test_launch_config_calls_reject_null_solver():
    L = S.library()
    c = S.LaunchConfig(128, 0, 10, 16, 1, 1)
    assert L.mdg_get_launch_config(None, ctypes.byref(c)) == 1
    assert L.mdg_set_launch_config(None, ctypes.byref(c)) == 1
    assert L.mdg_autotune(None, 3, None, None) == 1
    assert L.mdg_conserved_totals(None, None, None) == 1
    assert L.mdg_set_time(None, 0, 0.0, 0) == 1
    assert L.mdg_restart_write(None, 0, b"x") == 1
    assert L.mdg_restart_read(None, 0, b"x") == 1
    assert L.mdg_write_timers(None, 0, b"x") == 1
    n = ctypes.c_int()
    assert L.mdg_resident_cluster(None, ctypes.byref(n)) == 1


@pytest.mark.parametrize("field,value", [("precision", 7), ("max_problems", 0), ("max_zones", 2),
                                         ("steps_per_round", 0), ("threads", 96), ("hbm_bytes", 1000),
                                         ("hbm_bytes_2d", -1), ("hbm_bytes_2d", 1 << 20)])
def test_server_config_is_checked_before_any_device_work(field, value):
    c = S.ServerConfig(0, S.PREC_MIXED, 1 << 30, 64, 4096, 10, 64, 0)
    setattr(c, field, value)
    h = ctypes.c_void_p()
    assert S.library().mdg_server_create(ctypes.byref(c), ctypes.byref(h)) == 1
    assert not h.value
    assert S.library().mdg_last_error_message()


def test_server_calls_reject_null_handle():
    L = S.library()
    st = ctypes.c_int()
    assert L.mdg_server_poll(None, 1, ctypes.byref(st)) == 1
    assert L.mdg_server_run(None, 1, None) == 1
    assert L.mdg_server_start(None) == 1
    assert L.mdg_server_stop(None) == 1
    assert L.mdg_server_destroy(None) == 0


@pytest.mark.parametrize("precision,nprob,order,code", [(1, 1, 2, 5), (0, 2, 3, 5)])
def test_3d_solver_scope_checked_before_device_work(precision, nprob, order, code):
    """A 3-D solver advances one problem; its mixed-precision sweep is parabolic only."""
    pb = P.sedov_3d(12, 8, 16, r_dep=0.3).copy(hydro_interp_order=order)
    arr = (S.ProblemDesc * nprob)(*[S.desc_of(pb)] * nprob)
    h = ctypes.c_void_p()
    assert S.library().mdg_create(arr, nprob, precision, 0, ctypes.byref(h)) == code
    assert not h.value


def test_output_calls_reject_null_solver():
    L = S.library()
    assert L.mdg_snapshot(None, 0) == 1
    assert L.mdg_snapshot_read(None, None, None, None) == 1
    assert L.mdg_snapshot_write_ascii1(None, b"x") == 1
    assert L.mdg_dump_ascii1(None, 0, b"x") == 1


@pytest.mark.parametrize("mutate,nprob,code", [
    (dict(n=(24, 12, 1)), 1, 1),                        # n2 not a power of two
    (dict(n=(24, 16, 4)), 1, 1),                        # a 2-D grid has one phi zone
    (dict(dx=(1.0 / 24, 2.0 / 16, 1.0)), 1, 1),         # its phi zone spans 2 pi
    (dict(startx=(0.0, -0.5, 0.0)), 1, 1),              # theta over the whole sphere
    (dict(), 2, 5),                                     # one problem per dendritic solver
])
def test_2d_spherical_scope_checked_before_device_work(mutate, nprob, code):
    """2-D (r, theta) spherical problems run on the dendritic grid: its geometry rules
    are checked before any device work."""
    pb = P.sedov_2d_spherical(24, 16, r_dep=0.3).copy(**mutate)
    arr = (S.ProblemDesc * nprob)(*[S.desc_of(pb)] * nprob)
    h = ctypes.c_void_p()
    assert S.library().mdg_create(arr, nprob, 0, 0, ctypes.byref(h)) == code
    assert not h.value
    assert S.library().mdg_last_error_message()


@pytest.mark.parametrize("pb,precision,code", [
    (P.sod(64).copy(rcoord=P.RCOORD_SINH, rtrans=0.2), 0, 1),                        # Cartesian
    (P.spherical_1d("sedov", 64, 1.4, dr_min=0.01).copy(rtrans=-1.0), 0, 1),         # rtrans <= 0
    (P.spherical_1d("sedov", 64, 1.4).copy(rcoord=7), 0, 1),                          # unknown map
    (P.spherical_1d("noh", 64, 1.4).copy(rcoord=P.RCOORD_SINH, rtrans=0.2), 0, 5),    # Noh inflow boundary
    (P.spherical_1d("sedov", 64, 1.4).copy(thcoord=3), 0, 1),                         # unknown theta map
    (P.sod(64).copy(thcoord=P.THCOORD_POLYTH), 0, 1),                                 # Cartesian
    (P.spherical_1d("sedov", 64, 1.4).copy(thcoord=P.THCOORD_POLYTH, poly_xt=0.0), 0, 1),
    (P.spherical_1d("sedov", 64, 1.4, dr_min=0.01, coords="default").copy(rfact=(1.0e6, 1.5e6, 0.0)), 0, 1),
])
def test_radial_map_scope_checked_before_device_work(pb, precision, code):
    arr = (S.ProblemDesc * 1)(S.desc_of(pb))
    h = ctypes.c_void_p()
    assert S.library().mdg_create(arr, 1, precision, 0, ctypes.byref(h)) == code
    assert not h.value
