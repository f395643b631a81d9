"""Tabulated EOS inputs: the grid of the reference's nuclear EOS table and a seeded
synthetic table in its layout.

The reference reads a binary table (eos/burrows/eos_stuff.c:112-116) that is not part of
its source tree; its layout is TAB_ELEM (eos_stuff.c:7): `nrec` records of ny x nr x nt
doubles, jt fastest, on a grid uniform in log10 rho [r1, r2], log10 T (MeV) [t1, t2] and
Ye [y1, y2] with the sizes and bounds of DEFINE_EOSCONST_1 (eos_stuff.c:8-21: 16 records,
ny = 50, nr = 300, nt = 300, r 1 .. 15.5, t -2 .. 2, Ye 0.035 .. 0.56).  The synthetic
table fills the four records the zone update reads -- 1 energy (increasing in T, as the
temperature search needs), 2 log pressure, 3 entropy, 12 Gamma_1 -- with smooth functions
of the grid coordinates; the others are zero.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from .problems import uniform01

ERG_PER_UNIT = 0.95655684e18    # eos_stuff.c:784: e_eos = (u / rho) / 0.95655684e18 - const_hack


@dataclass(frozen=True)
class EosGrid:
    nrec: int = 16
    ny: int = 50
    nr: int = 300
    nt: int = 300
    r1: float = 1.0
    r2: float = 15.5
    t1: float = -2.0
    t2: float = 2.0
    y1: float = 0.035
    y2: float = 0.56
    const_hack: float = 0.0

    def axes(self):
        """log10 rho, log10 T and Ye at the table's grid points (as the reference's
        r1 + (jr-1) dr etc.)."""
        dr = (self.r2 - self.r1) / (self.nr - 1)
        dt = (self.t2 - self.t1) / (self.nt - 1)
        dy = (self.y2 - self.y1) / (self.ny - 1)
        return (self.r1 + np.arange(self.nr) * dr, self.t1 + np.arange(self.nt) * dt,
                self.y1 + np.arange(self.ny) * dy)


REFERENCE_GRID = EosGrid()


def synthetic_table(g: EosGrid = REFERENCE_GRID) -> np.ndarray:
    """A table of g's sizes in the reference layout: array [nrec][ny][nr][nt] (flattened
    it is TAB_ELEM's order)."""
    rl, tl, ye = g.axes()
    Y = ye[:, None, None]
    R = rl[None, :, None]
    T = tl[None, None, :]
    tab = np.zeros((g.nrec, g.ny, g.nr, g.nt))
    tab[0] = 2.0 + 0.3 * Y + 0.05 * R + 1.5 * (10.0 ** T) * (1.0 + 0.1 * np.sin(3.0 * R))   # energy
    tab[1] = -10.0 + 1.2 * R + 0.8 * T + 0.5 * Y + 0.02 * np.cos(2.0 * R + 5.0 * Y)       # log pressure
    tab[2] = 1.0 + 2.0 * T + 0.1 * R + Y                                                 # entropy
    if g.nrec >= 12:
        tab[11] = 1.3 + 0.05 * np.sin(R) + 0.1 * Y + 0.02 * T                           # Gamma_1
    return tab


def synthetic_zones(g: EosGrid, n: int, seed: int = 11, table: np.ndarray = None):
    """n zones inside the table: log10 rho, Ye and a target log10 T uniform inside the
    grid, the internal energy density u whose energy the table (bilinear in log rho and Ye,
    linear in T between rows) puts at that temperature, and a temperature guess drawn
    independently (the zone update starts its search at the guess's row).  Returns
    (rho, u, ye, temp_guess)."""
    tab = synthetic_table(g) if table is None else table
    w = uniform01(seed, 4 * n).reshape(n, 4)
    span = lambda a, b, x: a + (b - a) * (0.002 + 0.996 * x)
    rl = span(g.r1, g.r2, w[:, 0])
    ye = span(g.y1, g.y2, w[:, 1])
    tl = span(g.t1, g.t2, w[:, 2])
    tg = span(g.t1, g.t2, w[:, 3])
    dr = (g.r2 - g.r1) / (g.nr - 1)
    dt = (g.t2 - g.t1) / (g.nt - 1)
    dy = (g.y2 - g.y1) / (g.ny - 1)
    jr = np.minimum(((rl - g.r1) / dr).astype(int), g.nr - 2)
    jy = np.minimum(((ye - g.y1) / dy).astype(int), g.ny - 2)
    jt = np.minimum(((tl - g.t1) / dt).astype(int), g.nt - 2)
    fr = (rl - (g.r1 + jr * dr)) / dr
    fy = (ye - (g.y1 + jy * dy)) / dy
    ft = (tl - (g.t1 + jt * dt)) / dt
    E = tab[0]

    def at(k):
        return ((1 - fr) * (1 - fy) * E[jy, jr, k] + fy * (1 - fr) * E[jy + 1, jr, k]
                + (1 - fy) * fr * E[jy, jr + 1, k] + fy * fr * E[jy + 1, jr + 1, k])
    e = (1 - ft) * at(jt) + ft * at(jt + 1)
    rho = 10.0 ** rl
    u = rho * (e + g.const_hack) * ERG_PER_UNIT
    return rho, u, ye, 10.0 ** tg


class EosGridC(ctypes.Structure):
    """The grid as the C ABI takes it (mdg_eos_grid of include/medusa_b200.h)."""
    _fields_ = [("nrec", ctypes.c_int), ("ny", ctypes.c_int), ("nr", ctypes.c_int), ("nt", ctypes.c_int),
                ("r1", ctypes.c_double), ("r2", ctypes.c_double), ("t1", ctypes.c_double),
                ("t2", ctypes.c_double), ("y1", ctypes.c_double), ("y2", ctypes.c_double),
                ("const_hack", ctypes.c_double)]

    @classmethod
    def of(cls, g: EosGrid) -> "EosGridC":
        return cls(g.nrec, g.ny, g.nr, g.nt, g.r1, g.r2, g.t1, g.t2, g.y1, g.y2, g.const_hack)


class EosTable:
    """A tabulated EOS on the device (mdg_eos_table_create); given_rex runs the zone
    update of eos_given_rex_per_zone (eos/burrows/eos_stuff.c:768-902) for many zones."""

    def __init__(self, table: np.ndarray, grid: EosGrid = REFERENCE_GRID, device: int = 0):
        from .solver import _check, library
        L = library()
        _declare(L)
        t = np.ascontiguousarray(table, dtype=np.float64)
        if t.size != grid.nrec * grid.ny * grid.nr * grid.nt:
            raise ValueError("table size does not match the grid")
        self._h = ctypes.c_void_p()
        gc = EosGridC.of(grid)
        _check(L.mdg_eos_table_create(ctypes.byref(gc), t.ctypes.data, int(device), ctypes.byref(self._h)),
               "mdg_eos_table_create")
        self.grid = grid

    def given_rex(self, rho, u, ye, temp_guess):
        """Host arrays in, (temp, press, cs, ent, gam1) out."""
        from .solver import _check, library
        cols = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, ye)]
        n = cols[0].size
        temp = np.array(temp_guess, dtype=np.float64, copy=True).reshape(n)
        outs = [np.empty(n) for _ in range(4)]
        _check(library().mdg_eos_given_rex_host(self._h, n, *[c.ctypes.data for c in cols], temp.ctypes.data,
                                                *[o.ctypes.data for o in outs]), "mdg_eos_given_rex_host")
        return (temp,) + tuple(outs)

    def given_rex_device(self, n: int, rho: int, u: int, ye: int, temp: int, press: int, cs: int, ent: int,
                         gam1: int, stream: int = 0):
        """Device pointers (e.g. torch tensors' data_ptr()); queued on `stream`."""
        from .solver import _check, library
        _check(library().mdg_eos_given_rex(self._h, int(n), rho, u, ye, temp, press, cs, ent, gam1, stream),
               "mdg_eos_given_rex")

    def close(self):
        if self._h:
            from .solver import library
            library().mdg_eos_table_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _declare(L):
    vp, ll = ctypes.c_void_p, ctypes.c_longlong
    L.mdg_eos_table_create.argtypes = [ctypes.POINTER(EosGridC), vp, ctypes.c_int, ctypes.POINTER(vp)]
    L.mdg_eos_table_destroy.argtypes = [vp]
    L.mdg_eos_given_rex.argtypes = [vp, ll] + [vp] * 8 + [vp]
    L.mdg_eos_given_rex_host.argtypes = [vp, ll] + [vp] * 8
    for name in ("mdg_eos_table_create", "mdg_eos_table_destroy", "mdg_eos_given_rex", "mdg_eos_given_rex_host"):
        getattr(L, name).restype = ctypes.c_int

