"""Problem setups: the host-side counterpart of the reference's problems/init_*.c hooks.

Each function returns a :class:`Problem`: the grid, the physics switches that the
reference fixes at compile time (setups/*.mk -> build.h) and reads from its input.*
files, and the initial primitive state of the interior zones in the reference's zone
order (i-major: ``ic[(i*n2 + j), :]`` holds rho, u (internal energy density), v1, v2, v3,
with v^d the contravariant coordinate velocities).

The setups follow the reference files they cite but use the sizes, parameters and
initial conditions of the workloads this library is measured on (Sod 1024 zones,
Kelvin-Helmholtz 2048^2, ensembles of 1-D spherical Sod/Noh/Sedov problems).  All
random numbers come from splitmix64 (Steele, Lea & Flood 2014) on a caller-given seed,
so the same seed gives the same bits on every host.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

# geometry ids (decs.h:669-671)
CARTESIAN = 0
SPHERICAL = 1
# EOS ids (decs.h:674-675)
GAMMA_LAW = 0
POLYTROPIC = 1
# boundary kinds (decs.h:64-69)
OUTFLOW = 0
REFLECT = 1
EXTRAP = 2
PERIODIC = 3
PROB = 4
SPHERICAL_ORIGIN = 5
# problem-specific PROB boundary hooks
PROB_NONE = 0
PROB_NOH = 1
PROB_DUST = 2               # problems/init_dustcollapse.c:104-113 (outer v^r hook)

RCOORD_UNIFORM = 0          # radial maps r(x), metric_spherical_general.c:149-219
RCOORD_SINH = 1
RCOORD_SINH_MODIFIED = 2
RCOORD_LOG = 3              # r = rtrans exp(|x|/rtrans): log-spaced from r = rtrans (not a reference map)
THCOORD_UNIFORM = 0         # theta maps th(x), metric_spherical_general.c:222-290
THCOORD_POLYTH = 1
RFACT_DEFAULT = (10 * 1e5, 15 * 1e5, 5 * 1e5)   # rx_info.facta/b/c, io.c:5008-5010
POLY_XT_DEFAULT, POLY_ALPHA_DEFAULT = 1.2, 4.0  # thx_info, io.c:5014-5015

NG = 2
NPRIM = 5


@dataclasses.dataclass
class Problem:
    """A hydro problem: grid, physics switches, run controls and initial state."""
    name: str
    ndim: int
    geom: int
    n: tuple                      # (n1, n2, n3) interior zones
    startx: tuple                 # coordinate of the lower edge of zone 0 per direction
    dx: tuple                     # coordinate spacing per direction
    gam: float
    ic: np.ndarray                # [n1*n2*n3, 5] float64, i-major
    Kpoly: float = 1.0
    eos: int = GAMMA_LAW
    bc_lo: tuple = (OUTFLOW, OUTFLOW, OUTFLOW)
    bc_hi: tuple = (OUTFLOW, OUTFLOW, OUTFLOW)
    prob_kind: int = PROB_NONE
    cfl: float = 0.9              # io.c:5018 default
    dt_init_safety: float = 0.1   # io.c:5036
    dt_grow_safety: float = 1.1   # io.c:5035
    initial_dt: float = 1.0e100   # io.c:5063
    dtmax: float = 1.0e200        # io.c:5037
    dtmin: float = 1.0e-200       # io.c:5038
    tmax: float = 1.0e100
    rcoord: int = RCOORD_UNIFORM  # radial map of a spherical grid (the RCOORD build switch)
    rtrans: float = 1.0           # its transition radius (RCOORD_SINH, RCOORD_SINH_MODIFIED)
    rfact: tuple = RFACT_DEFAULT  # facta, factb, factc of RCOORD_SINH_MODIFIED
    thcoord: int = THCOORD_UNIFORM  # theta map of a spherical grid (the THCOORD build switch)
    poly_xt: float = POLY_XT_DEFAULT
    poly_alpha: float = POLY_ALPHA_DEFAULT
    monopole: int = 0             # self-gravity, monopole approximation (GRAV=SPHERICAL_MONOPOLE_GRAV)
    hydro_interp_order: int = 3   # io.c:5055
    enforce_floors: int = 0       # ENFORCE_FLOORS build switch (fluid.c:43-46)
    rho_floor: float = -1.0       # io.c:5082 default; problem hooks set their own
    e_floor: float = -1.0         # io.c:5081
    grav: tuple = (0.0, 0.0, 0.0) # fixed gravitational acceleration g0 (GRAV=FIXED_GRAV when non-zero)
    nsteps: Optional[int] = None  # fixed step count for the workload, if any
    cells: int = 0                # interior zone count when it is not n1*n2*n3 (dendritic grids)

    @property
    def ncell(self) -> int:
        if self.cells > 0:
            return int(self.cells)
        return int(self.n[0] * self.n[1] * self.n[2])

    def copy(self, **kw) -> "Problem":
        d = dataclasses.asdict(self)
        d["ic"] = self.ic.copy()
        d.update(kw)
        return Problem(**d)


# ----------------------------------------------------------------------------- PRNG
_MASK = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed: int, count: int) -> np.ndarray:
    """First ``count`` outputs of splitmix64 seeded with ``seed`` (uint64)."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, count: int) -> np.ndarray:
    """Uniform doubles in [0,1) from the top 53 bits of splitmix64."""
    return (splitmix64(seed, count) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


# ----------------------------------------------------------------------------- setups
def sod(n1: int = 1024, cfl: float = 0.8, tmax: float = 0.2) -> Problem:
    """Sod shock tube, problems/init_sod.c:31-99 (Toro test 1 states, gamma=1.4)."""
    gam = 1.4
    dx = 1.0 / n1
    rhol, el, ul = 1.0, 1.0 / (gam - 1.0), 0.0
    rhor, er, ur = 0.125, 0.1 / (gam - 1.0), 0.0
    ic = np.zeros((n1, NPRIM))
    for ii in range(n1):
        xl = ii * dx
        xr = xl + dx
        if xr < 0.5:
            ic[ii] = (rhol, el, ul, 0.0, 0.0)
        elif xl < 0.5:
            wl = (0.5 - xl) / dx
            wr = (xr - 0.5) / dx
            ic[ii] = (rhol * wl + rhor * wr, el * wl + er * wr, ul * wl + ur * wr, 0.0, 0.0)
        else:
            ic[ii] = (rhor, er, ur, 0.0, 0.0)
    return Problem(name="sod1d_%d" % n1, ndim=1, geom=CARTESIAN, n=(n1, 1, 1),
                   startx=(0.0, 0.0, 0.0), dx=(dx, 1.0, 1.0), gam=gam, ic=ic,
                   bc_lo=(OUTFLOW,) * 3, bc_hi=(OUTFLOW,) * 3, cfl=cfl, tmax=tmax)


def double_rarefaction(n1: int = 256, v: float = 2.0, cfl: float = 0.8, tmax: float = 0.15,
                       rho_floor: float = 1.0e-8, e_floor: float = 1.0e-8) -> Problem:
    """Two rarefactions running apart (problems/init_double_rare.c): rho=1, p=0.4, v=-v
    left of x=0.5 and +v right of it (the hook uses v=2), gamma=1.4, with the hook's floors
    rho 1e-8, e 1e-8 enforced (ENFORCE_FLOORS).  For v above 2 c/(gamma-1) = 3.74 the
    rarefactions open a vacuum and the centre zones approach the floors (raise them to
    make the clamp act)."""
    gam = 1.4
    dx = 1.0 / n1
    ic = np.zeros((n1, NPRIM))
    xr = (np.arange(n1) + 1) * dx
    left = xr < 0.5 + 1.0e-6
    ic[:, 0] = 1.0
    ic[:, 1] = 0.4 / (gam - 1.0)
    ic[:, 2] = np.where(left, -v, v)
    return Problem(name="double_rare1d_%d" % n1 if v == 2.0 else "double_rare1d_v%g_%d" % (v, n1), ndim=1, geom=CARTESIAN, n=(n1, 1, 1),
                   startx=(0.0, 0.0, 0.0), dx=(dx, 1.0, 1.0), gam=gam, ic=ic,
                   bc_lo=(OUTFLOW,) * 3, bc_hi=(OUTFLOW,) * 3, cfl=cfl, tmax=tmax,
                   enforce_floors=1, rho_floor=rho_floor, e_floor=e_floor)


def rayleigh_taylor_2d(n1: int = 128, n2: Optional[int] = None, g: float = -0.1, seed: int = 20240602,
                       noise: float = 0.01, cfl: float = 0.8, nsteps: Optional[int] = None,
                       tmax: float = 1.0e100) -> Problem:
    """2-D Rayleigh-Taylor with fixed gravity (the structure of problems/init_rt.c:26-125,
    GRAV=FIXED_GRAV): box [0, 0.5] x [0, 1], periodic in x and reflecting in y, heavy fluid
    (rho 2) over light (rho 1) at y = 0.5, hydrostatic pressure from p = 10/7 + 1/4 at
    y = 0 under g = (0, g), gamma = 1.4; the interface is seeded with velocity noise of
    amplitude `noise` in v_y (uniform in [-noise, noise], splitmix64 on `seed`)."""
    n2 = 2 * n1 if n2 is None else n2
    gam = 1.4
    dx0, dx1 = 0.5 / n1, 1.0 / n2
    x = (np.arange(n1) + 0.5) * dx0
    y = (np.arange(n2) + 0.5) * dx1
    X, Y = np.meshgrid(x, y, indexing="ij")
    rhotop, rhobot, pbase = 2.0, 1.0, 10.0 / 7.0 + 1.0 / 4.0
    top = Y >= 0.5
    rho = np.where(top, rhotop, rhobot)
    p = np.where(top, pbase + rhobot * g * 0.5 + rhotop * g * (Y - 0.5), pbase + rhobot * g * Y)
    u = uniform01(seed, n1 * n2).reshape(n1, n2)
    vy = noise * (2.0 * u - 1.0) * np.exp(-((Y - 0.5) / 0.05) ** 2)
    ic = np.zeros((n1 * n2, NPRIM))
    ic[:, 0] = rho.ravel()
    ic[:, 1] = (p / (gam - 1.0)).ravel()
    ic[:, 3] = vy.ravel()
    return Problem(name="rt2d_%dx%d" % (n1, n2), ndim=2, geom=CARTESIAN, n=(n1, n2, 1),
                   startx=(0.0, 0.0, 0.0), dx=(dx0, dx1, 1.0), gam=gam, ic=ic,
                   bc_lo=(PERIODIC, REFLECT, PERIODIC), bc_hi=(PERIODIC, REFLECT, PERIODIC),
                   cfl=cfl, nsteps=nsteps, tmax=tmax, grav=(0.0, g, 0.0))


def kelvin_helmholtz(n1: int = 2048, n2: Optional[int] = None, seed: int = 20240601,
                     cfl: float = 0.8, nsteps: int = 200) -> Problem:
    """2-D Kelvin-Helmholtz on the periodic unit square (the structure of
    problems/init_kh.c:23-89 with the shear-layer state of the measured workload):
    rho=2, v_x=+0.5 where |y-0.5|<0.25, else rho=1, v_x=-0.5; p=2.5; gamma=5/3;
    v_y = 0.01 sin(4 pi x); uniform noise of amplitude 1e-3 on v_x and v_y."""
    n2 = n1 if n2 is None else n2
    gam = 5.0 / 3.0
    dx0, dx1 = 1.0 / n1, 1.0 / n2
    x = (np.arange(n1) + 0.5) * dx0
    y = (np.arange(n2) + 0.5) * dx1
    X, Y = np.meshgrid(x, y, indexing="ij")
    inner = np.abs(Y - 0.5) < 0.25
    rho = np.where(inner, 2.0, 1.0)
    vx = np.where(inner, 0.5, -0.5)
    vy = 0.01 * np.sin(4.0 * math.pi * X)
    noise = uniform01(seed, 2 * n1 * n2).reshape(2, n1, n2)
    vx = vx + (2.0 * noise[0] - 1.0) * 1.0e-3
    vy = vy + (2.0 * noise[1] - 1.0) * 1.0e-3
    ic = np.zeros((n1 * n2, NPRIM))
    ic[:, 0] = rho.ravel()
    ic[:, 1] = 2.5 / (gam - 1.0)
    ic[:, 2] = vx.ravel()
    ic[:, 3] = vy.ravel()
    return Problem(name="kh2d_%dx%d" % (n1, n2), ndim=2, geom=CARTESIAN, n=(n1, n2, 1),
                   startx=(0.0, 0.0, 0.0), dx=(dx0, dx1, 1.0), gam=gam, ic=ic,
                   bc_lo=(PERIODIC, PERIODIC, PERIODIC), bc_hi=(PERIODIC, PERIODIC, PERIODIC),
                   cfl=cfl, nsteps=nsteps)


def spherical_1d(kind: str, n1: int, gam: float, rho_ratio: float = 10.0,
                 p_ratio: float = 100.0, r0: float = 0.5, cfl: float = 0.8,
                 tmax: float = 1.0e100, floors: bool = True, dr_min: Optional[float] = None,
                 coords: str = "sinh", r_in: Optional[float] = None) -> Problem:
    """1-D spherical problem on r in [0,1] (uniform radius; with dr_min the SINH radial
    map, innermost zones dr_min wide), SPHERICAL_ORIGIN inner boundary (bc.c:776-803);
    coords "log": r in [r_in, 1], log-spaced zones, reflecting inner boundary.

    kind='sod'   : rho, p = rho_ratio, p_ratio inside r<r0; 1, 1 outside; at rest;
                   OUTFLOW outer boundary.
    kind='sedov' : rho=1; p = p_ratio inside r<r0 (a small blast radius), the ambient p is 1e-5;
                   OUTFLOW outer boundary.
    kind='noh'   : problems/init_spherical_noh.c:14-61: rho=1, u=1e-6/(gam-1), v^r=-1;
                   PROB outer boundary with the Noh inflow (init_spherical_noh.c:63-79);
                   the hook's floors rho 1e-6, e 1e-7/(gam-1) (init_spherical_noh.c:22-23),
                   enforced (ENFORCE_FLOORS) unless floors=False.
    """
    _, dx, map_ = _radial_grid(n1, dr_min, coords, r_in)
    rc = np.array([_maps(map_).r((i + 0.5) * dx) for i in range(n1)])
    ic = np.zeros((n1, NPRIM))
    bc_hi = OUTFLOW
    prob_kind = PROB_NONE
    fl = dict()
    if kind == "sod":
        inside = rc < r0
        rho = np.where(inside, rho_ratio, 1.0)
        p = np.where(inside, p_ratio, 1.0)
        ic[:, 0] = rho
        ic[:, 1] = p / (gam - 1.0)
    elif kind == "sedov":
        inside = rc < r0
        p_amb = 1.0e-5
        ic[:, 0] = 1.0
        ic[:, 1] = np.where(inside, p_amb * p_ratio, p_amb) / (gam - 1.0)
    elif kind == "noh":
        if map_:
            raise ValueError("the Noh inflow boundary is built for the uniform radial map")
        ic[:, 0] = 1.0
        ic[:, 1] = 1.0e-6 / (gam - 1.0)
        ic[:, 2] = -1.0   # vr / scale[0][0], scale[0][0] = 1 for a uniform radius
        bc_hi = PROB
        prob_kind = PROB_NOH
        if floors:
            fl = dict(enforce_floors=1, rho_floor=1.0e-6, e_floor=1.0e-7 / (gam - 1.0))
    else:
        raise ValueError("unknown 1-D spherical problem kind %r" % kind)
    return Problem(name="sph1d_%s%s_%d" % (_map_tag(map_), kind, n1), ndim=1, geom=SPHERICAL,
                   n=(n1, 1, 1), startx=(0.0, -1.0, 0.0), dx=(dx, 2.0, 2.0 * math.pi), gam=gam, ic=ic,
                   bc_lo=(REFLECT if coords == "log" else SPHERICAL_ORIGIN, OUTFLOW, OUTFLOW),
                   bc_hi=(bc_hi, OUTFLOW, OUTFLOW),
                   prob_kind=prob_kind, cfl=cfl, tmax=tmax, **fl, **map_)


MAX_LOG2_ASPECT = 0.5   # utils.c:12


class CoordMaps:
    """The radial and theta maps r(x), th(x) of a spherical grid (RCOORD and THCOORD,
    metric_spherical_general.c:149-290), restated for the grid counts and the problem
    generators (the library evaluates its own copy)."""

    def __init__(self, rcoord=RCOORD_UNIFORM, rtrans=1.0, rfact=RFACT_DEFAULT, thcoord=THCOORD_UNIFORM,
                 poly_xt=POLY_XT_DEFAULT, poly_alpha=POLY_ALPHA_DEFAULT):
        self.rcoord, self.rtrans, self.rfact = rcoord, rtrans, tuple(rfact)
        self.thcoord, self.poly_xt, self.poly_alpha = thcoord, poly_xt, poly_alpha
        # init_coords (metric_spherical_general.c:565-567)
        self.poly_norm = 0.5 * math.pi * 1.0 / (1.0 + 1.0 / (poly_alpha + 1.0) * 1.0 / math.pow(poly_xt, poly_alpha))

    @classmethod
    def of(cls, pb):
        return cls(pb.rcoord, pb.rtrans, pb.rfact, pb.thcoord, pb.poly_xt, pb.poly_alpha)

    def r(self, x: float) -> float:
        ax = abs(x)
        if self.rcoord == RCOORD_SINH:
            return self.rtrans * math.sinh(ax / self.rtrans)
        if self.rcoord == RCOORD_SINH_MODIFIED:
            fa, fb, fc = self.rfact
            sig = lambda y: 1.0 / (1.0 + math.exp(-y))
            return self.rtrans * math.sinh(ax / self.rtrans) - fa * sig((ax - fb) / fc) + fa * sig(-fb / fc)
        if self.rcoord == RCOORD_LOG:
            return self.rtrans * math.exp(ax / self.rtrans)
        return ax

    def th(self, x: float) -> float:
        if x < -1.0:
            x = -2.0 - x
        if x > 1.0:
            x = 2.0 - x
        if self.thcoord == THCOORD_POLYTH:
            return self.poly_norm * x * (1.0 + math.pow(x / self.poly_xt, self.poly_alpha) /
                                         (self.poly_alpha + 1.0)) + 0.5 * math.pi
        return 0.5 * math.pi * (x + 1.0)


def _r_of_x(x: float, rtrans: Optional[float] = None) -> float:
    """r(x) of the UNIFORM map (rtrans None) or of the SINH map (metric_spherical_general.c:
    149-160)."""
    if rtrans is None:
        return abs(x)
    return rtrans * math.sinh(abs(x) / rtrans)


def sinh_rtrans(n1: int, dx0: float, r_out: float, rcoord: int = RCOORD_SINH,
                rfact: tuple = RFACT_DEFAULT) -> float:
    """Transition radius of the SINH (or SINH_MODIFIED) map whose n1 zones of coordinate
    width dx0 reach r_out: the root of r(n1 dx0) = r_out, by bracketing and bisection to a
    relative width of 1e-10 (the method of rtrans_solve, metric_spherical_general.c:16-78,
    which the reference's problem hooks call, e.g. problems/init_sedov.c:20).  Needs a map
    that stretches to r_out.  The zones then start about dx0 wide at the centre and widen
    geometrically outside r ~ rtrans."""
    X = n1 * dx0

    def f(rt):
        if X / rt >= 700.0:
            return math.inf
        return CoordMaps(rcoord, rt, rfact).r(X) - r_out

    lo = 0.1 * dx0
    while not math.isfinite(f(lo)):
        lo *= 1.1
    hi = 100.0 * r_out
    flo = f(lo)
    if flo * f(hi) > 0.0:
        raise ValueError("rtrans not bracketed: the map does not reach r_out")
    while abs((lo - hi) / hi) > 1.0e-10:
        mid = 0.5 * (lo + hi)
        fm = f(mid)
        if fm * flo <= 0.0:
            hi = mid
        else:
            lo, flo = mid, fm
    return 0.5 * (lo + hi)


def radial_edges(pb: Problem) -> np.ndarray:
    """r at the n1+1 radial zone edges of a spherical problem (its radial map)."""
    m = CoordMaps.of(pb)
    return np.array([m.r(pb.startx[0] + i * pb.dx[0]) for i in range(pb.n[0] + 1)])


def radial_centers(pb: Problem) -> np.ndarray:
    """r at the n1 radial zone centres (ijk_to_x then r_of_x, as the dumps place them)."""
    m = CoordMaps.of(pb)
    return np.array([m.r(pb.startx[0] + (i + 0.5) * pb.dx[0]) for i in range(pb.n[0])])


def dendritic_grid(n1: int, n2: int, n3: int, startx: tuple, dx: tuple, ndim: int = 3,
                   rtrans: Optional[float] = None, maps: Optional[CoordMaps] = None):
    """Zone counts of the dendritic spherical grid: nj[i] theta zones of radial row i and
    nk[i][j] phi zones of row (i, j), for the interior rows (the rules of compute_dj and
    compute_dk, utils.c:181-354, for a uniform radius and theta: theta zones double
    outwards from 2 at the centre and phi zones from 4 at each pole while the zone aspect
    ratio exceeds 2^0.5; on a 2-D grid every row has n3 = 1 phi zone; rtrans selects the
    SINH radial map, maps any pair of coordinate maps).  Returns (nj, nk) as lists; the
    interior zones in the reference's zone order are i, then j < nj[i], then k < nk[i][j]."""
    if maps is None:
        maps = CoordMaps(RCOORD_SINH, rtrans) if rtrans is not None else CoordMaps()
    _r_of = maps.r
    _th_of = maps.th
    nj = [0] * n1
    nj[0] = 2
    dth = _th_of(startx[1] + n2 * dx[1]) - _th_of(startx[1])
    for i in range(1, n1):
        r0 = _r_of(startx[0] + (i + 0.0) * dx[0])
        rc = _r_of(startx[0] + (i + 0.5) * dx[0])
        r1 = _r_of(startx[0] + (i + 1.0) * dx[0])
        ideal = rc * dth / (r1 - r0)
        nj[i] = nj[i - 1]
        if math.log2(ideal / nj[i]) > MAX_LOG2_ASPECT:
            nj[i] *= 2
        nj[i] = min(max(nj[i], nj[i - 1]), n2)
    dj = [n2 // v for v in nj]
    if ndim == 2:
        return nj, [[n3] * nj[i] for i in range(n1)]
    dph = n3 * dx[2]
    nk = []
    for i in range(n1):
        r0 = _r_of(startx[0] + (i + 0.0) * dx[0])
        rc = _r_of(startx[0] + (i + 0.5) * dx[0])
        r1 = _r_of(startx[0] + (i + 1.0) * dx[0])
        dr = r1 - r0
        row = [0] * nj[i]
        row[0] = 4
        for j in range(1, nj[i]):
            thc = _th_of(startx[1] + (j + 0.5) * dj[i] * dx[1])
            ideal = rc * math.sin(thc) * dph / dr
            if j < nj[i] // 2:
                row[j] = row[j - 1]
                if math.log2(ideal / row[j]) > MAX_LOG2_ASPECT:
                    row[j] *= 2
                if i == 0:
                    row[j] = min(row[j], n3)
                elif nj[i - 1] == nj[i]:
                    row[j] = min(max(row[j], nk[i - 1][j]), n3)
                else:
                    row[j] = min(max(row[j], nk[i - 1][j // 2]), n3)
            else:
                row[j] = row[nj[i] - 1 - j]
        nk.append(row)
    return nj, nk


def dendritic_refine_errors(n2: int, n3: int, nj: list, nk: list) -> int:
    """Cells (i, j, k) where phi refines 4-to-1 across a 2:1 theta refinement from radial
    row i to i+1 -- the grids that init_dendritic (utils.c:548-586) rejects.  nj, nk as
    dendritic_grid returns them (interior rows); the outer ghost row copies row n1-1."""
    n1 = len(nj)
    bad = 0
    for i0 in range(n1 - 1):
        dj0, dj1 = n2 // nj[i0], n2 // nj[i0 + 1]
        if dj0 // dj1 != 2:
            continue
        row1 = nk[i0 + 1]
        for j00 in range(nj[i0]):
            j10 = j00 * dj0 // dj1
            j11 = j10 + 1
            # the ghost column j = nj reflects column nj - 1
            k10 = row1[j10]
            k11 = row1[j11] if j11 < len(row1) else row1[2 * len(row1) - 1 - j11]
            dk0 = n3 // nk[i0][j00]
            if dk0 // (n3 // k10) == 4 or dk0 // (n3 // k11) == 4:
                bad += nk[i0][j00]
    return bad


def _radial_grid(n1: int, dr_min: Optional[float], coords: str = "sinh", r_in: Optional[float] = None):
    """(startx, dx0, map fields) of a radial grid on r in [0, 1]: uniform, or with dr_min
    the SINH map with innermost zones about dr_min wide (coords "sinh"), or the
    reference's default build maps, SINH_MODIFIED radius and POLYTH theta with the
    parse_input parameters (coords "default"); coords "log" is the grid on [r_in, 1] with
    log-spaced zones (RCOORD_LOG, rtrans = r_in, zone edges r_in (1/r_in)^(i/n1))."""
    startx = (0.0, -1.0, 0.0)
    if coords == "log":
        if not (r_in is not None and 0.0 < r_in < 1.0):
            raise ValueError("the log-spaced radius needs 0 < r_in < 1")
        return startx, r_in * math.log(1.0 / r_in) / n1, dict(rcoord=RCOORD_LOG, rtrans=r_in)
    if coords == "sinh_rt":
        # the SINH map with rtrans = r_in: uniform zones (dx wide) inside r ~ r_in, log-spaced
        # outside it (r ~ (r_in/2) exp(x/r_in)), n1 zones to r = 1
        if not (r_in is not None and 0.0 < r_in < 1.0):
            raise ValueError("coords 'sinh_rt' needs 0 < r_in < 1 (the transition radius)")
        return startx, r_in * math.asinh(1.0 / r_in) / n1, dict(rcoord=RCOORD_SINH, rtrans=r_in)
    if dr_min is None:
        return startx, 1.0 / n1, {}
    if coords == "default":
        rt = sinh_rtrans(n1, dr_min, 1.0, RCOORD_SINH_MODIFIED)
        return startx, dr_min, dict(rcoord=RCOORD_SINH_MODIFIED, rtrans=rt, thcoord=THCOORD_POLYTH)
    return startx, dr_min, dict(rcoord=RCOORD_SINH, rtrans=sinh_rtrans(n1, dr_min, 1.0))


def _maps(map_: dict) -> CoordMaps:
    return CoordMaps(map_.get("rcoord", RCOORD_UNIFORM), map_.get("rtrans", 1.0), RFACT_DEFAULT,
                     map_.get("thcoord", THCOORD_UNIFORM))


def _map_tag(map_: dict) -> str:
    if not map_:
        return ""
    if map_.get("rcoord") == RCOORD_LOG:
        return "log_"
    return "default_" if map_.get("thcoord", THCOORD_UNIFORM) == THCOORD_POLYTH else "sinh_"


def _blast_energy_rows(n1, startx, dx0, map_, r_dep, energy, gam, p_amb) -> np.ndarray:
    """Internal energy density per radial row of a blast: energy / (4/3 pi (r_e^3 - r_0^3))
    in the rows whose centre lies inside r_dep (r_e the outer edge of the last of them,
    r_0 the inner edge of the grid: 0 for a grid from the origin), the ambient
    p_amb / (gam - 1) elsewhere."""
    m = _maps(map_)
    rc = np.array([m.r(startx[0] + (i + 0.5) * dx0) for i in range(n1)])
    inside = rc < r_dep
    i_e = (np.nonzero(inside)[0].max() + 1) if inside.any() else 1
    r_e = m.r(startx[0] + i_e * dx0)
    r_0 = m.r(startx[0])
    u_dep = energy / (4.0 / 3.0 * math.pi * (r_e ** 3 - r_0 ** 3))
    return np.where(inside, u_dep, p_amb / (gam - 1.0))


def sedov_3d(n1: int = 384, n2: int = 128, n3: int = 256, gam: float = 1.4, energy: float = 1.0,
             r_dep: float = 0.02, p_amb: float = 1.0e-5, cfl: float = 0.8, tmax: float = 1.0e100,
             bc_inner: int = REFLECT, bc_pole: int = REFLECT, noise: float = 0.0,
             seed: int = 20240603, dr_min: Optional[float] = None, coords: str = "sinh",
             r_in: Optional[float] = None) -> Problem:
    """3-D Sedov blast on the dendritic spherical grid (the structure of
    problems/init_sedov.c:3-164): r in [0, 1] uniform, theta in [0, pi], phi in [0, 2 pi);
    rho = 1, p = p_amb, at rest, and the energy `energy` deposited as a uniform internal
    energy density in the zones whose centre lies inside r_dep (volume of those full
    shells: 4/3 pi r_e^3); reflecting inner and pole boundaries, periodic in phi.  With
    noise > 0 the density is scaled by 1 + noise*(2U-1) and the three coordinate
    velocities are set to 0.1*noise*(2U-1) (U uniform, splitmix64 on `seed`), which breaks
    the symmetry (shock tagging, rotation through the pole rows, restriction of v^phi).
    With dr_min the radius follows the SINH map instead (RCOORD=SINH, the map of the
    reference's own Sedov hook): the innermost zones are dr_min wide and the zone widths
    grow geometrically outwards to r = 1 (coords "default": the reference's default
    build maps, SINH_MODIFIED radius and POLYTH theta).  coords "log" puts the grid on
    r in [r_in, 1] with log-spaced zones (RCOORD_LOG): the inner boundary is the sphere
    r = r_in (reflecting by default) and the deposit fills the shells from r_in; coords
    "sinh_rt" is the SINH map with its transition radius at r_in: zones log-spaced from
    about r_in to 1 and uniform inside (the origin stays in the grid)."""
    startx, dx, map_ = _radial_grid(n1, dr_min, coords, r_in)
    dx = (dx, 2.0 / n2, 2.0 * math.pi / n3)
    nj, nk = dendritic_grid(n1, n2, n3, startx, dx, maps=_maps(map_))
    counts = np.array([sum(row) for row in nk])
    ncell = int(counts.sum())
    u_row = _blast_energy_rows(n1, startx, dx[0], map_, r_dep, energy, gam, p_amb)
    ic = np.zeros((ncell, NPRIM))
    ic[:, 0] = 1.0
    ic[:, 1] = np.repeat(u_row, counts)
    if noise > 0.0:
        u = uniform01(seed, 4 * ncell).reshape(ncell, 4)
        ic[:, 0] *= 1.0 + noise * (2.0 * u[:, 0] - 1.0)
        for v in range(3):
            ic[:, 2 + v] = 0.1 * noise * (2.0 * u[:, 1 + v] - 1.0)
    return Problem(name="sedov3d_%s%dx%dx%d" % (_map_tag(map_), n1, n2, n3), ndim=3, geom=SPHERICAL,
                   n=(n1, n2, n3), startx=startx, dx=dx, gam=gam, ic=ic,
                   bc_lo=(bc_inner, bc_pole, PERIODIC), bc_hi=(OUTFLOW, bc_pole, PERIODIC),
                   cfl=cfl, tmax=tmax, cells=ncell, **map_)


def sedov_2d_spherical(n1: int = 256, n2: int = 128, gam: float = 1.4, energy: float = 1.0, r_dep: float = 0.02,
                       p_amb: float = 1.0e-5, cfl: float = 0.8, tmax: float = 1.0e100, bc_inner: int = REFLECT,
                       bc_pole: int = REFLECT, noise: float = 0.0, seed: int = 20240604,
                       dr_min: Optional[float] = None, coords: str = "sinh",
                       r_in: Optional[float] = None) -> Problem:
    """Axisymmetric (r, theta) Sedov blast on the 2-D dendritic spherical grid: theta zones
    double outwards from 2 at the centre (compute_dj, utils.c:181-238); otherwise as
    sedov_3d (energy in the zones inside r_dep, seeded noise in density and velocities,
    the SINH radial map with dr_min, the default build maps with coords "default", the
    log-spaced radius on [r_in, 1] with coords "log", the SINH map with rtrans = r_in with
    coords "sinh_rt")."""
    startx, dx, map_ = _radial_grid(n1, dr_min, coords, r_in)
    dx = (dx, 2.0 / n2, 2.0 * math.pi)
    nj, _ = dendritic_grid(n1, n2, 1, startx, dx, ndim=2, maps=_maps(map_))
    ncell = int(sum(nj))
    ic = np.zeros((ncell, NPRIM))
    ic[:, 0] = 1.0
    ic[:, 1] = np.repeat(_blast_energy_rows(n1, startx, dx[0], map_, r_dep, energy, gam, p_amb), nj)
    if noise > 0.0:
        u = uniform01(seed, 4 * ncell).reshape(ncell, 4)
        ic[:, 0] *= 1.0 + noise * (2.0 * u[:, 0] - 1.0)
        for v in range(3):
            ic[:, 2 + v] = 0.1 * noise * (2.0 * u[:, 1 + v] - 1.0)
    return Problem(name="sedov2dsph_%s%dx%d" % (_map_tag(map_), n1, n2), ndim=2, geom=SPHERICAL,
                   n=(n1, n2, 1), startx=startx, dx=dx, gam=gam, ic=ic, bc_lo=(bc_inner, bc_pole, PERIODIC),
                   bc_hi=(OUTFLOW, bc_pole, PERIODIC), cfl=cfl, tmax=tmax, cells=ncell, **map_)


GNEWT = 6.67384e-8   # constants.h:3 (cgs)


def dust_collapse(n1: int = 200, n2: int = 16, n3: int = 32, ndim: int = 1, dr: float = 5.0e4,
                  r_out: float = 7.0e8, rho0: float = 1.0e9, r0: float = 6.5e8, t0: float = 1.0,
                  mach: float = 2.0, gam: float = 5.0 / 3.0, cfl: float = 0.9, tmax: float = 1.0e100,
                  radius: str = "sinh", floors: bool = True, hook: Optional[bool] = None) -> Problem:
    """Collapse of a uniform, nearly pressureless sphere under its own gravity in the
    monopole approximation (problems/init_dustcollapse.c, setups/dustcollapse_1d.mk; cgs):
    rho0 inside r0 (the zone that straddles r0 gets the volume-weighted share), the
    floor 1e-5 rho0 outside, p0 = rho0 (r0/t0/mach)^2 / gam everywhere, at rest;
    SPHERICAL_ORIGIN at the centre.  The radius follows the SINH map with innermost zones
    `dr` wide reaching r_out (rtrans_solve as the hook calls it), or with radius="uniform"
    zones of width r_out/n1.  In 1-D the outer boundary is outflow with the hook's
    v^r = -1/sqrt(r) (hook=True, the default there); the dendritic grids (ndim 2 or 3,
    SPHERICAL_ORIGIN poles, periodic phi) use plain outflow.  floors: the ENFORCE_FLOORS
    build with the hook's rho_floor = 1e-5 rho0 and e_floor = p0/(gam-1)."""
    if hook is None:
        hook = ndim == 1
    if hook and ndim != 1:
        raise ValueError("the dust-collapse boundary hook is built for 1-D grids")
    if radius == "sinh":
        dx0 = dr
        map_ = dict(rcoord=RCOORD_SINH, rtrans=sinh_rtrans(n1, dr, r_out))
    else:
        dx0 = r_out / n1
        map_ = {}
    rt = map_.get("rtrans")
    v0 = r0 / t0
    p0 = rho0 * (v0 / mach) ** 2 / gam
    rho_floor = 1.0e-5 * rho0
    e_floor = p0 / (gam - 1.0)
    rho_row = np.empty(n1)
    for i in range(n1):
        rm, rp = _r_of_x(i * dx0, rt), _r_of_x((i + 1) * dx0, rt)
        if rp < r0:
            rho_row[i] = rho0
        elif rm < r0:
            rho_row[i] = rho0 * (math.pow(r0, 3) - math.pow(rm, 3)) / (math.pow(rp, 3) - math.pow(rm, 3))
        else:
            rho_row[i] = rho_floor
    fl = dict(enforce_floors=1, rho_floor=rho_floor, e_floor=e_floor) if floors else \
        dict(rho_floor=rho_floor, e_floor=e_floor)
    if ndim == 1:
        counts = np.ones(n1, dtype=int)
        n, startx, dx = (n1, 1, 1), (0.0, -1.0, 0.0), (dx0, 2.0, 2.0 * math.pi)
        bc_lo = (SPHERICAL_ORIGIN, OUTFLOW, OUTFLOW)
        bc_hi = (PROB if hook else OUTFLOW, OUTFLOW, OUTFLOW)
        cells = 0
    else:
        n3e = n3 if ndim == 3 else 1
        startx, dx = (0.0, -1.0, 0.0), (dx0, 2.0 / n2, 2.0 * math.pi / n3e)
        nj, nk = dendritic_grid(n1, n2, n3e, startx, dx, ndim=ndim, rtrans=rt)
        counts = np.array([sum(row) for row in nk])
        n = (n1, n2, n3e)
        bc_lo = (SPHERICAL_ORIGIN, SPHERICAL_ORIGIN, PERIODIC)
        bc_hi = (OUTFLOW, SPHERICAL_ORIGIN, PERIODIC)
        cells = int(counts.sum())
    ncell = int(counts.sum())
    ic = np.zeros((ncell, NPRIM))
    ic[:, 0] = np.repeat(rho_row, counts)
    ic[:, 1] = p0 / (gam - 1.0)
    return Problem(name="dust%dd_%s%d" % (ndim, "sinh_" if map_ else "", n1), ndim=ndim, geom=SPHERICAL, n=n,
                   startx=startx, dx=dx, gam=gam, ic=ic, bc_lo=bc_lo, bc_hi=bc_hi,
                   prob_kind=PROB_DUST if hook else PROB_NONE, cfl=cfl, tmax=tmax, monopole=1, cells=cells,
                   **fl, **map_)


def ensemble_1d(count: int = 2048, seed: int = 7, nmin: int = 128, nmax: int = 8192,
                cfl: float = 0.8) -> list:
    """Ensemble of independent 1-D spherical problems: zone counts log-uniform in
    [nmin, nmax], kinds Sod/Noh/Sedov, density ratio log-uniform in [2, 100], pressure
    ratio log-uniform in [2, 1e4], gamma drawn from {4/3, 1.4, 5/3}."""
    u = uniform01(seed, 5 * count).reshape(count, 5)
    out = []
    gams = (4.0 / 3.0, 1.4, 5.0 / 3.0)
    kinds = ("sod", "noh", "sedov")
    for m in range(count):
        n1 = int(round(math.exp(math.log(nmin) + u[m, 0] * (math.log(nmax) - math.log(nmin)))))
        n1 = max(nmin, min(nmax, n1))
        kind = kinds[min(2, int(u[m, 1] * 3))]
        rr = math.exp(math.log(2.0) + u[m, 2] * (math.log(100.0) - math.log(2.0)))
        pr = math.exp(math.log(2.0) + u[m, 3] * (math.log(1.0e4) - math.log(2.0)))
        gam = gams[min(2, int(u[m, 4] * 3))]
        r0 = 0.5 if kind == "sod" else 0.05
        pb = spherical_1d(kind, n1, gam, rho_ratio=rr, p_ratio=pr, r0=r0, cfl=cfl)
        pb.name = "ens%04d_%s" % (m, pb.name)
        out.append(pb)
    return out


def blast_2d(n1: int = 64, n2: Optional[int] = None, p_in: float = 10.0, p_out: float = 0.01,
             radius: float = 0.1, bc: int = REFLECT, cfl: float = 0.8) -> Problem:
    """2-D Cartesian blast wave on the unit square (in the spirit of
    problems/init_sedov_cart.c): rho=1 at rest, p=p_in inside a circle of the given
    radius around (0.5, 0.5), p_out outside; the strong shock exercises the shock flags
    and the HLLE switch of step.c:711-755."""
    n2 = n1 if n2 is None else n2
    gam = 1.4
    dx0, dx1 = 1.0 / n1, 1.0 / n2
    x = (np.arange(n1) + 0.5) * dx0
    y = (np.arange(n2) + 0.5) * dx1
    X, Y = np.meshgrid(x, y, indexing="ij")
    r = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2)
    p = np.where(r < radius, p_in, p_out)
    ic = np.zeros((n1 * n2, NPRIM))
    ic[:, 0] = 1.0
    ic[:, 1] = (p / (gam - 1.0)).ravel()
    return Problem(name="blast2d_%dx%d" % (n1, n2), ndim=2, geom=CARTESIAN, n=(n1, n2, 1),
                   startx=(0.0, 0.0, 0.0), dx=(dx0, dx1, 1.0), gam=gam, ic=ic,
                   bc_lo=(bc, bc, bc), bc_hi=(bc, bc, bc), cfl=cfl)
