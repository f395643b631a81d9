"""Analytic solutions and error norms used to state the accuracy of a run.

* :func:`exact_riemann` - the exact solution of the 1-D Riemann problem of a gamma-law gas
  (Godunov's exact solver as described in Toro, "Riemann Solvers and Numerical Methods for
  Fluid Dynamics", 3rd ed., ch. 4: Newton iteration on the star pressure, then sampling);
  the analytic answer of the Sod shock tube (problems/init_sod.c).
* :func:`noh_spherical` - the spherical Noh implosion (Noh 1987, J. Comput. Phys. 72, 78):
  a shock moving out at D = (gamma-1) v0 / 2 behind which the gas is at rest with density
  rho0 ((gamma+1)/(gamma-1))^3 and specific internal energy v0^2/2; ahead of it the inflow
  is compressed geometrically, rho = rho0 (1 + v0 t / r)^2
  (problems/init_spherical_noh.c:63-79 drives the outer boundary with that inflow).
* :class:`SedovTaylor` - the spherical point blast (Sedov 1959; Kamm & Timmes 2007):
  the self-similar profile from the ODEs of the similarity variable, and xi0.
* :func:`l1_rel` - volume-weighted relative L1 distance, sum |a-b| dV / sum |b| dV.

Primitive states follow the library's layout: rho, u (internal energy density), v1, v2, v3.
"""
from __future__ import annotations

import math

import numpy as np


def _pressure_function(p, rk, pk, ck, gam):
    """Toro's f_K(p) and its derivative for one side K of the Riemann problem."""
    if p > pk:   # shock
        A = 2.0 / ((gam + 1.0) * rk)
        B = (gam - 1.0) / (gam + 1.0) * pk
        q = math.sqrt(A / (p + B))
        return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (B + p))
    # rarefaction
    e = (gam - 1.0) / (2.0 * gam)
    f = 2.0 * ck / (gam - 1.0) * ((p / pk) ** e - 1.0)
    return f, (p / pk) ** (-(gam + 1.0) / (2.0 * gam)) / (rk * ck)


def exact_riemann(left, right, gam: float, x: np.ndarray, t: float, x0: float = 0.5):
    """Exact solution (rho, v, p) at points x and time t > 0 of the Riemann problem with
    left/right states (rho, v, p) separated at x0."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(gam * pl / rl), math.sqrt(gam * pr / rr)
    # star pressure: Newton iteration from the two-rarefaction guess
    e = (gam - 1.0) / (2.0 * gam)
    p = ((cl + cr - 0.5 * (gam - 1.0) * (ur - ul)) / (cl / pl ** e + cr / pr ** e)) ** (1.0 / e)
    p = max(p, 1.0e-12)
    for _ in range(100):
        fl, dl = _pressure_function(p, rl, pl, cl, gam)
        fr, dr = _pressure_function(p, rr, pr, cr, gam)
        pn = p - (fl + fr + ur - ul) / (dl + dr)
        pn = max(pn, 1.0e-14)
        done = abs(pn - p) < 1.0e-15 * (pn + p)
        p = pn
        if done:
            break
    fl, _ = _pressure_function(p, rl, pl, cl, gam)
    fr, _ = _pressure_function(p, rr, pr, cr, gam)
    us = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    gm, gp = gam - 1.0, gam + 1.0
    s = (np.asarray(x, dtype=np.float64) - x0) / t
    rho, vel, pre = np.empty_like(s), np.empty_like(s), np.empty_like(s)
    for k, sk in enumerate(s):
        if sk <= us:   # left of the contact
            if p > pl:
                sh = ul - cl * math.sqrt(gp / (2 * gam) * p / pl + gm / (2 * gam))
                if sk <= sh:
                    rho[k], vel[k], pre[k] = rl, ul, pl
                else:
                    rho[k] = rl * (p / pl + gm / gp) / (gm / gp * p / pl + 1.0)
                    vel[k], pre[k] = us, p
            else:
                shl = ul - cl
                cs = cl * (p / pl) ** e
                stl = us - cs
                if sk <= shl:
                    rho[k], vel[k], pre[k] = rl, ul, pl
                elif sk > stl:
                    rho[k], vel[k], pre[k] = rl * (p / pl) ** (1.0 / gam), us, p
                else:
                    c = 2.0 / gp * (cl + gm / 2.0 * (ul - sk))
                    vel[k] = 2.0 / gp * (cl + gm / 2.0 * ul + sk)
                    rho[k] = rl * (c / cl) ** (2.0 / gm)
                    pre[k] = pl * (c / cl) ** (2.0 * gam / gm)
        else:          # right of the contact
            if p > pr:
                sh = ur + cr * math.sqrt(gp / (2 * gam) * p / pr + gm / (2 * gam))
                if sk >= sh:
                    rho[k], vel[k], pre[k] = rr, ur, pr
                else:
                    rho[k] = rr * (p / pr + gm / gp) / (gm / gp * p / pr + 1.0)
                    vel[k], pre[k] = us, p
            else:
                shr = ur + cr
                cs = cr * (p / pr) ** e
                stl = us + cs
                if sk >= shr:
                    rho[k], vel[k], pre[k] = rr, ur, pr
                elif sk < stl:
                    rho[k], vel[k], pre[k] = rr * (p / pr) ** (1.0 / gam), us, p
                else:
                    c = 2.0 / gp * (cr - gm / 2.0 * (ur - sk))
                    vel[k] = 2.0 / gp * (-cr + gm / 2.0 * ur + sk)
                    rho[k] = rr * (c / cr) ** (2.0 / gm)
                    pre[k] = pr * (c / cr) ** (2.0 * gam / gm)
    return rho, vel, pre


def sod_exact_state(n1: int, t: float, gam: float = 1.4) -> np.ndarray:
    """Zone-centre samples [n1, 5] of the exact Sod solution (left 1, 0, 1; right 0.125,
    0, 0.1; interface at 0.5) on [0, 1]."""
    x = (np.arange(n1) + 0.5) / n1
    rho, v, p = exact_riemann((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), gam, x, t, 0.5)
    out = np.zeros((n1, 5))
    out[:, 0], out[:, 1], out[:, 2] = rho, p / (gam - 1.0), v
    return out


def noh_spherical(r: np.ndarray, t: float, gam: float, v0: float = 1.0, rho0: float = 1.0,
                  u0: float = 1.0e-6) -> np.ndarray:
    """Spherical Noh solution [len(r), 5] at radii r and time t (inflow speed v0, upstream
    density rho0 and internal energy density u0/(gam-1) at t=0)."""
    r = np.asarray(r, dtype=np.float64)
    rs = 0.5 * (gam - 1.0) * v0 * t
    out = np.zeros((r.size, 5))
    inside = r < rs
    rho_in = rho0 * ((gam + 1.0) / (gam - 1.0)) ** 3
    rho_out = rho0 * (1.0 + v0 * t / np.maximum(r, 1.0e-300)) ** 2
    out[:, 0] = np.where(inside, rho_in, rho_out)
    # behind the shock: specific internal energy v0^2/2; ahead: adiabatic compression
    u_out = u0 / (gam - 1.0) * (rho_out / rho0) ** gam
    out[:, 1] = np.where(inside, rho_in * 0.5 * v0 * v0, u_out)
    out[:, 2] = np.where(inside, 0.0, -v0)
    return out


def spherical_volumes(n1: int, r_lo: float = 0.0, r_hi: float = 1.0) -> np.ndarray:
    """Zone volumes (up to the constant 4 pi / 3) of a uniform radial grid."""
    e = np.linspace(r_lo, r_hi, n1 + 1)
    return e[1:] ** 3 - e[:-1] ** 3


# R_s = xi0 (E t^2 / rho)^(1/5) of the spherical Sedov-Taylor blast (Sedov 1959; the
# constants used by G. I. Taylor 1950 and tabulated by Kamm & Timmes 2007)
SEDOV_XI0 = {1.4: 1.033, 5.0 / 3.0: 1.152}


def sedov_shock_radius(energy: float, t: float, rho: float = 1.0, gam: float = 1.4) -> float:
    """Shock radius of the point blast of energy `energy` in gas of density rho at time t."""
    return SEDOV_XI0[gam] * (energy * t * t / rho) ** 0.2


class SedovTaylor:
    """The spherical Sedov-Taylor point blast in a uniform gas at rest (the standard case
    of Kamm & Timmes 2007, LA-UR-07-2849: geometry j = 3, uniform density, strong shock).

    With the shock at R(t) = xi0 (E t^2 / rho0)^(1/5) and eta = r/R, Sedov's closed-form
    solution (Sedov 1959; Landau & Lifshitz, Fluid Mechanics, sec. 106) is parametric in
    the velocity variable V = 5 t v / (2 r), which runs from 2/(g+1) at the shock to 1/g
    at the centre:
        eta^5 = ((g+1) V/2)^-2  a^n1  b^n2,           a = (g+1)/(7-g) (5 - (3g-1) V)
        rho/rho0 = (g+1)/(g-1)  b^n3  a^n4  c^n5,      b = (g+1)/(g-1) (g V - 1)
                                                       c = (g+1)/(g-1) (1 - V)
        n1 = -(13g^2 - 7g + 12)/((3g-1)(2g+1)), n2 = 5(g-1)/(2g+1), n3 = 3/(2g+1),
        n4 = -n1/(2-g), n5 = -2/(2-g);
    the sound speed follows from the energy integral, c_s^2 = (2r/5t)^2 Z with
    Z = g(g-1)(1-V)V^2 / (2(gV-1)), so p = rho c_s^2 / g and v = (2r/5t) V.  xi0 follows
    from E = int (rho v^2/2 + p/(g-1)) dV over the blast (1.0328 for g = 1.4).  The
    parametrisation is singular at g = 2 (n4, n5); the configurations here have g < 2."""

    def __init__(self, gam: float = 1.4, npts: int = 20000):
        g = self.gam = float(gam)
        if not (1.0 < g < 2.0):
            raise ValueError("SedovTaylor: 1 < gamma < 2")
        n1 = -(13.0 * g * g - 7.0 * g + 12.0) / ((3.0 * g - 1.0) * (2.0 * g + 1.0))
        n2 = 5.0 * (g - 1.0) / (2.0 * g + 1.0)
        n3 = 3.0 / (2.0 * g + 1.0)
        n4 = -n1 / (2.0 - g)
        n5 = -2.0 / (2.0 - g)
        v0, v1 = 1.0 / g, 2.0 / (g + 1.0)
        # w = g V - 1, spaced geometrically towards the centre (eta ~ w^(n2/5) there) and
        # uniformly towards the shock, where the profiles are steepest in eta
        wmax = (g - 1.0) / (g + 1.0)
        w = np.unique(np.concatenate([np.geomspace(1.0e-30, wmax, npts), np.linspace(0.0, wmax, npts)[1:]]))
        V = (1.0 + w) / g
        V[-1] = v1
        a = (g + 1.0) / (7.0 - g) * (5.0 - (3.0 * g - 1.0) * V)
        b = (g + 1.0) / (g - 1.0) * w
        c = (g + 1.0) / (g - 1.0) * (1.0 - V)
        eta = (((g + 1.0) * V / 2.0) ** -2 * a ** n1 * b ** n2) ** 0.2
        G = (g + 1.0) / (g - 1.0) * b ** n3 * a ** n4 * c ** n5
        Z = g * (g - 1.0) * (1.0 - V) * V * V / (2.0 * w)
        # in units of R' = (2/5) R/t:  v = R' eta V,  p = rho0 R'^2 G eta^2 Z / g
        self.eta = np.concatenate([[0.0], eta])
        self.G = np.concatenate([[0.0], G])
        self.U = np.concatenate([[0.0], eta * V])
        self.P = np.concatenate([[G[0] * eta[0] ** 2 * Z[0] / g], G * eta * eta * Z / g])
        f = (0.5 * self.G * self.U ** 2 + self.P / (g - 1.0)) * self.eta ** 2
        integral = float(np.sum(0.5 * (f[1:] + f[:-1]) * np.diff(self.eta)))
        self.xi0 = (25.0 / (16.0 * math.pi * integral)) ** 0.2

    def shock_radius(self, energy: float, t: float, rho0: float = 1.0) -> float:
        return self.xi0 * (energy * t * t / rho0) ** 0.2

    def profile(self, r: np.ndarray, t: float, energy: float = 1.0, rho0: float = 1.0,
                p_amb: float = 0.0) -> np.ndarray:
        """Primitive state [len(r), 5] (rho, internal energy density p/(gamma-1), v^r, 0, 0)
        at radii r and time t > 0; outside the shock the gas at rest (rho0, p_amb)."""
        r = np.asarray(r, dtype=np.float64)
        R = self.shock_radius(energy, t, rho0)
        Rdot = 0.4 * R / t
        eta = r / R
        inside = eta < 1.0
        e = np.clip(eta, 0.0, 1.0)
        out = np.zeros((r.size, 5))
        out[:, 0] = np.where(inside, rho0 * np.interp(e, self.eta, self.G), rho0)
        p = np.where(inside, rho0 * Rdot * Rdot * np.interp(e, self.eta, self.P), p_amb)
        out[:, 1] = p / (self.gam - 1.0)
        out[:, 2] = np.where(inside, Rdot * np.interp(e, self.eta, self.U), 0.0)
        return out


def sedov_row_averages(edges: np.ndarray, t: float, gam: float = 1.4, energy: float = 1.0,
                       rho0: float = 1.0, p_amb: float = 0.0, sub: int = 32) -> np.ndarray:
    """Volume averages [len(edges)-1, 5] of the Sedov-Taylor state over the spherical shells
    between consecutive radial edges (sub points per shell, midpoint rule in r^3): density,
    internal energy density, radial momentum density / density (the mass-weighted v^r) and
    the total energy density rho v^2/2 + u in the fourth column."""
    S = SedovTaylor(gam)
    edges = np.asarray(edges, dtype=np.float64)
    lo, hi = edges[:-1], edges[1:]
    # points equally spaced in r^3 within each shell: each carries the same volume
    q = (np.arange(sub) + 0.5) / sub
    r = np.cbrt(lo[:, None] ** 3 + q[None, :] * (hi[:, None] ** 3 - lo[:, None] ** 3))
    w = S.profile(r.ravel(), t, energy, rho0, p_amb).reshape(r.shape[0], sub, 5)
    out = np.zeros((r.shape[0], 5))
    out[:, 0] = w[:, :, 0].mean(axis=1)
    out[:, 1] = w[:, :, 1].mean(axis=1)
    out[:, 2] = (w[:, :, 0] * w[:, :, 2]).mean(axis=1) / np.maximum(out[:, 0], 1.0e-300)
    out[:, 3] = (0.5 * w[:, :, 0] * w[:, :, 2] ** 2 + w[:, :, 1]).mean(axis=1)
    return out


def l1_rel(a: np.ndarray, b: np.ndarray, w=None) -> float:
    """sum |a - b| w / sum |b| w (w = zone volumes; uniform if None)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    w = np.ones_like(b) if w is None else np.asarray(w, dtype=np.float64)
    den = float(np.sum(np.abs(b) * w))
    return float(np.sum(np.abs(a - b) * w)) / (den if den > 0.0 else 1.0)
