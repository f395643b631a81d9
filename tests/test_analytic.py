"""The analytic Sedov-Taylor solution (medusa_b200.analytic.SedovTaylor, Sedov's closed form)
checked independently: against a direct integration of the self-similar Euler ODEs from
the strong-shock jump conditions (RK4 in ln eta, stopped at eta = 0.2 where integrating
inwards is still well conditioned), against the tabulated xi0 (Kamm & Timmes 2007), the
energy it carries, and its behaviour at the centre."""
import math

import numpy as np
import pytest

from medusa_b200 import analytic as A


def _ode_profile(g, eta_min=0.2, steps=20000):
    """(eta, G, U, P) from eta = 1 inwards: rho = rho0 G, v = R' U, p = rho0 R'^2 P with
    continuity, momentum and constant entropy along particle paths."""
    def rhs(s, y):
        eta = math.exp(s)
        G, U, P = y
        D = U - eta
        dU = (1.5 * U * G * D - 3.0 * P + 2.0 * g * P * U / eta) / (G * D * D - g * P)
        dG = -G * (dU + 2.0 * U / eta) / D
        dP = P * (3.0 / D + g * dG / G)
        return np.array([dG, dU, dP]) * eta

    h = math.log(eta_min) / steps
    s = 0.0
    y = np.array([(g + 1.0) / (g - 1.0), 2.0 / (g + 1.0), 2.0 / (g + 1.0)])
    out = [(1.0, *y)]
    for _ in range(steps):
        k1 = rhs(s, y)
        k2 = rhs(s + 0.5 * h, y + 0.5 * h * k1)
        k3 = rhs(s + 0.5 * h, y + 0.5 * h * k2)
        k4 = rhs(s + h, y + h * k3)
        y = y + h / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
        s += h
        out.append((math.exp(s), *y))
    return np.array(out[::-1])


@pytest.mark.parametrize("gam", [4.0 / 3.0, 1.4, 5.0 / 3.0])
def test_sedov_closed_form_matches_the_similarity_odes(gam):
    S = A.SedovTaylor(gam)
    t = _ode_profile(gam)
    for k, F in ((1, S.G), (2, S.U), (3, S.P)):
        got = np.interp(t[:, 0], S.eta, F)
        assert np.max(np.abs(got - t[:, k]) / np.abs(t[:, k])) <= 5.0e-6


def test_sedov_xi0_and_centre():
    for gam, xi0 in ((1.4, 1.033), (5.0 / 3.0, 1.152)):
        S = A.SedovTaylor(gam)
        assert abs(S.xi0 - xi0) <= 1.0e-3
        # at the centre v = (2 r / 5 t) / gamma and the pressure stays finite
        assert abs(S.U[1] / S.eta[1] - 1.0 / gam) <= 1.0e-9
        assert 0.2 < S.P[1] / (2.0 / (gam + 1.0)) < 0.5


def test_sedov_profile_carries_the_blast_energy():
    S = A.SedovTaylor(1.4)
    t = 0.05
    R = S.shock_radius(1.0, t)
    r = np.linspace(0.0, R, 400001)
    w = S.profile(r, t)
    e = 0.5 * w[:, 0] * w[:, 2] ** 2 + w[:, 1]
    energy = float(np.sum(0.5 * (e[1:] * r[1:] ** 2 + e[:-1] * r[:-1] ** 2) * np.diff(r))) * 4.0 * math.pi
    assert abs(energy - 1.0) <= 1.0e-4
    mass = float(np.sum(0.5 * (w[1:, 0] * r[1:] ** 2 + w[:-1, 0] * r[:-1] ** 2) * np.diff(r))) * 4.0 * math.pi
    assert abs(mass - 4.0 / 3.0 * math.pi * R ** 3) <= 1.0e-4 * mass   # the swept-up mass
    # the jump at the shock and the undisturbed gas outside
    out = S.profile(np.array([R * (1.0 - 1.0e-9), R * 1.01]), t, p_amb=1.0e-5)
    assert abs(out[0, 0] - 6.0) <= 1.0e-4 and out[1, 0] == 1.0 and out[1, 2] == 0.0
