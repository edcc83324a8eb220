"""Shared initial conditions and comparison helpers for the tests."""
from __future__ import annotations

import numpy as np


def shock_tube_1d(N, rhoL=10.0, pL=13.33, rhoR=1.0, pR=1e-6, gamma=5.0 / 3.0, x0=0.5):
    """Marti & Mueller problem 1 on N cells of [0,1]: left state for x < x0."""
    x = (np.arange(N) + 0.5) / N
    rho = np.where(x < x0, rhoL, rhoR)
    u = np.where(x < x0, pL, pR) / (gamma - 1)
    return x, rho, u, np.zeros(N)


def n_steps(dt, T):
    """Steps of the reference's `while t < T; ...; t += dt` loop."""
    t, n = 0.0, 0
    while t < T:
        t += dt
        n += 1
    return n, t


def jet_ic(dims, n, gamma=4.0 / 3.0, noise=0.03, seed=42, rho_amb=1.0, p_amb=1e-3):
    """Ambient medium (rho with seeded multiplicative noise, p, v = 0) on the
    padded grid, in the reference's AoS Fortran layout."""
    nv = 2 + dims
    shp = (nv,) + tuple(x + 6 for x in n[:dims])
    rng = np.random.default_rng(seed)
    P = np.zeros(shp, order="F")
    P[0] = rho_amb * (1.0 + noise * rng.standard_normal(shp[1:]))
    P[1] = p_amb / (gamma - 1)
    return P


def nozzle_params(dims, n, radius, rho=0.01, p=1e-3, lorentz=10.0, gamma=4.0 / 3.0):
    ux = np.sqrt(lorentz**2 - 1)
    c1 = n[1] / 2 if dims > 1 else 0.0
    c2 = n[2] / 2 if dims > 2 else 0.0
    return [radius, c1, c2, rho, p / (gamma - 1), ux, 0.0, 0.0][: 5 + dims]


def max_rel_diff(a, b, floor=1e-300):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.maximum(np.abs(b), floor)
    return float(np.max(np.abs(a - b) / den))


def per_field_rel(a, b, axis0=True):
    """Max relative difference per field (first axis), normalised by the
    field's max magnitude (conserved fields change sign)."""
    out = []
    for v in range(a.shape[0]):
        scale = max(float(np.max(np.abs(b[v]))), 1e-300)
        out.append(float(np.max(np.abs(a[v] - b[v]))) / scale)
    return out
