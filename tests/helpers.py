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


def c2p_cascade_cases(gamma=4.0 / 3.0, n=1500, seed=5):
    """Inputs that drive the 3D con2prim cascade (src/3dim/structs.jl:258-620)
    into every stage: (n_iter, U (5, n), guess (5, n)) triples. Relativistic
    states up to Lorentz 40 with a 1 % guess and n_iter 50 mostly converge in
    the 1DW Newton (stage 1) and some in the Noble 2D Newton (2); a 50 % guess
    with n_iter 3 exhausts the Newton stages and reaches the bisection (4) or
    fails (-1); cold states (p/rho 1e-8..1e-5) with n_iter 5 also reach the 5D
    primitive Newton (3)."""
    rng = np.random.default_rng(seed)

    def states(cold):
        P = np.zeros((5, n))
        P[0] = 10 ** rng.uniform(-4, 1, n)
        P[1] = P[0] * 10 ** (rng.uniform(-8, -5, n) if cold else rng.uniform(-6, 2, n)) / (gamma - 1)
        lor = 10 ** rng.uniform(0, np.log10(40.0), n)
        d = rng.normal(size=(3, n))
        d /= np.linalg.norm(d, axis=0)
        P[2:] = np.sqrt(lor**2 - 1) * d
        return P

    out = []
    for n_iter, pert, cold in ((50, 1e-2, False), (3, 0.5, False), (5, 0.3, True)):
        P = states(cold)
        guess = P * (1 + pert * rng.standard_normal(P.shape))
        guess[:2] = np.abs(guess[:2])
        out.append((n_iter, P, guess))
    return out


def c2p_pivot_cases(gamma=4.0 / 3.0, n=2000, seed=6):
    """2D states up to Lorentz 20 with a 30 % guess: the pivoted 4x4 LU of the
    2D con2prim (src/2dim/structs.jl:121-208) swaps rows in most cells.
    Returns (P (4, n), guess (4, n))."""
    rng = np.random.default_rng(seed)
    P = np.zeros((4, n))
    P[0] = 10 ** rng.uniform(-4, 1, n)
    P[1] = P[0] * 10 ** rng.uniform(-6, 2, n) / (gamma - 1)
    lor = 10 ** rng.uniform(0, np.log10(20.0), n)
    d = rng.normal(size=(2, n))
    d /= np.linalg.norm(d, axis=0)
    P[2:] = np.sqrt(lor**2 - 1) * d
    guess = P * (1 + 0.3 * rng.standard_normal(P.shape))
    guess[:2] = np.abs(guess[:2])
    return P, guess


def contact_1d(N, rhoL=10.0, rhoR=1.0, p=1.0, gamma=5.0 / 3.0):
    """An isolated stationary contact on N cells of [0, 1] with 3 ghosts per
    side: equal pressure, zero velocity, a density jump at x = 0.5. Padded AoS
    (3, N + 6), Fortran order."""
    x = (np.arange(N + 6) - 3 + 0.5) / N
    P = np.zeros((3, N + 6), order="F")
    P[0] = np.where(x < 0.5, rhoL, rhoR)
    P[1] = p / (gamma - 1)
    return P


def mm1_ghosted(N, gamma=5.0 / 3.0):
    """Marti & Mueller problem 1 on N cells of [0, 1] with 3 ghosts per side
    (the generic ghosted 1D solver). Returns (x of the interior, P (3, N + 6))."""
    x = (np.arange(N + 6) - 3 + 0.5) / N
    P = np.zeros((3, N + 6), order="F")
    P[0] = np.where(x < 0.5, 10.0, 1.0)
    P[1] = np.where(x < 0.5, 13.33, 1e-6) / (gamma - 1)
    return x[3:-3], P
