"""Exact solution of the 1D special-relativistic Riemann problem for an ideal
gas with no tangential velocity -- TEST INFRASTRUCTURE ONLY.

Restated from the published method of Marti & Mueller (1994, J. Fluid Mech.
258, 317; review: Living Rev. Relativ. 6, 7 (2003), section 4.3):
  * rarefactions from the Riemann invariant J+- = atanh(v) +- F(c_s) with
    F(c) = (1/sqrt(G-1)) ln((sqrt(G-1)+c)/(sqrt(G-1)-c)) for an isentrope,
  * shocks from the Taub adiabat and the relativistic jump conditions,
  * p* from v*_L(p) = v*_R(p) by bracketed root finding.
It is the known-answer pin for the 1D oracle (config: Marti & Mueller
problem 1, rho_L=10, p_L=13.33, rho_R=1, p_R~0, G=5/3).
"""
from __future__ import annotations

import math

import numpy as np
from scipy.optimize import brentq


def _h(rho, p, g):
    return 1.0 + g / (g - 1.0) * p / rho


def _cs(rho, p, g):
    return math.sqrt(g * p / (rho * _h(rho, p, g)))


def _raref(rho_a, p_a, v_a, p_b, g, sign):
    """Velocity and density behind a rarefaction; sign=+1 left wave, -1 right."""
    a = math.sqrt(g - 1.0)
    rho_b = rho_a * (p_b / p_a) ** (1.0 / g)
    ca, cb = _cs(rho_a, p_a, g), _cs(rho_b, p_b, g)
    A = (((a - cb) / (a + cb)) * ((a + ca) / (a - ca))) ** (sign * 2.0 / a)
    v_b = ((1 + v_a) * A - (1 - v_a)) / ((1 + v_a) * A + (1 - v_a))
    return v_b, rho_b


def _shock(rho_a, p_a, v_a, p_b, g, sign):
    """Velocity, density and shock speed behind a shock; sign=+1 right, -1 left."""
    h_a = _h(rho_a, p_a, g)
    dp = p_b - p_a
    A = 1.0 - (g - 1.0) * dp / (g * p_b)
    B = 1.0 - A
    Cc = -h_a * h_a - h_a / rho_a * dp
    h_b = (-B + math.sqrt(B * B - 4 * A * Cc)) / (2 * A)
    rho_b = g * p_b / ((g - 1.0) * (h_b - 1.0))
    j2 = dp / (h_a / rho_a - h_b / rho_b)
    j = sign * math.sqrt(j2)
    W_a = 1.0 / math.sqrt(1.0 - v_a * v_a)
    r2w2 = rho_a * rho_a * W_a * W_a
    Vs = (r2w2 * v_a + sign * abs(j) * math.sqrt(j2 + r2w2 * (1.0 - v_a * v_a))) / (r2w2 + j2)
    W_s = 1.0 / math.sqrt(1.0 - Vs * Vs)
    v_b = (h_a * W_a * v_a + W_s * dp / j) / (h_a * W_a + dp * (W_s * v_a / j + 1.0 / (rho_a * W_a)))
    return v_b, rho_b, Vs


def _wave(rho_a, p_a, v_a, p, g, sign):
    if p < p_a:
        v, rho = _raref(rho_a, p_a, v_a, p, g, sign)
        return v, rho, None
    return _shock(rho_a, p_a, v_a, p, g, -sign)


def star_state(rhoL, pL, vL, rhoR, pR, vR, g):
    """Returns (p*, v*, rho*_L, rho*_R, left shock speed or None, right shock speed or None)."""

    def f(p):
        return _wave(rhoL, pL, vL, p, g, +1)[0] - _wave(rhoR, pR, vR, p, g, -1)[0]

    lo, hi = min(pL, pR) * 1e-6 + 1e-300, max(pL, pR) * 1e3
    ps = brentq(f, lo, hi, xtol=1e-15, rtol=1e-14, maxiter=500)
    vLs, rLs, sL = _wave(rhoL, pL, vL, ps, g, +1)
    vRs, rRs, sR = _wave(rhoR, pR, vR, ps, g, -1)
    return ps, 0.5 * (vLs + vRs), rLs, rRs, sL, sR


def _fan(rho_a, p_a, v_a, p_star, xi, g, sign):
    """State inside a rarefaction fan at similarity coordinate xi."""

    def lam(p):
        v, rho = _raref(rho_a, p_a, v_a, p, g, sign)
        c = _cs(rho, p, g)
        return ((v - c) / (1 - v * c) if sign > 0 else (v + c) / (1 + v * c)) - xi

    p = brentq(lam, min(p_a, p_star), max(p_a, p_star), xtol=1e-15, rtol=1e-14)
    v, rho = _raref(rho_a, p_a, v_a, p, g, sign)
    return rho, p, v


def solve(rhoL, pL, vL, rhoR, pR, vR, g, x, t, x0=0.5):
    """Exact (rho, p, v) at positions x and time t > 0."""
    ps, vs, rLs, rRs, sL, sR = star_state(rhoL, pL, vL, rhoR, pR, vR, g)
    cL, cR = _cs(rhoL, pL, g), _cs(rhoR, pR, g)
    cLs, cRs = _cs(rLs, ps, g), _cs(rRs, ps, g)
    out = np.zeros((3, len(x)))
    for n, xx in enumerate(np.asarray(x, dtype=float)):
        xi = (xx - x0) / t
        if xi < vs:  # left of contact
            if sL is None:
                head = (vL - cL) / (1 - vL * cL)
                tail = (vs - cLs) / (1 - vs * cLs)
                if xi <= head:
                    st = (rhoL, pL, vL)
                elif xi >= tail:
                    st = (rLs, ps, vs)
                else:
                    st = _fan(rhoL, pL, vL, ps, xi, g, +1)
            else:
                st = (rhoL, pL, vL) if xi < sL else (rLs, ps, vs)
        else:
            if sR is None:
                head = (vR + cR) / (1 + vR * cR)
                tail = (vs + cRs) / (1 + vs * cRs)
                if xi >= head:
                    st = (rhoR, pR, vR)
                elif xi <= tail:
                    st = (rRs, ps, vs)
                else:
                    st = _fan(rhoR, pR, vR, ps, xi, g, -1)
            else:
                st = (rhoR, pR, vR) if xi > sR else (rRs, ps, vs)
        out[:, n] = st
    return out
