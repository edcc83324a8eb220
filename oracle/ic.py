"""Initial conditions of the reference's jet examples, restated in numpy --
TEST INFRASTRUCTURE ONLY (vb_init_prims is tested against it; the product never
imports it).

Follows examples/Jet3D/HARM_jet_breakout.jl:72-118 (3D) and
examples/Jet2D/HARM_jet_breakout.jl:37-72 (2D) on every padded cell: cell
(i, j, k), 1-based over the padded grid, sits at X = i dx, Y = j dy - box_Y,
Z = k dz - box_Z, dx = box_X / (Nx + 6), dy = 2 box_Y / (Ny + 6),
dz = 2 box_Z / (Nz + 6). The reference draws its density noise from
per-thread MersenneTwister streams (values depend on the thread schedule);
the library and this restatement use one standard normal per padded cell:
splitmix64 (Steele, Lea, Flood 2014) words of (seed, cell index) through
Box-Muller, so the two agree to floating-point rounding of log / sqrt / cos.
"""
from __future__ import annotations

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x):
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def cell_normal(seed, c):
    """Standard normal of padded cell index c (uint64 array) in stream seed."""
    c = np.asarray(c, dtype=np.uint64)
    s = np.uint64(seed)
    h1 = splitmix64(s ^ splitmix64(np.uint64(2) * c))
    h2 = splitmix64(s ^ splitmix64(np.uint64(2) * c + np.uint64(1)))
    u1 = ((h1 >> np.uint64(11)) + np.uint64(1)).astype(np.float64) * 2.0**-53
    u2 = (h2 >> np.uint64(11)).astype(np.float64) * 2.0**-53
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def example_params(dims):
    """The examples' values (examples/Jet3D/HARM_jet_breakout.jl:46-61,
    examples/Jet2D/HARM_jet_breakout.jl:26-36)."""
    p = dict(seed=42, noise=3e-2, r_max=100.0, rho0=2.5e-2, temp=1e-5, outer=1e-4, gamma0=10.0, engine_temp=1e-5)
    if dims == 3:
        p.update(box=(480.0, 120.0, 120.0), r_eng=5.0, engine_rho=1e-2)
    else:
        p.update(box=(800.0, 200.0, 0.0), r_eng=2.0, engine_rho=1e-3)
    return p


def star_jet(dims, n, **kw):
    """Primitive AoS array (Fortran order, (2 + dims, Nx+6, ...)) of the star + jet engine."""
    p = example_params(dims)
    p.update(kw)
    shp = tuple(x + 6 for x in n[:dims])
    idx = np.indices(shp, dtype=np.float64)  # 0-based padded (i, j[, k])
    c = np.zeros(shp, dtype=np.uint64)
    stride = 1
    for a in range(dims):
        c += np.indices(shp)[a].astype(np.uint64) * np.uint64(stride)
        stride *= shp[a]
    dx = [(1.0 if a == 0 else 2.0) * p["box"][a] / shp[a] for a in range(dims)]
    X = (idx[0] + 1) * dx[0]
    Y = (idx[1] + 1) * dx[1] - p["box"][1]
    R2 = X * X + Y * Y
    if dims == 3:
        Z = (idx[2] + 1) * dx[2] - p["box"][2]
        R2 = R2 + Z * Z
    R = np.sqrt(R2)
    nz = p["noise"] * cell_normal(p["seed"], c)
    f = p["r_max"] / np.where(R < p["r_eng"], p["r_eng"], R)
    rho = np.where(R < p["r_max"], p["rho0"] * f * f * (1.0 + nz), p["outer"])
    u = rho * p["temp"]
    eng = R < p["r_eng"]
    s = np.sqrt(X * X + Y * Y) if dims == 3 else Y
    with np.errstate(over="ignore"):  # cosh^8 -> inf far from the engine: v = 0 there, unused
        v = 1.0 / (1.0 - 1.0 / p["gamma0"] ** 2) / np.cosh(s / p["r_eng"]) ** 8
    ux = np.where(eng, p["gamma0"] * v, 0.0)
    rho = np.where(eng, rho * p["engine_rho"], rho)
    u = np.where(eng, rho * p["engine_temp"], u)
    P = np.zeros((2 + dims,) + shp, order="F")
    P[0], P[1], P[2] = rho, u, ux
    return P


def ambient(dims, n, rho=1.0, u=3e-3, noise=3e-2, seed=42):
    shp = tuple(x + 6 for x in n[:dims])
    c = np.arange(int(np.prod(shp)), dtype=np.uint64).reshape(shp, order="F")
    P = np.zeros((2 + dims,) + shp, order="F")
    P[0] = rho * (1.0 + noise * cell_normal(seed, c))
    P[1] = u
    return P
