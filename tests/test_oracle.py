"""CPU tests that pin the oracle (the C restatement of the reference) before
it is trusted as the parity reference of the GPU path.

The reference ships no tests or golden vectors and cannot run here (Julia),
so the pins are: the published exact solution of Marti & Mueller problem 1,
the self-convergence idea of examples/Shock1Dim/Resolution_comp.jl,
uniform-state preservation, mirror symmetry, conservation, the P->U->P round
trip, and the committed oracle fixtures of tests/golden/.
"""
import json
import os

import numpy as np
import pytest

from helpers import jet_ic, n_steps, nozzle_params, shock_tube_1d

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_exact_solver_matches_published_star_state():
    from oracle import exact_riemann as ER

    with open(os.path.join(GOLDEN, "mm1_star.json")) as f:
        star = json.load(f)
    ps, vs, rl, rr, sl, sr = ER.star_state(10.0, 13.33, 0.0, 1.0, 1e-6, 0.0, 5.0 / 3.0)
    got = {"p_star": ps, "v_star": vs, "rho_L_star": rl, "rho_R_star": rr, "shock_R": sr}
    for k, pub in star["published"].items():
        # the published values carry 3-4 significant digits
        assert abs(got[k] - pub) <= 6e-4 * max(1.0, abs(pub)), (k, got[k], pub)
        assert abs(got[k] - star["exact"][k]) <= 1e-9 * abs(star["exact"][k]), k


@pytest.mark.parametrize("rec", ["minmod", "ppm", "wenoz"])
def test_oracle_1d_converges_to_exact_solution(oracle, rec):
    from oracle import exact_riemann as ER

    g = 5.0 / 3.0
    errs = []
    for N in (128, 256, 512):
        x, rho, u, ux = shock_tube_1d(N, gamma=g)
        s = oracle.Solver1DRef(rho, u, ux, g, rec, 50, 1e-12)
        dx = 1.0 / N
        dt = 0.4 * dx
        n, t = n_steps(dt, 0.4)
        s.step(dt, dx, n)
        P = s.prims()
        assert np.all(np.isfinite(P))
        ex = ER.solve(10.0, 13.33, 0.0, 1.0, 1e-6, 0.0, g, x, t)
        errs.append(float(np.mean(np.abs(P[0] - ex[0]))))
    assert errs[0] > errs[1] > errs[2], errs
    assert errs[2] < 0.06, errs


@pytest.mark.parametrize("dims", [2, 3])
def test_oracle_uniform_state_is_preserved(oracle, dims):
    n = (10, 8, 6)[:dims]
    g = 4.0 / 3.0
    P = jet_ic(dims, n + (1,) * (3 - dims), gamma=g, noise=0.0)
    P[2] = 0.3  # uniform drift
    for rec in (oracle.MINMOD, oracle.PPM, oracle.WENOZ):
        for rs in (oracle.HLL, oracle.HLLC):
            s = oracle.SolverND(dims, n, P, g, 1e-8, 50, 1e-12, rec, rs, 2)
            s.set_grid(0.1, 0.1, 0.1)
            s.step(0.01, 3)
            Q = s.prims()
            assert np.max(np.abs(Q - P)) <= 1e-12 * np.max(np.abs(P)), (rec, rs)


def test_oracle_2d_mirror_symmetry(oracle):
    n = (16, 16)
    g = 4.0 / 3.0
    P = jet_ic(2, n + (1,), gamma=g, noise=0.03, seed=3)
    P[:] = 0.5 * (P + P[:, :, ::-1])  # symmetric in y
    P[3] = 0.0
    s = oracle.SolverND(2, n, P, g, 1e-8, 50, 1e-12, oracle.WENOZ, oracle.HLL, 2)
    s.set_grid(1 / 16, 1 / 16)
    s.set_boundary(0, oracle.BC_NOZZLE, nozzle_params(2, (16, 16, 1), 3.0, gamma=g))
    s.step(0.4 / 32, 5)
    Q = s.prims()
    M = Q[:, :, ::-1].copy()
    M[3] = -M[3]
    assert np.max(np.abs(Q - M)) <= 1e-12 * np.max(np.abs(Q))


@pytest.mark.parametrize("rs", ["hll", "hllc"])
def test_oracle_conservation(oracle, rs):
    """Outflow box whose edges stay at the same ambient state: the fluxes
    through opposite faces cancel, so sum(U) over the interior is conserved."""
    n = (24, 24)
    g = 4.0 / 3.0
    P = jet_ic(2, n + (1,), gamma=g, noise=0.0)
    xi, yj = np.meshgrid(np.arange(30) - 14.5, np.arange(30) - 14.5, indexing="ij")
    P[0] += 0.5 * np.exp(-(xi**2 + yj**2) / 8.0)
    rsv = oracle.HLL if rs == "hll" else oracle.HLLC
    s = oracle.SolverND(2, n, P, g, 1e-8, 50, 1e-12, oracle.WENOZ, rsv, 3)
    s.set_grid(1.0, 1.0)
    U0 = s.cons()[:, 3:-3, 3:-3].sum(axis=(1, 2))
    s.step(0.2, 4)
    U1 = s.cons()[:, 3:-3, 3:-3].sum(axis=(1, 2))
    for v in range(4):
        scale = max(abs(U0[0]), abs(U0[1]))
        assert abs(U1[v] - U0[v]) <= 1e-12 * scale, (v, U0[v], U1[v])


def test_oracle_con2prim_round_trip(oracle):
    rng = np.random.default_rng(1)
    for dims in (1, 2, 3):
        for _ in range(300):
            g = rng.choice([4.0 / 3.0, 5.0 / 3.0])
            rho = 10 ** rng.uniform(-4, 1)
            p = rho * 10 ** rng.uniform(-6, 2)
            lor = 10 ** rng.uniform(0, np.log10(40.0 if dims == 3 else 10.0))
            d = rng.normal(size=dims)
            d /= np.linalg.norm(d)
            uvec = np.sqrt(lor**2 - 1) * d
            if dims == 3 and (rho / lor < 1e-6 or p / (g - 1) < 1e-6):
                continue  # the 3D solver floors rho and u at 1e-8 by design (src/3dim/structs.jl:602-603)
            P = np.concatenate([[rho, p / (g - 1)], uvec])
            U = oracle.prim2con(dims, g, P)
            guess = P * (1 + 1e-3 * rng.standard_normal(P.shape))
            Q, r = oracle.con2prim(dims, g, 200, 1e-13, U, guess)
            assert r >= 1, (dims, P, r)
            # compare through the conserved state (primitive u is ill-conditioned when p << rho)
            assert np.max(np.abs(oracle.prim2con(dims, g, Q) - U)) <= 1e-9 * np.max(np.abs(U)), (dims, P, Q)


def test_oracle_reproduces_golden_fixtures(oracle):
    import sys

    sys.path.insert(0, GOLDEN)
    import make_golden as MG

    gold = np.load(os.path.join(GOLDEN, "oracle_small.npz"))
    for rec, N, steps in MG.CASES_1D:
        _, P, U, _, _ = MG.run_1d_case(rec, N, steps)
        np.testing.assert_array_equal(P, gold[f"r1d_{rec}_P"])
        np.testing.assert_array_equal(U, gold[f"r1d_{rec}_U"])
    for c in MG.CASES_ND:
        _, P, U, _, _ = MG.run_nd_case(c)
        name = MG.nd_case_name(c)
        np.testing.assert_array_equal(P, gold[name + "_P"])
        np.testing.assert_array_equal(U, gold[name + "_U"])


def test_oracle_3d_con2prim_floors_like_the_reference(oracle):
    """u below 1e-8 comes back floored at 1e-8 (src/3dim/structs.jl:603)."""
    g = 4.0 / 3.0
    P = np.array([1e-3, 1e-10, 0.5, 0.1, -0.2])
    U = oracle.prim2con(3, g, P)
    Q, r = oracle.con2prim(3, g, 50, 1e-12, U, P)
    assert r >= 1 and Q[1] == 1e-8


def test_ic_noise_stream_is_standard_normal_and_reproducible():
    """The counter-based noise of the initial conditions: N(0, 1) moments,
    no correlation between neighbouring cells, the same values for the same
    (seed, cell) and different ones for another seed."""
    from oracle import ic

    c = np.arange(1 << 20, dtype=np.uint64)
    z = ic.cell_normal(42, c)
    assert abs(z.mean()) < 5e-3 and abs(z.std() - 1.0) < 5e-3
    assert abs(np.corrcoef(z[:-1], z[1:])[0, 1]) < 5e-3
    assert np.array_equal(z[1000:2000], ic.cell_normal(42, c[1000:2000]))
    assert np.mean(np.abs(z - ic.cell_normal(43, c))) > 0.5


def test_ic_star_jet_follows_the_examples():
    """Engine region, envelope and outer medium of the 3D example's initial
    condition (examples/Jet3D/HARM_jet_breakout.jl:82-114) on a small grid."""
    from oracle import ic

    P = ic.star_jet(3, (58, 26, 26))  # 64 x 32 x 32 padded: dx = 7.5
    rho, u, ux = P[0], P[1], P[2]
    assert np.all(P[3] == 0) and np.all(P[4] == 0)
    assert np.all(rho > 0) and np.all(u > 0)
    # cell (1,16,16) 1-based: X = 7.5, Y = Z = 0 -> inside R_max, outside R_eng (5): no jet
    assert ux[0, 15, 15] == 0.0 and abs(rho[0, 15, 15] / (2.5e-2 * (100 / 7.5) ** 2) - 1) < 0.2
    assert np.all(rho[-1] == 1e-4)  # X = 480 is outside R_max
    assert np.allclose(u[rho == 1e-4], 1e-9)


def test_cascade_inputs_reach_every_con2prim_stage(oracle):
    """The inputs of the GPU cascade test reach every stage of the 3D
    con2prim (1DW, Noble 2D, 5D Newton, bisection) and its failure exit, so
    the bitwise comparison there covers each stage's code."""
    from collections import Counter

    from helpers import c2p_cascade_cases

    g = 4.0 / 3.0
    hist = Counter()
    for n_iter, P, guess in c2p_cascade_cases(g):
        for i in range(P.shape[1]):
            U = oracle.prim2con(3, g, P[:, i])
            _, r = oracle.con2prim(3, g, n_iter, 1e-12, U, guess[:, i])
            hist[r] += 1
    print(dict(sorted(hist.items())))
    for stage in (1, 2, 3, 4, -1):
        assert hist[stage] >= 10, (stage, dict(hist))


def test_pivot_inputs_swap_rows_in_the_2d_lu(oracle):
    """The inputs of the GPU pivoting test make the 2D con2prim's scaled
    partial pivoting swap rows in at least a third of the cells."""
    from helpers import c2p_pivot_cases

    g = 4.0 / 3.0
    P, guess = c2p_pivot_cases(g)
    with_swaps = 0
    for i in range(P.shape[1]):
        U = oracle.prim2con(2, g, P[:, i])
        oracle.lu4_swaps_take()
        oracle.con2prim(2, g, 50, 1e-12, U, guess[:, i])
        with_swaps += oracle.lu4_swaps_take() > 0
    assert with_swaps >= P.shape[1] // 3, with_swaps


@pytest.mark.parametrize("rec", ["minmod", "ppm", "wenoz"])
def test_hllc_keeps_an_isolated_contact_exact(oracle, rec):
    """Known answer of the HLLC solver (Mignone & Bodo 2005): a stationary
    contact (equal p, v = 0, density jump) is an exact solution of the
    scheme, so the density stays exactly two-valued and p, v exactly
    unchanged after 40 SSP-RK3 steps; the HLL flux of the reference smears it
    over several cells."""
    from helpers import contact_1d

    g = 5.0 / 3.0
    N = 64
    dev = {}
    for rs in (oracle.HLL, oracle.HLLC):
        s = oracle.SolverND(1, (N,), contact_1d(N, gamma=g), g, 1e-10, 50, 1e-12, oracle.RECON[rec], rs, 3)
        s.set_grid(1.0 / N)
        s.step(0.4 / N, 40)
        Q = s.prims()[:, 3:-3]
        dev[rs] = float(np.max(np.minimum(np.abs(Q[0] - 10.0), np.abs(Q[0] - 1.0))))
        if rs == oracle.HLLC:
            assert dev[rs] == 0.0
            assert np.all(Q[1] * (g - 1) == 1.0) and np.all(Q[2] == 0.0)
    assert dev[oracle.HLL] > 1.0, dev


@pytest.mark.parametrize("rec", ["minmod", "ppm", "wenoz"])
def test_hllc_converges_to_the_exact_solution_like_hll(oracle, rec):
    """Marti & Mueller problem 1 through the ghosted 1D solver with SSP-RK3:
    with HLLC the L1 density error against the exact solution falls with N at
    least as HLL's does (within 5 % at every N)."""
    from oracle import exact_riemann as ER

    from helpers import mm1_ghosted

    g = 5.0 / 3.0
    errs = {}
    for rs in (oracle.HLL, oracle.HLLC):
        errs[rs] = []
        for N in (128, 256, 512):
            x, P = mm1_ghosted(N, g)
            s = oracle.SolverND(1, (N,), P, g, 1e-10, 50, 1e-12, oracle.RECON[rec], rs, 3)
            dt = 0.4 / N
            s.set_grid(1.0 / N)
            n, t = n_steps(dt, 0.4)
            s.step(dt, n)
            Q = s.prims()[:, 3:-3]
            assert np.all(np.isfinite(Q))
            ex = ER.solve(10.0, 13.33, 0.0, 1.0, 1e-6, 0.0, g, x, t)
            errs[rs].append(float(np.mean(np.abs(Q[0] - ex[0]))))
    for rs in errs:
        e = errs[rs]
        assert e[0] > e[1] > e[2], (rs, e)
    assert all(c <= 1.05 * h for c, h in zip(errs[oracle.HLLC], errs[oracle.HLL])), errs
    assert errs[oracle.HLLC][2] < 0.05, errs
