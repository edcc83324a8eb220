"""GPU parity tests: the CUDA path, called through the C ABI, against the CPU
oracle on the same seeded inputs.

Bar: the plain FP64 path matches the oracle to a max relative difference of
1e-10 per conserved field (normalised by the field's max magnitude) after
the stated step count; with -fmad=false it is expected to be bit-identical
and the tests also report how many values differ at all.
"""
import os
import sys

import numpy as np
import pytest

from helpers import jet_ic, n_steps, nozzle_params, per_field_rel, shock_tube_1d

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-10  # FP64 parity bar per conserved field


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLDEN, "oracle_small.npz"))


@pytest.fixture(scope="module")
def MG():
    sys.path.insert(0, GOLDEN)
    import make_golden

    return make_golden


def _solver_nd(dims, n, P, gamma, dxs, **opt):
    from verona_b200 import Solver

    s = Solver(dims, n[:dims], gamma, dxs, **opt)
    return s


@pytest.mark.parametrize("rec", ["minmod", "ppm", "wenoz"])
def test_ref1d_matches_golden_bitwise(gold, MG, rec):
    from verona_b200 import Solver

    for r, N, steps in MG.CASES_1D:
        if r != rec:
            continue
        g = 5.0 / 3.0
        x, rho, u, ux = shock_tube_1d(N, gamma=g)
        s = Solver(1, (N,), g, (1.0 / N,), nghost=0, recon=rec, n_iter=50, tol=1e-12)
        s.load_prims(np.asfortranarray(np.stack([rho, u, ux])))
        s.step(0.4 / N, steps)
        P = s.prims()
        np.testing.assert_array_equal(P, gold[f"r1d_{rec}_P"])
        np.testing.assert_array_equal(s.cons(), gold[f"r1d_{rec}_U"])


@pytest.mark.parametrize("rec", ["minmod", "ppm", "wenoz"])
def test_ref1d_shock_tube_full_run_matches_oracle(oracle, rec):
    """Config 1: N = 1024, t = 0.4, CFL 0.4, through the Verona1D mirror."""
    from verona_b200 import EosTypes, Verona1D

    g = 5.0 / 3.0
    N = 1024
    x, rho, u, ux = shock_tube_1d(N, gamma=g)
    dx = 1.0 / N
    dt = 0.4 * dx
    P = Verona1D.ParVector1D(N, rho, u, ux)
    out = Verona1D.HARM_HLL(P, N, dt, dx, 0.4, EosTypes.Polytrope(g), 0.4 / 3, rec, 50, 1e-12)
    assert len(out) == 4  # t = 0 plus three dumps
    s = oracle.Solver1DRef(rho, u, ux, g, rec, 50, 1e-12)
    n, _ = n_steps(dt, 0.4)
    s.step(dt, dx, n)
    ref = s.prims()
    got = np.stack([P.arr1, P.arr2, P.arr3])
    assert max(per_field_rel(got, ref)) <= TOL
    print(f"{rec}: {int(np.sum(got != ref))} of {got.size} values differ from the oracle")


def test_nd_matches_golden(gold, MG):
    from verona_b200 import Solver

    for c in MG.CASES_ND:
        dims, n, rec, rs, rk, steps = c
        g = 4.0 / 3.0
        P0 = jet_ic(dims, n, gamma=g, noise=0.03, seed=7)
        dxs = [1.0 / n[a] for a in range(dims)]
        s = Solver(dims, n[:dims], g, dxs, recon=rec, riemann=rs, rk=rk, n_iter=50, tol=1e-12, floor=1e-8)
        s.set_boundary(0, 2, nozzle_params(dims, n, 3.0, gamma=g))
        s.load_prims(P0)
        dt = 0.4 / sum(1.0 / d for d in dxs)
        s.step(dt, steps)
        name = MG.nd_case_name(c)
        P, U = s.prims(), s.cons()
        eP = per_field_rel(P, gold[name + "_P"])
        eU = per_field_rel(U, gold[name + "_U"])
        print(name, "max rel P", max(eP), "U", max(eU), "differing:", int(np.sum(P != gold[name + "_P"])))
        assert max(eU) <= TOL and max(eP) <= TOL, (name, eP, eU)


@pytest.mark.parametrize("dims,n,steps", [(2, (64, 48, 1), 20), (3, (24, 20, 18), 8)])
@pytest.mark.parametrize("rk", [2, 3])
def test_jet_parity_with_decaying_inflow(oracle, dims, n, steps, rk):
    """A reference-style jet (WENOZ + HLL) with the TurnOff boundary: x-lo fixed
    with a u^x decay that switches on mid-run, zero-gradient elsewhere."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    P0 = jet_ic(dims, n, gamma=g, noise=0.03, seed=11)
    # jet state in the x-lo ghosts inside r < 4 cells
    yy = np.arange(n[1] + 6) - 3 + 0.5 - n[1] / 2
    zz = (np.arange(n[2] + 6) - 3 + 0.5 - n[2] / 2) if dims == 3 else np.zeros(1)
    Y, Z = np.meshgrid(yy, zz, indexing="ij")
    inside = (Y**2 + Z**2) < 16.0
    m = inside if dims == 3 else inside[:, 0]
    for i in range(3):
        for v, val in ((0, 0.01), (1, 3e-3), (2, np.sqrt(99.0))):
            P0[v, i][m] = val
    dxs = [1.0 / n[0]] * dims
    dt = 0.4 / sum(1.0 / d for d in dxs)
    decay = (2, 3.5 * dt, 1e9, 1 - dt / 0.05)
    s = Solver(dims, n[:dims], g, dxs, recon="wenoz", riemann="hll", rk=rk, n_iter=50, tol=1e-12, floor=1e-8)
    s.set_boundary(0, 1, decay)
    s.load_prims(P0)
    s.step(dt, steps)
    o = oracle.SolverND(dims, n[:dims], P0, g, 1e-8, 50, 1e-12, oracle.WENOZ, oracle.HLL, rk)
    o.set_grid(*(dxs + [1.0] * (3 - dims)))
    o.set_boundary(0, oracle.BC_FIXED, decay)
    o.step(dt, steps)
    eU = per_field_rel(s.cons(), o.cons())
    eP = per_field_rel(s.prims(), o.prims())
    print(dims, rk, "U", eU, "P", eP)
    assert max(eU) <= TOL and max(eP) <= TOL


def test_fp32_bulk_close_to_fp64():
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (32, 24, 24)
    P0 = jet_ic(3, n, gamma=g, noise=0.03, seed=5)
    dxs = [1.0 / 32] * 3
    dt = 0.4 / sum(1.0 / d for d in dxs)
    out = {}
    for prec in ("fp64", "fp32"):
        s = Solver(3, n, g, dxs, recon="wenoz", riemann="hllc", rk=3, precision=prec, n_iter=50, tol=1e-12,
                   floor=1e-8)
        s.set_boundary(0, 2, nozzle_params(3, n, 4.0, gamma=g))
        s.load_prims(P0)
        s.step(dt, 10)
        out[prec] = s.prims()
        assert s.counters()[0] == 0
    a, b = out["fp32"][:, 3:-3, 3:-3, 3:-3], out["fp64"][:, 3:-3, 3:-3, 3:-3]
    l1_rho = np.mean(np.abs(a[0] - b[0])) / np.mean(np.abs(b[0]))
    l1_p = np.mean(np.abs(a[1] - b[1])) / np.mean(np.abs(b[1]))
    print("fp32 bulk: L1 rho", l1_rho, "L1 p", l1_p)
    assert l1_rho < 1e-5 and l1_p < 1e-5


def test_max_signal_speed_matches_numpy():
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (20, 18, 16)
    rng = np.random.default_rng(2)
    P0 = jet_ic(3, n, gamma=g, noise=0.2, seed=2)
    P0[2:] = rng.uniform(-3, 3, size=P0[2:].shape)
    s = Solver(3, n, g, (0.1, 0.1, 0.1))
    s.load_prims(P0)
    c = s.max_signal_speed()
    Q = P0[:, 3:-3, 3:-3, 3:-3]
    lor = np.sqrt(Q[2] ** 2 + Q[3] ** 2 + Q[4] ** 2 + 1)
    cs = np.sqrt(g * (g - 1) * Q[1] / (Q[0] + g * Q[1]))
    sig = cs**2 / (lor**2 * (1 - cs**2))
    best = 0.0
    for d in range(3):
        v = Q[2 + d] / lor
        r = np.sqrt(sig * (1 - v**2 + sig))
        best = max(best, np.max(np.abs((v + r) / (1 + sig))), np.max(np.abs((v - r) / (1 + sig))))
    assert abs(c - best) <= 1e-14 * best


def test_host_and_device_loads_agree():
    import torch

    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (16, 12)
    P0 = jet_ic(2, n + (1,), gamma=g, seed=9)
    a = Solver(2, n, g, (0.1, 0.1))
    a.load_prims(P0)
    b = Solver(2, n, g, (0.1, 0.1))
    b.load_prims(torch.from_numpy(np.ascontiguousarray(P0.transpose(2, 1, 0))).cuda())
    a.step(0.01, 3)
    b.step(0.01, 3)
    np.testing.assert_array_equal(a.prims(), b.prims())
    d = b.store_prims()
    np.testing.assert_array_equal(d.cpu().numpy().transpose(2, 1, 0), a.prims())


def test_reference_mirror_3d_harm_hll(oracle):
    """Verona3D.HARM_HLL with the TurnOff-equivalent boundary, against the oracle."""
    from verona_b200 import EosTypes, Verona3D

    g = 4.0 / 3.0
    n = (16, 12, 12)
    P0 = jet_ic(3, n, gamma=g, seed=13)
    P0[2, :3, 4:10, 4:10] = 3.0
    P = Verona3D.ParVector3D(*n)
    P.arr[:] = P0
    dx = 0.05
    dt = 0.4 / (3 / dx)
    Tmax, drops = 12 * dt, 4 * dt
    bnd = Verona3D.turnoff_boundary(dt, 0.1, 9 * dt)
    dumps = []
    i = Verona3D.HARM_HLL(None, P, (1, 1, 1), (4, 4, 4), dt, dx, dx, dx, Tmax, EosTypes.Polytrope(g), drops, 1e-8,
                          ".", False, 50, 1e-12, bnd, dump=lambda k, t, s: dumps.append(k))
    assert i == len(dumps) - 1 and i >= 2
    o = oracle.SolverND(3, n, P0, g, 1e-8, 50, 1e-12, oracle.WENOZ, oracle.HLL, 2)
    o.set_grid(dx, dx, dx)
    for face, kind, par in bnd:
        o.set_boundary(face, kind, par)
    steps, _ = n_steps(dt, Tmax)
    o.step(dt, steps)
    assert max(per_field_rel(P.arr, o.prims())) <= TOL


def test_healthy_run_has_no_failures_and_counts_iterations():
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (24, 16, 16)
    s = Solver(3, n, g, (0.05,) * 3, stats=1, n_iter=50, tol=1e-12, floor=1e-8)
    s.set_boundary(0, 2, nozzle_params(3, n, 3.0, gamma=g))
    s.load_prims(jet_ic(3, n, gamma=g))
    s.step(0.005, 4)
    c = s.counters()
    assert c[0] == 0
    assert c[3] == 2 * 4 * 24 * 16 * 16  # cells solved: 2 stages x 4 steps
    assert c[2] >= c[3]


def test_errors_are_reported_not_trapped():
    from verona_b200 import Solver, VBError

    s = Solver(2, (8, 8), 4.0 / 3.0, (0.1, 0.1))
    with pytest.raises(VBError, match="vb_load_prims first"):
        s.step(0.01, 1)
    with pytest.raises(VBError, match="face"):
        s.set_boundary(5, 0)


@pytest.mark.parametrize("rec", [0, 1, 2])
@pytest.mark.parametrize("rs", [0, 1])
@pytest.mark.parametrize("rk", [2, 3])
@pytest.mark.parametrize("variant", ["fused", "split", "box"])
def test_zmarch_kernel_parity(oracle, rec, rs, rk, variant):
    """3D grids with x/y extents that are multiples of the 32x8 tile run the
    z-marching kernel; 70 cells in z make two z-ranges, the second partial."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (32, 16, 70)
    P0 = jet_ic(3, n, gamma=g, noise=0.03, seed=21)
    dxs = [1.0 / 32] * 3
    dt = 0.4 / sum(1.0 / d for d in dxs)
    noz = nozzle_params(3, n, 5.0, gamma=g)
    s = Solver(3, n, g, dxs, recon=rec, riemann=rs, rk=rk, n_iter=50, tol=1e-12, floor=1e-8)
    s.set_tuning(split_con2prim=int(variant == "split"), force_box=int(variant == "box"))
    s.set_boundary(0, 2, noz)
    s.load_prims(P0)
    s.step(dt, 2)
    o = oracle.SolverND(3, n, P0, g, 1e-8, 50, 1e-12, rec, rs, rk)
    o.set_grid(*dxs)
    o.set_boundary(0, oracle.BC_NOZZLE, noz)
    o.step(dt, 2)
    got, ref = s.prims(), o.prims()
    eU = per_field_rel(s.cons(), o.cons())
    eP = per_field_rel(got, ref)
    print("zm", rec, rs, rk, "U", max(eU), "P", max(eP), "differing", int(np.sum(got != ref)))
    assert max(eU) <= TOL and max(eP) <= TOL


@pytest.mark.parametrize("rs", ["hll", "hllc"])
@pytest.mark.parametrize("variant", ["split", "fused"])
@pytest.mark.parametrize("rec", ["wenoz", "ppm", "minmod"])
def test_fp32_pair_kernel_matches_scalar_kernel(rs, variant, rec):
    """The z-pair FP32 stencil kernel (two cells per thread on packed FP32
    instructions) against the one-cell-per-thread FP32 kernel and the FP64
    path, for every reconstruction (WENOZ on packed pairs; PPM and MINMOD
    lane by lane through the scalar FP32 limiters). 69 cells in z give a
    64-cell range and a 5-cell range, whose last pair is incomplete. The two
    FP32 kernels round differently (hand-written packed contraction, folded
    constants, the HLL / HLLC flux), so they agree to FP32 rounding, and each
    stays within the FP32-bulk error bar of the FP64 run."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (32, 16, 69)
    P0 = jet_ic(3, n, gamma=g, noise=0.03, seed=8)
    dxs = [1.0 / 32] * 3
    dt = 0.4 / sum(1.0 / d for d in dxs)
    out = {}
    for name, prec, pairs in (("fp64", "fp64", 0), ("scalar", "fp32", 0), ("pairs", "fp32", 1)):
        s = Solver(3, n, g, dxs, recon=rec, riemann=rs, rk=3, precision=prec, n_iter=50, tol=1e-12, floor=1e-8)
        s.set_tuning(split_con2prim=int(variant == "split"), fp32_pairs=pairs)
        s.set_boundary(0, 2, nozzle_params(3, n, 5.0, gamma=g))
        s.load_prims(P0)
        s.step(dt, 6)
        out[name] = s.prims()[:, 3:-3, 3:-3, 3:-3]
        assert s.counters()[0] == 0
        assert np.all(np.isfinite(out[name]))

    def l1(a, b, v):
        return float(np.mean(np.abs(a[v] - b[v])) / np.mean(np.abs(b[v])))

    for v in range(5):
        d = l1(out["pairs"], out["scalar"], v) if v < 2 else float(
            np.mean(np.abs(out["pairs"][v] - out["scalar"][v])))
        print(rec, rs, variant, "var", v, "pairs vs scalar FP32:", d)
        assert d < 2e-6
    for name in ("scalar", "pairs"):
        e = (l1(out[name], out["fp64"], 0), l1(out[name], out["fp64"], 1))
        print(rec, rs, variant, name, "L1 rho, p vs FP64:", e)
        assert max(e) < 1e-5


def _hllc_star_pressure(g, rho, p, u):
    """p* of the HLLC star state (Mignone & Bodo 2005) between the 1D states
    (rho, p, -u) and (rho, p, +u), u the normal four-velocity: the face is
    left to the HLL flux where p* <= 0."""
    def side(uu):
        gam = np.sqrt(1 + uu * uu)
        v = uu / gam
        w = rho + g / (g - 1) * p
        U = np.array([rho * gam, w * gam * gam * v, w * gam * gam - p])
        F = np.array([rho * gam * v, w * gam * gam * v * v + p, w * gam * gam * v])
        sig = g * p / w / (gam * gam * (1 - g * p / w))
        r = np.sqrt(sig * (1 - v * v + sig))
        return U, F, (v + r) / (1 + sig), (v - r) / (1 + sig)

    UL, FL, lpL, lmL = side(-u)
    UR, FR, lpR, lmR = side(u)
    lR, lL = max(lpL, lpR), min(lmL, lmR)
    Uh = (lR * UR - lL * UL - (FR - FL)) / (lR - lL)
    Fh = (lR * FL - lL * FR + lR * lL * (UR - UL)) / (lR - lL)
    b = Uh[2] + Fh[1]
    ls = 2 * Uh[1] / (b + np.sqrt(max(b * b - 4 * Fh[2] * Uh[1], 0.0)))
    return Fh[1] - Fh[2] * ls


@pytest.mark.parametrize("variant", ["split", "fused"])
def test_fp32_pair_kernel_hllc_fallback_faces(variant):
    """Streams that move apart along x and along z (the pair axis): at the
    two separating planes the HLLC star pressure is negative, so those faces
    take the HLL flux, the rest the HLLC star flux (lanes of one pair differ
    where a pair straddles the z plane). The z-pair kernel forms the passive
    components' HLL flux only where a lane falls back; it must agree with the
    one-cell-per-thread FP32 kernel to FP32 rounding and stay within the
    FP32-bulk bar of the FP64 run."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (32, 16, 69)
    assert _hllc_star_pressure(g, 1.0, 0.1, 0.5) < 0
    P0 = jet_ic(3, n, gamma=g, noise=0.03, seed=11, p_amb=0.1)
    P0[2, : 3 + n[0] // 2] = -0.5
    P0[2, 3 + n[0] // 2 :] = 0.5
    P0[4, :, :, : 3 + 34] = -0.5
    P0[4, :, :, 3 + 34 :] = 0.5
    dxs = [1.0 / 32] * 3
    dt = 0.4 / sum(1.0 / d for d in dxs)
    out = {}
    for name, prec, pairs in (("fp64", "fp64", 0), ("scalar", "fp32", 0), ("pairs", "fp32", 1)):
        s = Solver(3, n, g, dxs, recon="wenoz", riemann="hllc", rk=3, precision=prec, n_iter=50, tol=1e-12,
                   floor=1e-8)
        s.set_tuning(split_con2prim=int(variant == "split"), fp32_pairs=pairs)
        s.load_prims(P0)
        s.step(dt, 6)
        out[name] = s.prims()[:, 3:-3, 3:-3, 3:-3]
        assert s.counters()[0] == 0
        assert np.all(np.isfinite(out[name]))

    def l1(a, b, v):
        return float(np.mean(np.abs(a[v] - b[v])) / np.mean(np.abs(b[v])))

    for v in range(5):
        d = l1(out["pairs"], out["scalar"], v) if v < 2 else float(
            np.mean(np.abs(out["pairs"][v] - out["scalar"][v])))
        print(variant, "var", v, "pairs vs scalar FP32:", d)
        assert d < 2e-6
    for name in ("scalar", "pairs"):
        e = (l1(out[name], out["fp64"], 0), l1(out[name], out["fp64"], 1))
        print(variant, name, "L1 rho, p vs FP64:", e)
        assert max(e) < 1e-5


@pytest.mark.parametrize("rs", ["hll", "hllc"])
@pytest.mark.parametrize("variant", ["split", "fused"])
def test_tma_tiles_match_cp_async_planes_bitwise(rs, variant):
    """The z-pair kernel with its planes brought in as TMA tiles (a ring of 6
    plane boxes per CTA) against the same kernel staging the planes by
    per-thread loads and 4-byte asynchronous copies: identical arithmetic on
    identical values, so P and U agree bitwise. 64 cells in x give two tiles,
    the second box reaching past the padded row (70 cells, pitched to 72),
    where TMA fills zeros that no stencil reads; 69 cells in z end in an
    incomplete pair."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (64, 16, 69)
    P0 = jet_ic(3, n, gamma=g, noise=0.03, seed=9)
    dxs = [1.0 / 64] * 3
    dt = 0.4 / sum(1.0 / d for d in dxs)
    out = {}
    for tma in (0, 1):
        s = Solver(3, n, g, dxs, recon="wenoz", riemann=rs, rk=3, precision="fp32", n_iter=50, tol=1e-12, floor=1e-8)
        s.set_tuning(split_con2prim=int(variant == "split"), fp32_pairs=1, tma_tiles=tma)
        assert s.get_tuning()["tma_tiles"] == tma
        assert s.tma_tiles_active == bool(tma)
        s.set_boundary(0, 2, nozzle_params(3, n, 5.0, gamma=g))
        s.load_prims(P0)
        s.step(dt, 5)
        c = s.counters()
        assert c[0] == 0 and c[4] == 0  # no con2prim failure, no plane wait ran out
        out[tma] = (s.prims(), s.cons())
        assert np.all(np.isfinite(out[tma][0]))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("rec,rs", [("wenoz", "hllc"), ("ppm", "hll"), ("minmod", "hllc")])
def test_2d_tma_tiles_match_loaded_tiles_bitwise(precision, rec, rs):
    """The 2D box-tile stage kernel with its tile (halo on both axes, every
    variable) brought in as one TMA tile, against the same kernel staging
    each axis-extended tile by per-thread loads: the same values reach the
    same arithmetic, so in FP64 (built without FMA contraction) P and U agree
    bitwise. The FP32-bulk units are built with contraction, and the compiler
    may fuse a multiply-add in one instantiation and not the other, so there
    the two agree to FP32 rounding (max 1e-7 relative per field measured).
    70 x 21 interior cells leave partial tiles on both axes, whose boxes reach
    past the padded extents (TMA fills zeros there, which no valid cell
    reads)."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (70, 21, 1)
    P0 = jet_ic(2, n, gamma=g, noise=0.03, seed=12)
    dxs = [1.0 / 70] * 2
    dt = 0.4 / sum(1.0 / d for d in dxs)
    out = {}
    for tma in (0, 1):
        s = Solver(2, n[:2], g, dxs, recon=rec, riemann=rs, rk=3, precision=precision, n_iter=50, tol=1e-12,
                   floor=1e-8)
        s.set_tuning(tma_tiles=tma)
        assert s.tma_tiles_active == bool(tma)
        s.set_boundary(0, 2, nozzle_params(2, n, 3.0, gamma=g))
        s.load_prims(P0)
        s.step(dt, 6)
        c = s.counters()
        assert c[0] == 0 and c[4] == 0
        out[tma] = (s.prims(), s.cons())
        assert np.all(np.isfinite(out[tma][0]))
    eP, eU = max(per_field_rel(out[1][0], out[0][0])), max(per_field_rel(out[1][1], out[0][1]))
    print(precision, rec, rs, "TMA vs loaded: differing P", int(np.sum(out[0][0] != out[1][0])), "max rel P", eP,
          "U", eU)
    if precision == "fp64":
        assert np.array_equal(out[0][0], out[1][0])
        assert np.array_equal(out[0][1], out[1][1])
    else:
        assert eP < 1e-6 and eU < 1e-6


def test_diverging_reference_newton_is_counted_as_failure():
    """A 1D tube the reference's 1D Newton cannot follow at CFL 0.4 (from the
    seeded batch workload): the single-grid solver keeps the reference's
    values and counts the cells whose state became non-finite as failures."""
    from verona_b200 import Solver
    from verona_b200.batch import riemann_problems

    specs, prims = riemann_problems(42, gamma=5.0 / 3.0)
    sp = specs[62]
    s = Solver(1, sp["n"], 5.0 / 3.0, (sp["dx"],), recon=sp["recon"], riemann="hllc", rk=3, n_iter=50, tol=1e-12,
               floor=1e-8)
    s.load_prims(prims[62])
    s.step(sp["dt"], 10)
    bad = int(np.sum(~np.isfinite(s.prims())))
    c = s.counters()
    print("non-finite values", bad, "counters", c.tolist())
    assert bad > 0 and c[0] > 0


@pytest.mark.parametrize("rec", ["minmod", "ppm", "wenoz"])
def test_hllc_keeps_an_isolated_contact_exact_on_the_gpu(oracle, rec):
    """GPU twin of the HLLC known answer: the stationary contact stays exactly
    two-valued (p and v exactly unchanged) after 40 SSP-RK3 steps of the
    ghosted 1D solver, bit-identical to the oracle."""
    from helpers import contact_1d
    from verona_b200 import Solver

    g = 5.0 / 3.0
    N = 64
    P0 = contact_1d(N, gamma=g)
    s = Solver(1, (N,), g, (1.0 / N,), recon=rec, riemann="hllc", rk=3, n_iter=50, tol=1e-12, floor=1e-10)
    s.load_prims(P0)
    s.step(0.4 / N, 40)
    got = s.prims()
    o = oracle.SolverND(1, (N,), P0, g, 1e-10, 50, 1e-12, oracle.RECON[rec], oracle.HLLC, 3)
    o.set_grid(1.0 / N)
    o.step(0.4 / N, 40)
    np.testing.assert_array_equal(got, o.prims())
    Q = got[:, 3:-3]
    assert np.max(np.minimum(np.abs(Q[0] - 10.0), np.abs(Q[0] - 1.0))) == 0.0
    assert np.all(Q[1] * (g - 1) == 1.0) and np.all(Q[2] == 0.0)


@pytest.mark.parametrize("rec", ["minmod", "ppm", "wenoz"])
def test_hllc_shock_tube_matches_oracle_and_exact_solution(oracle, rec):
    """Marti & Mueller problem 1 (config 1's states) through the ghosted 1D
    solver with HLLC + SSP-RK3 at N = 512 to t = 0.4: bit-identical to the
    oracle, and within the oracle's L1 density error of the exact solution."""
    from oracle import exact_riemann as ER

    from helpers import mm1_ghosted
    from verona_b200 import Solver

    g = 5.0 / 3.0
    N = 512
    x, P0 = mm1_ghosted(N, g)
    dt = 0.4 / N
    n, t = n_steps(dt, 0.4)
    s = Solver(1, (N,), g, (1.0 / N,), recon=rec, riemann="hllc", rk=3, n_iter=50, tol=1e-12, floor=1e-10)
    s.load_prims(P0)
    s.step(dt, n)
    got = s.prims()
    o = oracle.SolverND(1, (N,), P0, g, 1e-10, 50, 1e-12, oracle.RECON[rec], oracle.HLLC, 3)
    o.set_grid(1.0 / N)
    o.step(dt, n)
    ref = o.prims()
    assert max(per_field_rel(got, ref)) <= TOL
    print(f"{rec}: {int(np.sum(got != ref))} of {got.size} values differ from the oracle")
    ex = ER.solve(10.0, 13.33, 0.0, 1.0, 1e-6, 0.0, g, x, t)
    assert float(np.mean(np.abs(got[0, 3:-3] - ex[0]))) < 0.05


@pytest.mark.parametrize("rec", [0, 1, 2])
@pytest.mark.parametrize("rs", [0, 1])
@pytest.mark.parametrize("variant", ["fused", "split", "box"])
def test_fp64_contracted_path_within_parity_bar(oracle, rec, rs, variant):
    """The plain FP64 path with FMA contraction (vb_tuning.fp64_contract):
    not bit-identical to the reference's rounding, but within the parity bar
    of 1e-10 per conserved field of the oracle after 6 SSP-RK3 steps of a jet
    on the z-marching grid (70 cells in z: two z-ranges, the second partial),
    for every kernel variant."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (32, 16, 70)
    P0 = jet_ic(3, n, gamma=g, noise=0.03, seed=23)
    dxs = [1.0 / 32] * 3
    dt = 0.4 / sum(1.0 / d for d in dxs)
    noz = nozzle_params(3, n, 5.0, gamma=g)
    s = Solver(3, n, g, dxs, recon=rec, riemann=rs, rk=3, n_iter=50, tol=1e-12, floor=1e-8)
    s.set_tuning(split_con2prim=int(variant == "split"), force_box=int(variant == "box"), fp64_contract=1)
    assert s.get_tuning()["fp64_contract"] == 1
    s.set_boundary(0, 2, noz)
    s.load_prims(P0)
    s.step(dt, 6)
    o = oracle.SolverND(3, n, P0, g, 1e-8, 50, 1e-12, rec, rs, 3)
    o.set_grid(*dxs)
    o.set_boundary(0, oracle.BC_NOZZLE, noz)
    o.step(dt, 6)
    got, ref = s.prims(), o.prims()
    eU = per_field_rel(s.cons(), o.cons())
    eP = per_field_rel(got, ref)
    print("contracted", rec, rs, variant, "U", max(eU), "P", max(eP), "differing", int(np.sum(got != ref)))
    assert max(eU) <= TOL and max(eP) <= TOL
    assert np.sum(got != ref) > 0  # the contracted kernels did run


@pytest.mark.parametrize("dims", [1, 2])
@pytest.mark.parametrize("contract", [0, 1])
def test_fp64_1d_2d_inflow_within_parity_bar(oracle, dims, contract):
    """The FP64 box-tile kernels of the 1D and 2D grids (the 2D tiles by TMA),
    WENOZ + HLLC + SSP-RK3 with an inflow (2D: the nozzle; 1D: FIXED x-lo
    ghosts holding u^x = 3), against the oracle after 10 steps: bit-identical
    with the reference's rounding, within 1e-10 per field with FMA
    contraction (vb_tuning.fp64_contract)."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (200, 1, 1) if dims == 1 else (64, 48, 1)
    P0 = jet_ic(dims, n, gamma=g, noise=0.03, seed=24)
    dxs = [1.0 / n[0]] * dims
    dt = 0.4 / sum(1.0 / d for d in dxs)
    if dims == 1:
        P0[2, :3] = 3.0  # an inflow into the tube through the x-lo ghosts
    s = Solver(dims, n[:dims], g, dxs, recon="wenoz", riemann="hllc", rk=3, n_iter=50, tol=1e-12, floor=1e-8)
    s.set_tuning(fp64_contract=contract)
    o = oracle.SolverND(dims, n[:dims], P0, g, 1e-8, 50, 1e-12, oracle.WENOZ, oracle.HLLC, 3)
    o.set_grid(*(dxs + [1.0] * (3 - dims)))
    if dims == 2:
        noz = nozzle_params(2, n, 4.0, gamma=g)
        s.set_boundary(0, 2, noz)
        o.set_boundary(0, oracle.BC_NOZZLE, noz)
    else:
        s.set_boundary(0, 1)
        o.set_boundary(0, oracle.BC_FIXED, (-1.0, 0.0, 0.0, 1.0))
    s.load_prims(P0)
    s.step(dt, 10)
    o.step(dt, 10)
    got, ref = s.prims(), o.prims()
    eU = per_field_rel(s.cons(), o.cons())
    eP = per_field_rel(got, ref)
    print("inflow", dims, "contract", contract, "U", max(eU), "P", max(eP), "differing", int(np.sum(got != ref)),
          "max |P|", float(np.max(np.abs(got))))
    if contract == 0:
        np.testing.assert_array_equal(got, ref)
    assert max(eU) <= TOL and max(eP) <= TOL


@pytest.mark.parametrize("rec", ["minmod", "wenoz"])
def test_fp64_contracted_1d_shock_tube_within_parity_bar(oracle, rec):
    """Marti & Mueller problem 1 through the ghosted 1D solver with the
    FMA-contracted FP64 kernels, HLLC + SSP-RK3, N = 256, 60 steps: within
    1e-10 per field of the oracle."""
    from helpers import mm1_ghosted
    from verona_b200 import Solver

    g = 5.0 / 3.0
    N = 256
    _, P0 = mm1_ghosted(N, g)
    s = Solver(1, (N,), g, (1.0 / N,), recon=rec, riemann="hllc", rk=3, n_iter=50, tol=1e-12, floor=1e-10)
    s.set_tuning(fp64_contract=1)
    s.load_prims(P0)
    s.step(0.4 / N, 60)
    o = oracle.SolverND(1, (N,), P0, g, 1e-10, 50, 1e-12, oracle.RECON[rec], oracle.HLLC, 3)
    o.set_grid(1.0 / N)
    o.step(0.4 / N, 60)
    got, ref = s.prims(), o.prims()
    e = per_field_rel(got, ref)
    print("contracted mm1", rec, e, "differing", int(np.sum(got != ref)))
    assert max(e) <= TOL


@pytest.mark.parametrize("dims", [1, 2, 3])
@pytest.mark.parametrize("rec", [0, 1, 2])
@pytest.mark.parametrize("rs", [0, 1])
def test_fp64_static_ambient_matches_oracle_bitwise(oracle, dims, rec, rs):
    """A noise-free ambient (equal neighbours, v = 0 exactly) with a nozzle
    (2D, 3D) or a FIXED inflow (1D): the static region feeds exact zeros to
    the smoothness ratios, the velocities' face values, the HLL/HLLC
    numerators and the con2prim, which the FP64 kernels divide without the
    IEEE sequence (qdiv). The result must stay bit-identical to the oracle,
    which divides the plain way."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = {1: (128, 1, 1), 2: (64, 40, 1), 3: (32, 16, 24)}[dims]
    P0 = jet_ic(dims, n, gamma=g, noise=0.0)
    dxs = [1.0 / n[0]] * dims
    dt = 0.4 / sum(1.0 / d for d in dxs)
    if dims == 1:
        P0[2, :3] = 3.0
    s = Solver(dims, n[:dims], g, dxs, recon=rec, riemann=rs, rk=3, n_iter=50, tol=1e-12, floor=1e-8)
    o = oracle.SolverND(dims, n[:dims], P0, g, 1e-8, 50, 1e-12, rec, rs, 3)
    o.set_grid(*(dxs + [1.0] * (3 - dims)))
    if dims == 1:
        s.set_boundary(0, 1)
        o.set_boundary(0, oracle.BC_FIXED, (-1.0, 0.0, 0.0, 1.0))
    else:
        noz = nozzle_params(dims, n, 4.0, gamma=g)
        s.set_boundary(0, 2, noz)
        o.set_boundary(0, oracle.BC_NOZZLE, noz)
    s.load_prims(P0)
    s.step(dt, 4)
    o.step(dt, 4)
    got, ref = s.prims(), o.prims()
    print("static", dims, rec, rs, "differing", int(np.sum(got != ref)))
    np.testing.assert_array_equal(got, ref)
    assert max(per_field_rel(s.cons(), o.cons())) <= TOL


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_2d_split_con2prim_matches_fused_bitwise(precision):
    """The 2D box stage with its con2prim in a separate kernel
    (split_con2prim = 1: the box kernel writes U, k_c2p_2d solves each cell
    from it) against the fused box stage: the same U and the same guess
    reach the same per-cell Newton, so every value agrees bit for bit."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (64, 40, 1)
    P0 = jet_ic(2, n, gamma=g, noise=0.03, seed=26)
    dxs = [1.0 / 64] * 2
    dt = 0.4 / sum(1.0 / d for d in dxs)
    out = []
    for split in (0, 1):
        s = Solver(2, n[:2], g, dxs, recon="wenoz", riemann="hllc", rk=3, precision=precision, n_iter=50,
                   tol=1e-12, floor=1e-8, stats=1)
        s.set_tuning(split_con2prim=split)
        s.set_boundary(0, 2, nozzle_params(2, n, 4.0, gamma=g))
        s.load_prims(P0)
        s.step(dt, 5)
        out.append((s.prims(), s.cons(), s.counters()))
    np.testing.assert_array_equal(out[1][0], out[0][0])
    np.testing.assert_array_equal(out[1][1], out[0][1])
    assert list(out[1][2]) == list(out[0][2]) and out[0][2][3] > 0


@pytest.mark.parametrize("precision,gate", [("fp64", 0), ("fp32", 0), ("fp32", 1)])
def test_2d_previous_w_con2prim(oracle, precision, gate):
    """The previous-W con2prim guess in 2D (VB_GUESS_PREVIOUS_W: the W Newton
    on the state padded to three momenta, gated to FP32 where options.c2p_fp32
    admits the cell) against the oracle's reference 2D Newton on the 2D jet:
    FP64 within the Newton tolerance per field, FP32 bulk within its L1 bar."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (64, 40, 1)
    P0 = jet_ic(2, n, gamma=g, noise=0.03, seed=27)
    dxs = [1.0 / 64] * 2
    dt = 0.4 / sum(1.0 / d for d in dxs)
    noz = nozzle_params(2, n, 4.0, gamma=g)
    s = Solver(2, n[:2], g, dxs, recon="wenoz", riemann="hllc", rk=3, precision=precision, guess="previous_w",
               n_iter=50, tol=1e-12, floor=1e-8, stats=1, c2p_fp32=gate)
    s.set_boundary(0, 2, noz)
    s.load_prims(P0)
    s.step(dt, 8)
    o = oracle.SolverND(2, n[:2], P0, g, 1e-8, 50, 1e-12, oracle.WENOZ, oracle.HLLC, 3)
    o.set_grid(*(dxs + [1.0]))
    o.set_boundary(0, oracle.BC_NOZZLE, noz)
    o.step(dt, 8)
    got, ref = s.prims(), o.prims()
    c = s.counters()
    assert c[0] == 0 and np.all(np.isfinite(got)) and c[3] > 0
    if precision == "fp64":
        e = per_field_rel(got, ref)
        print("2D previous-W FP64 vs oracle: max rel per field", e, "iterations per cell", c[2] / c[3])
        assert max(e) < 1e-8
    else:
        a, b = got[:, 3:-3, 3:-3], ref[:, 3:-3, 3:-3]
        l1 = [float(np.mean(np.abs(a[v] - b[v])) / np.mean(np.abs(b[v]))) for v in (0, 1)]
        print("2D previous-W FP32 gate", gate, "L1 rho, p vs oracle", l1)
        assert max(l1) < 1e-5
