"""GPU point-kernel parity: the device reconstruction, Riemann fluxes and
con2prim (vb_point_*) on arrays of random and jet-like states, bitwise
against the oracle's scalar restatement of the same reference functions."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _states(rng, n, dims, jet=False):
    P = np.zeros((2 + dims, n))
    if jet:
        P[0] = np.where(rng.random(n) < 0.5, 0.01, 1.0) * (1 + 0.05 * rng.random(n))
        P[1] = 3e-3 * (1 + rng.random(n))
        P[2] = np.where(rng.random(n) < 0.5, 9.95 * rng.random(n), 0.3 * rng.standard_normal(n))
        P[3:] = 0.1 * rng.standard_normal((dims - 1, n))
    else:
        P[0] = 10 ** rng.uniform(-4, 1, n)
        P[1] = P[0] * 10 ** rng.uniform(-6, 2, n)
        P[2:] = 3 * rng.standard_normal((dims, n))
    return P


@pytest.mark.parametrize("method", [0, 1, 2])
def test_point_recon_bitwise(oracle, method):
    import torch

    from verona_b200 import _lib as L

    rng = np.random.default_rng(method)
    n = 4000
    q = rng.standard_normal((5, n)) * 10 ** rng.uniform(-3, 1, (1, n))
    q[:, ::7] = q[2, ::7]  # flat stencils (beta = 0)
    q[1, 1::11] = q[2, 1::11]
    dq, dout = _dev(q), torch.zeros((2, n), dtype=torch.float64, device="cuda")
    L.check(L.lib().vb_point_recon(method, C.c_void_p(dq.data_ptr()), C.c_void_p(dout.data_ptr()), n, None))
    got = dout.cpu().numpy()
    ref = np.array([oracle.recon(method, q[:, i]) for i in range(n)]).T
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("dims", [1, 2, 3])
@pytest.mark.parametrize("riemann", [0, 1])
@pytest.mark.parametrize("jet", [False, True])
def test_point_flux_bitwise(oracle, dims, riemann, jet):
    import torch

    from verona_b200 import _lib as L

    rng = np.random.default_rng(10 * dims + riemann + (100 if jet else 0))
    n = 3000
    PL, PR = _states(rng, n, dims, jet), _states(rng, n, dims, jet)
    for axis in range(dims):
        dl, dr = _dev(PL), _dev(PR)
        dF = torch.zeros((2 + dims, n), dtype=torch.float64, device="cuda")
        L.check(L.lib().vb_point_flux(dims, axis, riemann, 4.0 / 3.0, C.c_void_p(dl.data_ptr()),
                                      C.c_void_p(dr.data_ptr()), C.c_void_p(dF.data_ptr()), n, None))
        got = dF.cpu().numpy()
        ref = np.array([oracle.face_flux(dims, axis, riemann, 4.0 / 3.0, PL[:, i], PR[:, i]) for i in range(n)]).T
        same = (got == ref) | (np.isnan(got) & np.isnan(ref))
        assert same.all(), (axis, np.argwhere(~same)[:5].tolist())


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_point_con2prim_bitwise(oracle, dims):
    import torch

    from verona_b200 import _lib as L

    rng = np.random.default_rng(dims)
    n = 2000
    g = 4.0 / 3.0
    P = _states(rng, n, dims)
    P[2:] *= 0.5
    U = np.stack([oracle.prim2con(dims, g, P[:, i]) for i in range(n)], axis=1)
    guess = P * (1 + 1e-2 * rng.standard_normal(P.shape))
    dU, dP = _dev(U), _dev(guess)
    dr = torch.zeros(n, dtype=torch.int32, device="cuda")
    L.check(L.lib().vb_point_con2prim(dims, g, 50, 1e-12, C.c_void_p(dU.data_ptr()), C.c_void_p(dP.data_ptr()),
                                      C.c_void_p(dr.data_ptr()), n, None))
    got, ret = dP.cpu().numpy(), dr.cpu().numpy()
    for i in range(n):
        ref, r = oracle.con2prim(dims, g, 50, 1e-12, U[:, i], guess[:, i])
        same = (got[:, i] == ref) | (np.isnan(got[:, i]) & np.isnan(ref))
        assert same.all() and ret[i] == r, (i, got[:, i], ref, ret[i], r)


def _gpu_con2prim(dims, g, n_iter, U, guess):
    import torch

    from verona_b200 import _lib as L

    n = U.shape[1]
    dU, dP = _dev(U), _dev(guess)
    dr = torch.zeros(n, dtype=torch.int32, device="cuda")
    L.check(L.lib().vb_point_con2prim(dims, g, n_iter, 1e-12, C.c_void_p(dU.data_ptr()), C.c_void_p(dP.data_ptr()),
                                      C.c_void_p(dr.data_ptr()), n, None))
    return dP.cpu().numpy(), dr.cpu().numpy()


def test_point_con2prim_every_cascade_stage_bitwise(oracle):
    """The 3D cascade driven into each of its stages (1DW, Noble 2D with line
    search, 5D primitive Newton, bisection) and its failure exit
    (src/3dim/structs.jl:258-620): the GPU returns the same stage and the same
    bits as the oracle in every cell, and every stage occurs."""
    from collections import Counter

    from helpers import c2p_cascade_cases

    g = 4.0 / 3.0
    hist = Counter()
    for n_iter, P, guess in c2p_cascade_cases(g):
        U = np.stack([oracle.prim2con(3, g, P[:, i]) for i in range(P.shape[1])], axis=1)
        got, ret = _gpu_con2prim(3, g, n_iter, U, guess)
        for i in range(P.shape[1]):
            ref, r = oracle.con2prim(3, g, n_iter, 1e-12, U[:, i], guess[:, i])
            same = (got[:, i] == ref) | (np.isnan(got[:, i]) & np.isnan(ref))
            assert same.all() and ret[i] == r, (n_iter, i, got[:, i], ref, ret[i], r)
            hist[r] += 1
    print("stages:", dict(sorted(hist.items())))
    for stage in (1, 2, 3, 4, -1):
        assert hist[stage] >= 10, (stage, dict(hist))


def test_point_con2prim_2d_pivoting_bitwise(oracle):
    """The 2D con2prim's scaled partial pivoting (LU_dec_pivot!,
    src/2dim/structs.jl:121-208) on states where it swaps rows in most cells:
    bitwise against the oracle, iteration counts included."""
    from helpers import c2p_pivot_cases

    g = 4.0 / 3.0
    P, guess = c2p_pivot_cases(g)
    U = np.stack([oracle.prim2con(2, g, P[:, i]) for i in range(P.shape[1])], axis=1)
    got, ret = _gpu_con2prim(2, g, 50, U, guess)
    with_swaps = 0
    for i in range(P.shape[1]):
        oracle.lu4_swaps_take()
        ref, r = oracle.con2prim(2, g, 50, 1e-12, U[:, i], guess[:, i])
        with_swaps += oracle.lu4_swaps_take() > 0
        same = (got[:, i] == ref) | (np.isnan(got[:, i]) & np.isnan(ref))
        assert same.all() and ret[i] == r, (i, got[:, i], ref, ret[i], r)
    assert with_swaps >= P.shape[1] // 3, with_swaps
