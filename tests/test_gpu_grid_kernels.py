"""GPU tests of the one-kernel-at-a-time entry points (vb_grid_*): each against
the oracle's restatement of the same reference kernel, on the same arrays,
bit for bit (FP64), for 1D, 2D and 3D grids."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G = 4.0 / 3.0
FLOOR = 1e-8


def _lib():
    from verona_b200 import _lib as L

    lib = L.lib()
    vp, d, i = C.c_void_p, C.c_double, C.c_int
    sig = {
        "vb_grid_fluxes": [i, i, i, i, vp, d, d, i, i, i, vp, vp],
        "vb_grid_update": [i, i, i, i, vp, vp, vp, vp, d, d, d, d, vp, vp],
        "vb_grid_con2prim": [i, i, i, i, vp, d, i, d, vp, vp, vp],
        "vb_grid_prim2con": [i, i, i, i, vp, d, vp, vp],
        "vb_grid_limit": [i, i, i, i, vp, d, vp],
    }
    for k, a in sig.items():
        getattr(lib, k).argtypes = a
        getattr(lib, k).restype = C.c_int
    lib.vb_grid_last_error.restype = C.c_char_p
    return lib


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).transpose(tuple(range(a.ndim - 1, -1, -1))))).cuda()


def _host(t):
    import torch

    torch.cuda.synchronize()
    a = t.cpu().numpy()
    return np.asfortranarray(a.transpose(tuple(range(a.ndim - 1, -1, -1))))


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _state(dims, n, seed):
    """Jet-like padded state: noisy ambient plus a relativistic stream."""
    rng = np.random.default_rng(seed)
    nv = 2 + dims
    shp = (nv,) + tuple(x + 6 for x in n)
    P = np.zeros(shp, order="F")
    P[0] = 10 ** rng.uniform(-2, 0.5, shp[1:])
    P[1] = 10 ** rng.uniform(-3, 0, shp[1:])
    for m in range(dims):
        P[2 + m] = rng.normal(0, 2.0, shp[1:])
    return P


CASES = [(1, (40,)), (2, (24, 17)), (3, (12, 10, 9))]


@pytest.mark.parametrize("dims,n", CASES)
@pytest.mark.parametrize("rec", [0, 1, 2])
@pytest.mark.parametrize("rs", [0, 1])
def test_grid_fluxes_match_oracle(dims, n, rec, rs):
    from oracle import oracle as O

    lib = _lib()
    P = _state(dims, n, 10 * dims + rec)
    Pd = _dev(P)
    nn = list(n) + [1] * (3 - dims)
    for axis in range(dims):
        Fd = _dev(np.zeros_like(P))
        assert lib.vb_grid_fluxes(dims, *nn, _p(Pd), G, FLOOR, axis, rec, rs, _p(Fd), None) == 0
        ref = O.k_fluxes(P, G, FLOOR, axis, rec, rs)
        got = _host(Fd)
        assert np.array_equal(got, ref, equal_nan=True), (axis, float(np.nanmax(np.abs(got - ref))))


@pytest.mark.parametrize("dims,n", CASES)
def test_grid_update_con2prim_prim2con_limit_match_oracle(dims, n):
    from oracle import oracle as O

    lib = _lib()
    nn = list(n) + [1] * (3 - dims)
    P = _state(dims, n, 7 + dims)
    # prim2con on all cells
    Ud = _dev(np.zeros_like(P))
    assert lib.vb_grid_prim2con(dims, *nn, _p(_dev(P)), G, _p(Ud), None) == 0
    U = O.k_ptou(P, G)
    assert np.array_equal(_host(Ud), U)
    # update with the WENOZ + HLLC fluxes of every axis
    Fs = [O.k_fluxes(P, G, FLOOR, a, O.WENOZ, O.HLLC) for a in range(dims)]
    dt, dxs = 0.2 / max(n), [1.0 / x for x in n]
    Fd = [_dev(f) for f in Fs] + [None] * (3 - dims)
    Ubd = _dev(U)
    assert lib.vb_grid_update(dims, *nn, _p(_dev(U)), *[_p(f) for f in Fd], dt, *(dxs + [1.0] * (3 - dims)),
                              _p(Ubd), None) == 0
    Ub = O.k_update(U, dt, dxs, Fs)
    # cells outside the interior are not written by either: compare the interior
    sl = (slice(None),) + (slice(3, -3),) * dims
    assert np.array_equal(_host(Ubd)[sl], Ub[sl])
    # con2prim of the updated state from the old primitives, with failure count
    import torch

    Pd = _dev(P)
    fails = torch.zeros(1, dtype=torch.int64, device="cuda")
    assert lib.vb_grid_con2prim(dims, *nn, _p(_dev(Ub)), G, 50, 1e-12, _p(Pd), _p(fails), None) == 0
    ref = O.k_utop(Ub, P, G, 50, 1e-12)
    got = _host(Pd)
    assert np.array_equal(got, ref, equal_nan=True)
    # failures are cells where every stage of the solver gave up; a stage that
    # converges to a non-finite state (sqrt of a negative, as in the reference)
    # also leaves NaN, so the count bounds the NaN cells from below
    nan_cells = int(np.isnan(ref[0][sl[1:]]).sum())
    assert int(fails.item()) <= nan_cells
    if dims < 3:
        assert int(fails.item()) == nan_cells
    # limit on all cells
    Ld = _dev(got)
    assert lib.vb_grid_limit(dims, *nn, _p(Ld), 0.05, None) == 0
    assert np.array_equal(_host(Ld), O.k_limit(got, 0.05), equal_nan=True)
