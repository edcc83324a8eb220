"""GPU test of vb_max_signal_speed_noalloc, the CFL reduction for callers that
cannot let the library allocate device memory (a host whose memory pool
already owns the GPU, or one that must avoid the device synchronisation an
allocation can cause). It takes the caller's arrays, keeps its partial maxima
in a fixed array inside the library, and must give the same answer as the
allocating entry point vb_max_signal_speed.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import jet_ic

pytestmark = pytest.mark.gpu


def _noalloc(dims, n, gamma, P_dev, out_dev):
    from verona_b200 import _lib

    L = _lib.lib()
    f = L.vb_max_signal_speed_noalloc
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    L.vb_noalloc_last_error.restype = C.c_char_p
    n = tuple(n) + (1,) * (3 - len(n))
    return f(dims, n[0], n[1], n[2], gamma, C.c_void_p(P_dev.data_ptr()), C.c_void_p(out_dev.data_ptr()), None)


def _case(dims, n, seed, gamma=4.0 / 3.0):
    P = jet_ic(dims, tuple(n) + (1,) * (3 - len(n)), gamma=gamma, noise=0.2, seed=seed)
    rng = np.random.default_rng(seed)
    P[2:] = rng.uniform(-4, 4, size=P[2:].shape)
    return P


@pytest.mark.parametrize("dims,n", [(3, (40, 33, 27)), (2, (300, 170)), (1, (5000,))])
def test_noalloc_matches_allocating_entry_point_twice_in_a_row(dims, n):
    import torch

    from verona_b200 import Solver

    g = 4.0 / 3.0
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for call, seed in enumerate((3, 4)):  # two calls in a row, different states
        P = _case(dims, n, seed + 10 * dims)
        P_dev = torch.from_numpy(np.ascontiguousarray(P.transpose(tuple(range(P.ndim - 1, -1, -1))))).cuda()
        rc = _noalloc(dims, n, g, P_dev, out)
        assert rc == 0, rc
        torch.cuda.synchronize()
        got = float(out.item())
        s = Solver(dims, n, g, (0.1,) * dims)
        s.load_prims(P_dev)
        ref = s.max_signal_speed()
        s.close()
        assert got > 0.0
        assert abs(got - ref) <= 1e-14 * ref, (call, got, ref)


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    from verona_b200 import _lib

    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _noalloc(3, (1024, 1024, 257), 4.0 / 3.0, dummy, out)
    assert rc == _lib.ERR_ARG
    msg = _lib.lib().vb_noalloc_last_error().decode()
    assert "exceed the maximum" in msg


def _device_state(dims, n, seed, gamma=4.0 / 3.0):
    """Random primitive state in the reference layout built on the device
    (C-order shape (n2+6, n1+6, n0+6, nv) = Fortran (nv, n0+6, n1+6, n2+6))."""
    import torch

    gen = torch.Generator(device="cuda").manual_seed(seed)
    shp = tuple(x + 6 for x in reversed(n)) + (2 + dims,)
    P = torch.empty(shp, dtype=torch.float64, device="cuda")
    P[..., 0] = 1.0 + 0.2 * torch.rand(shp[:-1], generator=gen, device="cuda", dtype=torch.float64)
    P[..., 1] = 3e-3 / (gamma - 1) * (1.0 + torch.rand(shp[:-1], generator=gen, device="cuda", dtype=torch.float64))
    P[..., 2:] = 8.0 * torch.rand(shp[:-1] + (dims,), generator=gen, device="cuda", dtype=torch.float64) - 4.0
    return P


@pytest.mark.parametrize("dims,n", [(3, (512, 512, 512)), (1, (1 << 28,))])
def test_noalloc_at_full_size(dims, n):
    """The 512^3 grid of the 3D jet (4096 partial maxima, so the final
    reduction loops over the scratch 16 times) and the largest 1D grid the
    scratch accepts (2^28 cells: all 8192 partials), against the allocating
    entry point."""
    import torch

    from verona_b200 import Solver

    g = 4.0 / 3.0
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    P_dev = _device_state(dims, n, seed=7 + dims)
    assert _noalloc(dims, n, g, P_dev, out) == 0
    torch.cuda.synchronize()
    got = float(out.item())
    s = Solver(dims, n, g, (0.1,) * dims)
    s.load_prims(P_dev)
    del P_dev
    ref = s.max_signal_speed()
    s.close()
    assert got > 0.0
    assert abs(got - ref) <= 1e-14 * ref, (got, ref)
