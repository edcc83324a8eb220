"""GPU tests of the asynchronous dump (vb_dump_begin / vb_dump_wait): the
snapshot is exactly the interior of P in the reference's dump layout
(src/3dim/saving.jl: P.arr[:, 4:end-3, 4:end-3, 4:end-3]), it keeps the state
of the moment it was taken while later steps run, and its NaN values are
counted as the reference's NaN check would find them."""
import numpy as np
import pytest

from helpers import jet_ic, nozzle_params

pytestmark = pytest.mark.gpu


def _pinned(shape):
    import torch

    t = torch.empty(tuple(reversed(shape)), dtype=torch.float64, pin_memory=True)
    return t, t.numpy().transpose(tuple(range(len(shape) - 1, -1, -1)))


def _interior(P, dims):
    return P[(slice(None),) + (slice(3, -3),) * dims]


@pytest.mark.parametrize("dims,n,prec", [(1, (300,), "fp64"), (2, (40, 24), "fp64"), (3, (32, 16, 20), "fp64"),
                                         (3, (32, 16, 20), "fp32")])
def test_dump_is_the_interior_and_keeps_its_moment(dims, n, prec):
    from verona_b200 import Solver

    g = 4.0 / 3.0
    dxs = [1.0 / n[0]] * dims
    s = Solver(dims, n, g, dxs, recon="wenoz", riemann="hllc", rk=3, precision=prec, n_iter=50, tol=1e-12,
               floor=1e-8)
    if dims > 1:
        s.set_boundary(0, 2, nozzle_params(dims, n, 4.0, gamma=g))
    P0 = jet_ic(dims, n, gamma=g, seed=9)
    if dims == 1:  # no nozzle in 1D: a pressure jump makes the state evolve
        P0[1, : P0.shape[1] // 2] *= 100.0
    s.load_prims(P0)
    dt = 0.4 / sum(1.0 / d for d in dxs)
    s.step(dt, 2)
    before = s.prims()
    keep, out = _pinned(s.interior_shape)
    s.dump_begin(out)
    s.step(dt, 3)  # runs while the copy is in flight
    nans = s.dump_wait()
    assert nans == 0
    assert np.array_equal(out, _interior(before, dims))
    assert not np.array_equal(_interior(s.prims(), dims), out)
    # a second dump of the current state, twice in a row, and the same again after waiting
    keep2, out2 = _pinned(s.interior_shape)
    s.dump_begin(out)
    s.dump_begin(out2)
    assert s.dump_wait() == 0
    now = _interior(s.prims(), dims)
    assert np.array_equal(out, now) and np.array_equal(out2, now)


def test_dump_counts_nan_values_of_the_interior_only():
    from verona_b200 import Solver

    n = (16, 12, 10)
    P = jet_ic(3, n, seed=2)
    P[0, 5, 6, 7] = np.nan
    P[3, 9, 4, 4] = np.nan
    P[1, 0, 5, 5] = np.nan  # a ghost cell: not part of the dump
    s = Solver(3, n, 4.0 / 3.0, [1.0] * 3)
    s.load_prims(P)
    keep, out = _pinned(s.interior_shape)
    s.dump_begin(out)
    assert s.dump_wait() == 2
    assert np.isnan(out).sum() == 2


def test_dump_errors():
    from verona_b200 import Solver
    from verona_b200._lib import VBError

    s = Solver(2, (8, 8), 4.0 / 3.0, [1.0, 1.0])
    with pytest.raises(VBError, match="no state loaded"):
        s.dump_begin(np.zeros(s.interior_shape, order="F"))
    with pytest.raises(VBError, match="no dump in flight"):
        s.dump_wait()
