"""GPU tests of the device initial-condition generator (vb_init_prims)
against its numpy restatement (oracle/ic.py): the examples' star + jet engine
in 2D and 3D and the ambient medium, P and U = PtoU(P), FP64 and FP32 bulk,
and a run that steps from it."""
import numpy as np
import pytest

from helpers import per_field_rel

pytestmark = pytest.mark.gpu


def _prim2con(P, g):
    nv = P.shape[0]
    vel = P[2:]
    gam = np.sqrt(1.0 + np.sum(vel * vel, axis=0))
    w = g * P[1] + P[0]
    U = np.empty_like(P)
    U[0] = gam * P[0]
    U[1] = (g - 1) * P[1] - gam * gam * w
    for m in range(nv - 2):
        U[2 + m] = vel[m] * gam * w
    return U


@pytest.mark.parametrize("dims,n", [(2, (122, 58)), (3, (42, 26, 18))])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_star_jet_matches_restatement(dims, n, prec):
    from oracle import ic
    from verona_b200 import Solver

    g = 4.0 / 3.0
    # a box small enough that cells fall inside the engine radius on these grids
    box = (96.0, 24.0, 0.0) if dims == 2 else (48.0, 12.0, 12.0)
    s = Solver(dims, n, g, [1.0] * dims, precision=prec)
    s.init_prims("star_jet", box=box)
    got, ref = s.prims(), ic.star_jet(dims, n, box=box)
    if prec == "fp32":
        ref32 = ref.astype(np.float32).astype(np.float64)
        assert max(per_field_rel(got, ref32)) <= 1e-6
    else:
        e = per_field_rel(got, ref)
        print(dims, "P max rel diff per field", e)
        assert max(e) <= 1e-13
        assert max(per_field_rel(s.cons(), _prim2con(ref, g))) <= 1e-13
    assert np.count_nonzero(got[2]) > 0  # the engine region is on the grid


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_ambient_matches_restatement(dims):
    from oracle import ic
    from verona_b200 import Solver

    n = {1: (200,), 2: (40, 24), 3: (16, 12, 10)}[dims]
    s = Solver(dims, n, 5.0 / 3.0, [1.0] * dims)
    s.init_prims("ambient", rho=2.0, u=0.5, noise=0.1, seed=7)
    e = per_field_rel(s.prims(), ic.ambient(dims, n, rho=2.0, u=0.5, noise=0.1, seed=7))
    assert max(e) <= 1e-13, e


def test_steps_from_the_device_condition_like_from_a_host_load():
    """A state generated on the device, and the same state read back and
    loaded from the host, step to identical results (U = PtoU(P) is formed the
    same way by both paths)."""
    from verona_b200 import Solver

    g = 4.0 / 3.0
    n = (32, 16, 24)
    opts = dict(recon="wenoz", riemann="hllc", rk=3, n_iter=50, tol=1e-12, floor=1e-8)
    a = Solver(3, n, g, [1.0 / 32] * 3, **opts)
    a.init_prims("star_jet", box=(48.0, 12.0, 12.0))
    b = Solver(3, n, g, [1.0 / 32] * 3, **opts)
    b.load_prims(a.prims())
    assert np.array_equal(a.cons(), b.cons())
    for s in (a, b):
        s.step(1e-3, 3)
    assert np.array_equal(a.prims(), b.prims())
    assert a.counters()[0] == 0


def test_rejects_unsupported_requests():
    from verona_b200 import Solver
    from verona_b200._lib import VBError

    s = Solver(1, (64,), 5.0 / 3.0, [1.0])
    with pytest.raises(VBError, match="2D or 3D"):
        s.init_prims("star_jet")
    with pytest.raises(VBError, match="r_eng"):
        Solver(2, (16, 16), 4.0 / 3.0, [1.0, 1.0]).init_prims("star_jet", r_eng=0.0)
