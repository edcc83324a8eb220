"""Failure paths on the GPU, made without faulting, trapping or hanging it.

* A bounded device wait that runs out: the batch kernel's wait of a tile for
  the previous stage of its problem, with its bound set to one poll, so that
  waits on dependencies still in flight give up. The launch must end, the
  host must learn of it through vb_batch_check (VB_ERR_TIMEOUT, the count in
  VB_CNT_TIMEOUT), and the context must stay usable: after a rollback with
  the default bound the batch reproduces a fresh run bit for bit.
* Corrupted conserved states made on the host (NaN, |S| >= E, negative
  energy, negative density, negative internal energy, and cells given a
  tight iteration cap) through the con2prim entry points: the GPU returns
  the same codes, failure counts and bits (NaN included) as the oracle. The
  reference marks cells without a root with NaN (src/3dim/structs.jl:612-619)
  and has no other failure signal.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import per_field_rel

pytestmark = pytest.mark.gpu

G = 5.0 / 3.0
OPTS = dict(riemann="hllc", n_iter=50, tol=1e-12, floor=1e-8)


def _quadrant(n, seed):
    from verona_b200.batch import _state

    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    P = np.zeros((4, n + 6, n + 6), order="F")
    x = (np.arange(n + 6) - 3 + 0.5) * dx
    X, Y = np.meshgrid(x, x, indexing="ij")
    for m in ((X >= 0.5) & (Y >= 0.5), (X < 0.5) & (Y >= 0.5), (X < 0.5) & (Y < 0.5), (X >= 0.5) & (Y < 0.5)):
        s = _state(rng, G, 2)
        for v in range(4):
            P[v][m] = s[v]
    return {"dims": 2, "n": (n, n), "recon": "wenoz", "dx": dx, "dy": dx, "dt": 0.4 / (2 * n)}, P


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_wait_that_runs_out_is_reported_and_recoverable(precision):
    from verona_b200 import _lib
    from verona_b200.batch import Batch

    spec, P = _quadrant(512, seed=5)
    b = Batch([spec], G, rk=3, precision=precision, **OPTS)
    b.load_prims(0, P)
    b.checkpoint()
    b.reset_counters()
    # one poll: a stage-2 tile taken while stage-1 tiles of its problem are
    # still running gives up at once, and every tile after it in turn
    b.set_wait_limit(1)
    b.step(2)
    rc = b.check()
    cnt = b.counters()
    print("timed-out launch:", rc, b.last_error, "timeouts", int(cnt[4]))
    assert rc == _lib.ERR_TIMEOUT and "gave up" in b.last_error
    assert cnt[4] > 0
    # the context is usable: default bound, restore, run again
    b.set_wait_limit(0)
    b.rollback()
    b.reset_counters()
    b.step(2)
    assert b.check() == 0 and b.counters()[4] == 0
    got = b.prims(0)
    b.close()
    f = Batch([spec], G, rk=3, precision=precision, **OPTS)
    f.load_prims(0, P)
    f.step(2)
    assert f.check() == 0
    np.testing.assert_array_equal(got, f.prims(0))
    f.close()


def _corrupt(dims, n, seed, g):
    """Healthy relativistic states with every fifth one corrupted in one of
    five ways; returns (U (nv, n), guess P (nv, n), kind per state)."""
    from oracle import oracle as O

    rng = np.random.default_rng(seed)
    nv = 2 + dims
    P = np.zeros((nv, n))
    P[0] = 10 ** rng.uniform(-2, 0.5, n)
    P[1] = 10 ** rng.uniform(-3, 0, n)
    P[2:] = rng.normal(0, 1.5, (dims, n))
    kind = np.full(n, -1)
    Pc = P.copy()
    Pc[1, 4::25] = -Pc[1, 4::25]  # negative internal energy, through PtoU
    U = np.stack([O.prim2con(dims, g, Pc[:, i]) for i in range(n)], axis=1)
    kind[4::25] = 4
    U[0, 0::25] = np.nan  # NaN density
    kind[0::25] = 0
    E = -U[1]
    U[2, 1::25] = 1.5 * E[1::25]  # |S| >= E
    kind[1::25] = 1
    U[1, 2::25] = np.abs(U[1, 2::25])  # negative energy (E < 0)
    kind[2::25] = 2
    U[0, 3::25] = -U[0, 3::25]  # negative density
    kind[3::25] = 3
    return U, P, kind


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_point_con2prim_on_corrupted_states_matches_oracle(oracle, dims):
    import torch

    from verona_b200 import _lib as L

    g = 4.0 / 3.0
    n = 1000
    U, guess, kind = _corrupt(dims, n, 40 + dims, g)
    out = {}
    for n_iter in (50, 4):  # a tight iteration cap too: more cells exhaust every stage
        dU = torch.from_numpy(np.ascontiguousarray(U)).cuda()
        dP = torch.from_numpy(np.ascontiguousarray(guess)).cuda()
        dr = torch.zeros(n, dtype=torch.int32, device="cuda")
        L.check(L.lib().vb_point_con2prim(dims, g, n_iter, 1e-12, C.c_void_p(dU.data_ptr()),
                                          C.c_void_p(dP.data_ptr()), C.c_void_p(dr.data_ptr()), n, None))
        got, ret = dP.cpu().numpy(), dr.cpu().numpy()
        codes = []
        for i in range(n):
            ref, r = oracle.con2prim(dims, g, n_iter, 1e-12, U[:, i], guess[:, i])
            same = (got[:, i] == ref) | (np.isnan(got[:, i]) & np.isnan(ref))
            assert same.all() and ret[i] == r, (n_iter, i, kind[i], got[:, i], ref, ret[i], r)
            codes.append(r)
        codes = np.array(codes)
        out[n_iter] = (codes, np.isnan(got).any(axis=0))
    bad = kind >= 0
    nan50 = out[50][1]
    print(dims, "NaN results among corrupted / healthy:", int(nan50[bad].sum()), int(nan50[~bad].sum()),
          "codes -1 at n_iter 4:", int((out[4][0] == -1).sum()))
    assert nan50[kind == 0].all()  # a NaN input never comes back finite
    assert not nan50[~bad].any()  # healthy states converge
    if dims == 3:
        assert (out[4][0] == -1).sum() > 0  # the cascade's failure exit is reached and matched


@pytest.mark.parametrize("dims", [1, 2, 3])
@pytest.mark.parametrize("n_iter", [50, 4])
def test_grid_con2prim_failure_count_on_corrupted_states(oracle, dims, n_iter):
    """vb_grid_con2prim on an interior with corrupted cells: the primitives
    equal the oracle's kernel bit for bit (NaN included), and the failure
    count is the number of cells where the oracle's solver returns a negative
    code (the 3D cascade's failure exit, the 2D Newton's singular Jacobian;
    the 1D Newton has no failure exit, and a NaN it produces is left to the
    caller's NaN check, as in the reference)."""
    import torch

    from oracle import oracle as O

    from verona_b200 import _lib as L

    g = 4.0 / 3.0
    n = {1: (200,), 2: (20, 10), 3: (10, 8, 5)}[dims]
    cells = int(np.prod(n))
    Ui, Pi, _ = _corrupt(dims, cells, 60 + dims, g)
    nv = 2 + dims
    shp = (nv,) + tuple(x + 6 for x in n)
    U = np.zeros(shp, order="F")
    P = np.zeros(shp, order="F")
    U[0], P[0], P[1] = 1.0, 1.0, 1e-2
    U[1] = -1.0
    sl = (slice(None),) + (slice(3, -3),) * dims
    U[sl] = Ui.reshape((nv,) + n, order="F")
    P[sl] = Pi.reshape((nv,) + n, order="F")

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a.transpose(tuple(range(a.ndim - 1, -1, -1))))).cuda()

    lib = L.lib()
    f = lib.vb_grid_con2prim
    f.argtypes = [C.c_int] * 4 + [C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    nn = tuple(n) + (1,) * (3 - dims)
    Pd = dev(P)
    fails = torch.zeros(1, dtype=torch.int64, device="cuda")
    assert f(dims, *nn, C.c_void_p(dev(U).data_ptr()), g, n_iter, 1e-12, C.c_void_p(Pd.data_ptr()),
             C.c_void_p(fails.data_ptr()), None) == 0
    a = Pd.cpu().numpy()
    got = np.asfortranarray(a.transpose(tuple(range(a.ndim - 1, -1, -1))))
    ref = O.k_utop(U, P, g, n_iter, 1e-12)
    assert np.array_equal(got, ref, equal_nan=True)
    codes = np.array([oracle.con2prim(dims, g, n_iter, 1e-12, Ui[:, i], Pi[:, i])[1] for i in range(cells)])
    expect = int(np.sum(codes < 0))
    print(dims, n_iter, "failures", int(fails.item()), "oracle codes < 0", expect, "NaN cells",
          int(np.isnan(ref[sl]).any(axis=0).sum()))
    assert int(fails.item()) == expect
    assert max(per_field_rel(np.nan_to_num(got), np.nan_to_num(ref))) == 0.0
