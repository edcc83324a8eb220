"""GPU tests of the batch of independent problems (vb_batch_*): every problem
of a batch against the oracle's single-grid time loop (FP64, bit-level), the
FP32-bulk batch against the single-grid FP32 solver, tile variants, CUDA-graph
replays, checkpoint/rollback and the autotuner."""
import numpy as np
import pytest

from helpers import per_field_rel

pytestmark = pytest.mark.gpu

G = 5.0 / 3.0
OPTS = dict(riemann="hllc", n_iter=50, tol=1e-12, floor=1e-8)


def _problems(seed=3):
    """Small mixed batch: pencil counts from 1 to 6 per 1D problem, 2D problems
    of 1 to 12 tiles (square and rectangular), every reconstruction."""
    from verona_b200.batch import _state, riemann_problems

    specs, prims = riemann_problems(seed, n1d=5, n2d=3, n1d_range=(5, 700), n2d_range=(9, 60), gamma=G)
    rng = np.random.default_rng(seed + 1)
    nx, ny = 45, 23
    dx, dy = 1.0 / nx, 1.0 / ny
    P = np.zeros((4, nx + 6, ny + 6), order="F")
    X, Y = np.meshgrid((np.arange(nx + 6) - 2.5) * dx, (np.arange(ny + 6) - 2.5) * dy, indexing="ij")
    for k, m in enumerate(((X >= 0.4) & (Y >= 0.6), (X < 0.4) & (Y >= 0.6), (X < 0.4) & (Y < 0.6),
                           (X >= 0.4) & (Y < 0.6))):
        s = _state(rng, G, 2)
        for v in range(4):
            P[v][m] = s[v]
    specs.append({"dims": 2, "n": (nx, ny), "recon": "ppm", "dx": dx, "dy": dy, "dt": 0.4 / (1 / dx + 1 / dy)})
    prims.append(P)
    return specs, prims


def _oracle(spec, P0, rk, nsteps):
    from oracle import oracle as O

    s = O.SolverND(spec["dims"], spec["n"][: spec["dims"]], P0, G, OPTS["floor"], OPTS["n_iter"], OPTS["tol"],
                   O.RECON[spec["recon"]], O.HLLC, rk)
    s.set_grid(spec["dx"], spec.get("dy", 1.0))
    s.step(spec["dt"], nsteps)
    return s.prims()


def _interior(a, dims):
    return a[:, 3:-3] if dims == 1 else a[:, 3:-3, 3:-3]


def _run(specs, prims, nsteps, precision="fp64", rk=3, variant=None, ctas=0, split=None):
    from verona_b200.batch import Batch

    b = Batch(specs, G, rk=rk, precision=precision, **OPTS)
    if variant is not None:
        b.set_tuning(variant, ctas)
    for i, P in enumerate(prims):
        b.load_prims(i, P)
    for n in split or [nsteps]:
        b.step(n)
    out = [b.prims(i) for i in range(len(specs))]
    cnt = b.counters()
    b.close()
    return out, cnt


@pytest.mark.parametrize("rk", [2, 3])
def test_fp64_batch_matches_oracle(rk):
    specs, prims = _problems()
    nsteps = 4
    out, cnt = _run(specs, prims, nsteps, rk=rk)
    assert cnt[4] == 0 and cnt[0] == 0, cnt
    worst = 0.0
    for spec, P0, got in zip(specs, prims, out):
        ref = _oracle(spec, P0, rk, nsteps)
        d = spec["dims"]
        rel = max(per_field_rel(_interior(got, d), _interior(ref, d)))
        worst = max(worst, rel)
        assert rel <= 1e-10, (spec, rel)
    print(f"rk{rk}: {len(specs)} problems, worst max relative difference vs oracle {worst:.3e}")


def test_fp64_variants_and_graph_replays_agree():
    specs, prims = _problems(seed=5)
    from verona_b200.batch import variants

    base, _ = _run(specs, prims, 4, variant=0)
    for v in range(1, len(variants("fp64"))):
        other, _ = _run(specs, prims, 4, variant=v, ctas=1)
        for a, b in zip(base, other):
            assert np.array_equal(a, b, equal_nan=True)
    # 4 steps as one launch == 1 + 3 == 2 + 2 launches (cached graphs, buffer parity)
    for split in ([1, 3], [2, 2]):
        other, _ = _run(specs, prims, 4, split=split)
        for a, b in zip(base, other):
            assert np.array_equal(a, b, equal_nan=True)


def test_fp32_batch_matches_single_grid_fp32_and_oracle():
    from verona_b200 import Solver

    specs, prims = _problems(seed=7)
    nsteps = 3
    out, cnt = _run(specs, prims, nsteps, precision="fp32", rk=3)
    assert cnt[4] == 0, cnt
    for spec, P0, got in zip(specs, prims, out):
        d = spec["dims"]
        dx = (spec["dx"],) if d == 1 else (spec["dx"], spec["dy"])
        s = Solver(d, spec["n"][:d], G, dx, recon=spec["recon"], rk=3, precision="fp32", **OPTS)
        s.load_prims(P0)
        s.step(spec["dt"], nsteps)
        single = s.prims()
        s.close()
        rel = max(per_field_rel(_interior(got, d), _interior(single, d)))
        assert rel <= 1e-5, (spec, rel)
        ref = _oracle(spec, P0, 3, nsteps)
        l1 = float(np.abs(_interior(got, d)[0] - _interior(ref, d)[0]).mean() / np.abs(_interior(ref, d)[0]).mean())
        assert l1 <= 1e-5, (spec, l1)


def test_checkpoint_rollback_and_time():
    from verona_b200.batch import Batch

    specs, prims = _problems(seed=9)
    b = Batch(specs, G, rk=3, precision="fp32", **OPTS)
    for i, P in enumerate(prims):
        b.load_prims(i, P)
    b.step(2)
    b.checkpoint()
    b.step(3)
    a = [b.prims(i) for i in range(len(specs))]
    t = [b.time(i) for i in range(len(specs))]
    b.rollback()
    assert all(abs(b.time(i) - 2 * s["dt"]) < 1e-15 for i, s in enumerate(specs))
    b.step(3)
    for i in range(len(specs)):
        assert np.array_equal(a[i], b.prims(i), equal_nan=True)
        assert b.time(i) == t[i]
    b.close()


def test_autotuner_picks_and_caches(tmp_path):
    from verona_b200.autotune import tune_batch
    from verona_b200.batch import Batch, riemann_problems

    specs, prims = riemann_problems(11, n1d=24, n2d=8, n1d_range=(256, 2048), n2d_range=(64, 256), gamma=G)
    b = Batch(specs, G, rk=3, precision="fp32", **OPTS)
    for i, P in enumerate(prims):
        b.load_prims(i, P)
    before = [b.prims(i) for i in (0, len(specs) - 1)]
    path = str(tmp_path / "tune.json")
    r = tune_batch(b, steps=1, ctas_candidates=(0, 1), path=path)
    print("autotuner:", {k: r[k] for k in ("variant", "ctas_per_sm", "shape", "ms_per_step")})
    assert not r["cached"] and len(r["candidates"]) >= 2
    assert b.tuning["variant"] == r["variant"]
    # tuning left the state as it was
    after = [b.prims(i) for i in (0, len(specs) - 1)]
    for x, y in zip(before, after):
        assert np.array_equal(x, y, equal_nan=True)
    r2 = tune_batch(b, path=path)
    assert r2["cached"] and r2["variant"] == r["variant"]
    b.close()


def _jet_problems():
    """Jets and tubes with every boundary kind, as (spec, P0, boundaries):
    a 2D jet through a NOZZLE on x-lo; a 2D jet held in FIXED x-lo ghosts
    whose u^x decays from mid-run on (the examples' TurnOff); a 2D jet through
    a NOZZLE on y-lo; a 1D tube fed through FIXED x-lo ghosts with a decay,
    its x-hi a NOZZLE (a fixed state in 1D); and a 2D quadrant problem with
    outflow on every face."""
    from helpers import jet_ic, nozzle_params

    from verona_b200.batch import _state

    g = 4.0 / 3.0
    out = []
    n = (48, 40, 1)
    dx = 1.0 / 48
    dt = 0.4 / (1 / dx + 1 / dx)
    P = jet_ic(2, n, gamma=g, noise=0.03, seed=31)
    spec = {"dims": 2, "n": n[:2], "recon": "wenoz", "dx": dx, "dy": dx, "dt": dt}
    out.append((spec, P, [(0, 2, nozzle_params(2, n, 4.0, gamma=g))]))
    P = jet_ic(2, n, gamma=g, noise=0.03, seed=32)
    yy = np.arange(n[1] + 6) - 3 + 0.5 - n[1] / 2
    for i in range(3):
        m = np.abs(yy) < 4.0
        P[0, i, m], P[1, i, m], P[2, i, m] = 0.01, 3e-3, np.sqrt(99.0)
    spec = dict(spec, recon="ppm")
    out.append((spec, P, [(0, 1, (2.0, 2.5 * dt, 1e9, 1 - dt / 0.05))]))
    n2 = (36, 52, 1)
    P = jet_ic(2, n2, gamma=g, noise=0.03, seed=33)
    spec = {"dims": 2, "n": n2[:2], "recon": "minmod", "dx": 1 / 36, "dy": 1 / 52, "dt": 0.4 / (36 + 52)}
    out.append((spec, P, [(2, 2, [3.5, 18.0, 0.0, 0.05, 3e-3, 0.0, 2.0])]))
    N = 300
    P = jet_ic(1, (N, 1, 1), gamma=g, noise=0.03, seed=34)
    P[2, :3] = 1.5
    spec = {"dims": 1, "n": (N,), "recon": "wenoz", "dx": 1 / N, "dy": 1.0, "dt": 0.4 / N}
    out.append((spec, P, [(0, 1, (2.0, 3.5 * spec["dt"], 1e9, 0.9)), (1, 2, [1.0, 0, 0, 2.0, 0.01, -0.5])]))
    rng = np.random.default_rng(35)
    S = 40
    P = np.zeros((4, S + 6, S + 6), order="F")
    x = (np.arange(S + 6) - 2.5) / S
    X, Y = np.meshgrid(x, x, indexing="ij")
    for m in ((X >= 0.5) & (Y >= 0.5), (X < 0.5) & (Y >= 0.5), (X < 0.5) & (Y < 0.5), (X >= 0.5) & (Y < 0.5)):
        s = _state(rng, g, 2)
        for v in range(4):
            P[v][m] = s[v]
    out.append(({"dims": 2, "n": (S, S), "recon": "wenoz", "dx": 1 / S, "dy": 1 / S, "dt": 0.4 / (2 * S)}, P, []))
    return g, out


@pytest.mark.parametrize("rk", [2, 3])
def test_fp64_batch_of_jets_matches_oracle_bitwise(rk):
    """Jets in the batch (many Riemann and jet problems in one launch): per-problem NOZZLE / FIXED-with-decay / OUTFLOW faces, each
    problem bit-identical to the oracle's single-grid run with the same
    boundaries, over 9 steps split 4 + 5 (two launches, so the device time that
    switches the decays on carries across launches), and the host times
    equal to the single grid's t."""
    from oracle import oracle as O

    from verona_b200.batch import Batch

    g, probs = _jet_problems()
    b = Batch([p[0] for p in probs], g, rk=rk, precision="fp64", **OPTS)
    for i, (spec, P0, bcs) in enumerate(probs):
        b.load_prims(i, P0)
        for face, kind, par in bcs:
            b.set_boundary(i, face, kind, par)
    b.step(4)
    b.step(5)
    assert b.check() == 0
    cnt = b.counters()
    assert cnt[0] == 0, cnt
    for i, (spec, P0, bcs) in enumerate(probs):
        d = spec["dims"]
        o = O.SolverND(d, spec["n"][:d], P0, g, OPTS["floor"], OPTS["n_iter"], OPTS["tol"], O.RECON[spec["recon"]],
                       O.HLLC, rk)
        o.set_grid(spec["dx"], spec.get("dy", 1.0))
        for face, kind, par in bcs:
            o.set_boundary(face, kind, par if kind != 1 or len(par) else (-1.0, 0.0, 0.0, 1.0))
        o.step(spec["dt"], 9)
        got, ref = _interior(b.prims(i), d), _interior(o.prims(), d)
        assert np.array_equal(got, ref), (i, spec, max(per_field_rel(got, ref)))
        assert b.time(i) == o.t, (i, b.time(i), o.t)
    b.close()


def test_fp32_batch_of_jets_close_to_single_grid():
    """The same jets in the FP32-bulk batch against the single-grid FP32-bulk
    solver with the same boundaries: within 1e-5 of each field's maximum."""
    from verona_b200 import Solver
    from verona_b200.batch import Batch

    g, probs = _jet_problems()
    b = Batch([p[0] for p in probs], g, rk=3, precision="fp32", **OPTS)
    for i, (spec, P0, bcs) in enumerate(probs):
        b.load_prims(i, P0)
        for face, kind, par in bcs:
            b.set_boundary(i, face, kind, par)
    b.step(9)
    assert b.check() == 0
    for i, (spec, P0, bcs) in enumerate(probs):
        d = spec["dims"]
        dx = (spec["dx"],) if d == 1 else (spec["dx"], spec["dy"])
        s = Solver(d, spec["n"][:d], g, dx, recon=spec["recon"], rk=3, precision="fp32", **OPTS)
        for face, kind, par in bcs:
            s.set_boundary(face, kind, par)
        s.load_prims(P0)
        s.step(spec["dt"], 9)
        rel = max(per_field_rel(_interior(b.prims(i), d), _interior(s.prims(), d)))
        s.close()
        assert rel <= 1e-5, (i, spec, rel)
    b.close()
