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
