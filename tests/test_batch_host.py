"""CPU tests of the batch API's host side: argument validation (before any
CUDA call), the seeded uneven workload generator and the tuning cache path."""
import ctypes as C
import math

import numpy as np
import pytest


def _create(problems, **kw):
    from verona_b200 import _lib as L
    from verona_b200.batch import BatchProblem, _sig

    lib = _sig()
    arr = (BatchProblem * len(problems))(*[BatchProblem(*p) for p in problems])
    opts = L.default_options(**kw)
    h = C.c_void_p()
    rc = lib.vb_batch_create(C.byref(h), len(problems), arr, 5.0 / 3.0, C.byref(opts))
    return rc, lib.vb_batch_last_error(None).decode()


@pytest.mark.parametrize("prob,word", [
    ((3, 10, 10, 0, 0.1, 0.1, 0.01), "dims"),
    ((1, 10, 2, 0, 0.1, 0.1, 0.01), "size"),
    ((2, 10, 0, 0, 0.1, 0.1, 0.01), "size"),
    ((1, 10, 1, 7, 0.1, 0.1, 0.01), "recon"),
    ((1, 10, 1, 0, 0.0, 0.1, 0.01), "dx"),
    ((2, 10, 10, 0, 0.1, 0.1, -1.0), "dt"),
])
def test_invalid_problems_are_rejected(prob, word):
    rc, msg = _create([(1, 16, 1, 0, 0.1, 0.1, 0.01), prob])
    assert rc == -1 and word in msg and "problem 1" in msg


def test_invalid_options_are_rejected():
    ok = [(1, 16, 1, 0, 0.1, 0.1, 0.01)]
    rc, msg = _create(ok, guess="learned")
    assert rc == -4 and "previous-state guess" in msg
    rc, msg = _create(ok, rk=4)
    assert rc == -1 and "rk" in msg


def test_riemann_problem_generator_is_seeded_and_in_range():
    from verona_b200.batch import riemann_problems

    g = 5.0 / 3.0
    s1, p1 = riemann_problems(4, n1d=12, n2d=4, n2d_range=(128, 160), gamma=g)
    s2, p2 = riemann_problems(4, n1d=12, n2d=4, n2d_range=(128, 160), gamma=g)
    assert s1 == s2 and all(np.array_equal(a, b) for a, b in zip(p1, p2))
    s3, _ = riemann_problems(5, n1d=12, n2d=4, n2d_range=(128, 160), gamma=g)
    assert s3 != s1
    for spec, P in zip(s1, p1):
        d = spec["dims"]
        n = spec["n"]
        assert P.shape == (2 + d,) + tuple(x + 6 for x in n[:d])
        if d == 1:
            assert 256 <= n[0] <= 8192 and spec["dt"] == pytest.approx(0.4 / n[0])
        else:
            assert 128 <= n[0] <= 160 and n[0] == n[1] and spec["dt"] == pytest.approx(0.4 / (2 * n[0]))
        rho, p = P[0], (g - 1) * P[1]
        lor = np.sqrt(1 + (P[2:] ** 2).sum(0))
        assert rho.min() >= 0.1 - 1e-12 and rho.max() <= 10 + 1e-9
        assert p.min() >= 1e-4 * (1 - 1e-12) and p.max() <= 20 * (1 + 1e-12)
        assert lor.max() <= 1 / math.sqrt(1 - 0.81) + 1e-12
        assert spec["recon"] in ("minmod", "ppm", "wenoz")


def test_tuning_cache_path_follows_environment(monkeypatch, tmp_path):
    from verona_b200 import autotune

    monkeypatch.setenv("VB_TUNE_CACHE", str(tmp_path / "t.json"))
    assert autotune.cache_path() == str(tmp_path / "t.json")
    monkeypatch.delenv("VB_TUNE_CACHE")
    assert autotune.cache_path().endswith("batch_tuning.json")
