"""CPU pin of the MLP reference (oracle/mlp_ref.py): its backward equals
central finite differences of its forward."""
import numpy as np


def test_reference_gradient_matches_finite_differences():
    from oracle import mlp_ref

    rng = np.random.default_rng(0)
    p = rng.normal(size=8705) * 0.1
    x = rng.normal(size=(64, 4))
    t = rng.normal(size=64)
    _, g = mlp_ref.loss_and_grad(p, x, t)
    e = 1e-6
    for i in list(range(0, 8705, 211)) + [8704]:
        q = p.copy()
        q[i] += e
        lp, _ = mlp_ref.loss_and_grad(q, x, t)
        q[i] -= 2 * e
        lm, _ = mlp_ref.loss_and_grad(q, x, t)
        fd = (lp - lm) / (2 * e)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    from oracle import mlp_ref

    x = np.array([1.0, 1.0 + 2.0**-8, 1.0 + 3 * 2.0**-9, -2.5, 3.14159])
    r = mlp_ref.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2.0**-7 and r[3] == -2.5
    assert abs(r[4] - 3.14159) < 2.0**-7 * 3.14159
