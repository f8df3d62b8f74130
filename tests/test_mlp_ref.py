"""The CPU reference of the warm-start MLP, pinned by finite differences.

The exact (float64) gradient of oracle/mlp_ref.py is checked against central
differences of its own loss, and the BF16 rounding helper against values
whose BF16 neighbours are known.
"""
import numpy as np

import mlp_ref


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -2.5, 0.0, 1e-3], dtype=np.float32)
    r = mlp_ref.bf16(x)
    # ties to even: 1 + 2^-8 -> 1, 1 + 3*2^-8 -> 1 + 2^-6
    assert list(r[:4]) == [1.0, 1.0, 1.0 + 2 ** -7, 1.0 + 2 ** -6]
    assert r[4] == -2.5 and r[5] == 0.0
    assert abs(r[6] - 1e-3) <= 1e-3 * 2 ** -8


def test_exact_gradient_matches_finite_differences():
    n_in, width, depth, n_out = 3, 8, 2, 5
    rng = np.random.default_rng(0)
    sh = mlp_ref.shapes(n_in, width, depth, n_out)
    p = np.concatenate([np.concatenate([rng.normal(0, 0.5, (o, i)).ravel() * (np.arange(i) < li)[None, :].repeat(o, 0).ravel(),
                                        rng.normal(0, 0.1, o)]) for (o, i, li) in sh])
    x = rng.uniform(-1, 1, (6, n_in))
    t = rng.normal(0, 1, (6, n_out))
    loss, g = mlp_ref.loss_and_grad(p, x, t, n_in, width, depth, n_out, bf16_points=False)
    live = np.concatenate([np.concatenate([(np.arange(i) < li)[None, :].repeat(o, 0).ravel(), np.ones(o, bool)])
                           for (o, i, li) in sh])
    idx = rng.choice(np.flatnonzero(live), 60, replace=False)
    h = 1e-6
    for k in idx:
        q = p.copy()
        q[k] += h
        lp, _ = mlp_ref.loss_and_grad(q, x, t, n_in, width, depth, n_out, bf16_points=False)
        q[k] -= 2 * h
        lm, _ = mlp_ref.loss_and_grad(q, x, t, n_in, width, depth, n_out, bf16_points=False)
        assert abs((lp - lm) / (2 * h) - g[k]) <= 1e-7 + 1e-6 * abs(g[k])
    assert np.all(g[~live] == 0.0)
