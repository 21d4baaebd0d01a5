"""The numpy MLP oracle itself: analytic gradient against central differences."""
import numpy as np


def test_oracle_gradient_matches_finite_differences():
    from oracle import mlp
    rng = np.random.default_rng(0)
    p = rng.standard_normal(mlp.N_PARAMS) * 0.2
    x = rng.standard_normal((7, mlp.F))
    t = rng.standard_normal((7, mlp.O))
    mask = (rng.random((7, mlp.O)) > 0.3).astype(float)
    loss, g = mlp.loss_and_grad(p, x, t, mask)
    idx = rng.choice(mlp.N_PARAMS, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (mlp.loss_and_grad(p + e, x, t, mask)[0] - mlp.loss_and_grad(p - e, x, t, mask)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i])


def test_bf16_rounding_is_nearest_even():
    from oracle import mlp
    x = np.array([1.0, 1.00390625, 1.0078125, -3.14159, 1e-3], np.float32)
    r = mlp.bf16_round(x)
    assert r[0] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)
