"""The CPU oracle of the controller network: its analytic gradient against
central finite differences (float64), so it can check the GPU kernels."""
import numpy as np

from oracle import mlp


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(mlp.N_PARAMS) * 0.3
    X = rng.standard_normal((37, mlp.N_IN))
    y = rng.uniform(0.2, 1.0, 37)
    loss, g = mlp.loss_and_grad(p, X, y, over_weight=3.0)
    idx = rng.choice(mlp.N_PARAMS, 60, replace=False)
    idx = np.concatenate([idx, [mlp.OFF_B3, mlp.OFF_W3, mlp.OFF_B1, mlp.OFF_B2]])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp.loss_and_grad(pp, X, y, 3.0)[0] - mlp.loss_and_grad(pm, X, y, 3.0)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g).max()), (i, fd, g[i])


def test_bf16_round():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-30], np.float32)
    r = mlp.bf16_round(a)
    # bfloat16 keeps 8 significant bits
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125)
    assert abs(r[3] - a[3]) <= 2 ** -7 * abs(a[3])


def test_theta_range():
    rng = np.random.default_rng(1)
    p = rng.standard_normal(mlp.N_PARAMS) * 3
    th, _ = mlp.forward(p, rng.standard_normal((100, mlp.N_IN)) * 10)
    assert th.min() >= 0.2 and th.max() <= 1.0
