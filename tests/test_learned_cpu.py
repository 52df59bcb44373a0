"""The neural-operator oracle (numpy FP64) pinned by central finite differences, and the
parameter layout shared with the GPU kernels (no GPU needed)."""
import numpy as np

from oracle import neural_operator as NO
from slepc_b200 import learned as L

DIMS = (8, 4, 3, 2, 6, 3)  # N, width, modes, layers, hidden, nout


def _problem(seed, B=2):
    rng = np.random.default_rng(seed)
    N, W, M, Ly, H, K = DIMS
    theta = L.init_params(*DIMS, seed=seed).astype(np.float64)
    theta += 0.05 * rng.standard_normal(theta.size)  # nonzero biases too
    F = rng.standard_normal((B, 3, N * N))
    T = rng.standard_normal((B, K, N * N))
    T /= np.linalg.norm(T, axis=2, keepdims=True)
    return theta, F, T


def test_oracle_gradient_matches_finite_differences():
    theta, F, T = _problem(0)
    _, g = NO.loss_grad(theta, F, T, DIMS)
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.choice(theta.size, 60, replace=False), [0, theta.size - 1]])
    h = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (NO.loss(NO.forward(tp, F, DIMS)[0], T)[0] - NO.loss(NO.forward(tm, F, DIMS)[0], T)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd), (i, fd, g[i])


def test_oracle_directional_derivative():
    theta, F, T = _problem(2, B=3)
    _, g = NO.loss_grad(theta, F, T, DIMS)
    d = np.random.default_rng(3).standard_normal(theta.size)
    h = 1e-6
    fd = (NO.loss(NO.forward(theta + h * d, F, DIMS)[0], T)[0] - NO.loss(NO.forward(theta - h * d, F, DIMS)[0], T)[0]) / (2 * h)
    assert abs(fd - g @ d) <= 1e-6 * max(1.0, abs(fd))


def test_parameter_layout_and_features():
    assert L.init_params(*DIMS).size == sum(int(np.prod(s)) for _, s in NO.sizes(*DIMS))
    kappa = np.exp(np.arange(16.0).reshape(4, 4) / 10)
    f = L.features(kappa)
    assert f.shape == (3, 16) and f.dtype == np.float32
    np.testing.assert_allclose(f[0], np.log(kappa).ravel(), rtol=1e-6)
    np.testing.assert_allclose(f[1].reshape(4, 4)[0], (np.arange(4) + 0.5) / 4)   # x varies along a row
    np.testing.assert_allclose(f[2].reshape(4, 4)[:, 0], (np.arange(4) + 0.5) / 4)  # y varies down a column
