"""The learned-delta network's CPU restatement (oracle/mlp_ref.py) against
central finite differences: the oracle the CUDA kernels are checked
against is itself checked here (CPU only)."""
import numpy as np

from oracle import mlp_ref as R


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    X = rng.standard_normal((40, R.IN))
    T = rng.standard_normal(40)
    p = R.init_params(11) + 0.05 * rng.standard_normal(R.P)
    _, g = R.loss_and_grad(p, X, T)
    h = 1e-6
    for q in rng.choice(R.P, 60, replace=False):
        e = np.zeros(R.P)
        e[q] = h
        fd = (R.loss_and_grad(p + e, X, T)[0] - R.loss_and_grad(p - e, X, T)[0]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-7 * max(1.0, abs(g[q]))


def test_oracle_adam_reduces_loss():
    rng = np.random.default_rng(5)
    X = rng.standard_normal((256, R.IN))
    T = np.sin(X[:, 0]) + 0.5 * X[:, 1]
    p0 = R.init_params(7)
    l0 = R.loss_and_grad(p0, X, T)[0]
    p1 = R.adam(p0, X, T, epochs=200, lr=1e-2)
    assert R.loss_and_grad(p1, X, T)[0] < 0.2 * l0
