"""ORACLE -- test infrastructure only.

CPU restatement (numpy, FP64) of the learned-delta network of
ma57_b200/csrc/gpu/mlp.cu: forward pass, the gradient of the mean squared
error, and Adam. Used by tests to check the CUDA kernels' gradients and
training steps; nothing in the product imports it.

Parameter vector layout: W1 (H x IN, row-major), b1 (H), W2 (H x H), b2 (H),
w3 (H), b3.
"""
import numpy as np

IN, H = 8, 32
P = H * IN + H + H * H + H + H + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + H * IN].reshape(H, IN); o += H * IN
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def init_params(seed):
    """Xavier-style uniform initialisation from a seed (deterministic)."""
    rng = np.random.default_rng(seed)
    W1 = rng.uniform(-1, 1, (H, IN)) * np.sqrt(6.0 / (IN + H))
    W2 = rng.uniform(-1, 1, (H, H)) * np.sqrt(6.0 / (2 * H))
    w3 = rng.uniform(-1, 1, H) * np.sqrt(6.0 / (H + 1))
    return np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(H), w3, [0.0]])


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    H1 = np.tanh(X @ W1.T + b1)
    H2 = np.tanh(H1 @ W2.T + b2)
    return H2 @ w3 + b3, H1, H2


def loss_and_grad(p, X, T):
    """Mean squared error (1/B) sum (y - t)^2 and its gradient."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    B = X.shape[0]
    y, H1, H2 = forward(p, X)
    e = y - T
    dy = 2.0 * e / B
    D2 = np.outer(dy, w3) * (1.0 - H2 ** 2)
    D1 = (D2 @ W2) * (1.0 - H1 ** 2)
    g = np.concatenate([(D1.T @ X).ravel(), D1.sum(0), (D2.T @ H1).ravel(), D2.sum(0), H2.T @ dy, [dy.sum()]])
    return float(np.mean(e ** 2)), g


def adam(p, X, T, epochs, lr, minibatch=0, b1=0.9, b2=0.999, eps=1e-8):
    p = np.array(p, dtype=np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    B = X.shape[0]
    mb = B if minibatch <= 0 or minibatch > B else minibatch
    t = 0
    for _ in range(epochs):
        for off in range(0, B, mb):
            _, g = loss_and_grad(p, X[off:off + mb], T[off:off + mb])
            t += 1
            m = b1 * m + (1 - b1) * g
            v = b2 * v + (1 - b2) * g * g
            p -= lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return p
