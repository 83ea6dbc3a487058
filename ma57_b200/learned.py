"""Learned first-attempt delta for Mode::StaticRegularized.

The reference's StaticRegularized mode (solver.hpp:328-417) factors with one
static-pivot delta, checks the inertia against the expected sign pattern and,
on failure, multiplies delta by a growth factor and factors again. Along an
interior-point sequence the delta that finally passes drifts with the
barrier parameter, and every failed attempt costs a full factorization.

`DeltaModel` predicts the first-attempt delta of every front from
statistics of that front of the matrix being factorized (diagonal
magnitudes, expected-sign counts, column norms, sizes), with a small
multilayer perceptron trained and evaluated on the GPU by the library's own
kernels (symla_mlp_*). The prediction is in decades above a base delta, the
plain escalation's first attempt (a fixed fraction of max|K|), so that it
is the number of escalation steps to skip: a quantity that stays in the
training range while the matrix scale drifts along the sequence. Training
targets are log10(accepted / base) of the deltas the escalation loop itself
accepted on earlier matrices of the sequence. The prediction goes in as
`symla_regularize_opts.front_delta`; when it fails the inertia check the
plain escalation takes over, one growth step above the smallest delta the
failed attempt used, so correctness never depends on the model.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import scipy.sparse as sp

from . import _lib as L

NFEAT = L.MLP_INPUTS
_TINY = 1e-300


def front_features(sym, A_lower, expected_sign=None) -> np.ndarray:
    """Per-front statistics (one row per supernode of `sym`, a SymbolicFactor):
    log10 max / min / mean |a_jj| over the front's pivot columns, the fraction
    of those columns whose expected sign is negative, log10 of the largest
    column 2-norm, log10 m, and two statistics of the whole matrix (log10 of
    the median |a_jj| and of max |a_ij|), which carry the scale the sequence
    is at. A_lower: the stored lower triangle."""
    A = sp.csc_matrix(A_lower)
    full = (A + sp.tril(A, -1).T).tocsc()
    perm = np.asarray(sym.perm)
    n = A.shape[0]
    d = np.abs(full.diagonal())[perm]
    colnorm = np.sqrt(np.asarray(full.multiply(full).sum(axis=0)).ravel())[perm]
    sign = np.zeros(n) if expected_sign is None else np.asarray(expected_sign, dtype=np.float64)[perm]
    amax = max(float(np.abs(A.data).max()) if A.nnz else 0.0, _TINY)
    dmed = math.log10(float(np.median(d)) + _TINY)
    rows = []
    for s in sym.supernodes:
        c0, c1 = s.firstCol, s.firstCol + s.ncols
        dc = d[c0:c1]
        rows.append([
            math.log10(dc.max() + _TINY), math.log10(dc.min() + _TINY), math.log10(dc.mean() + _TINY),
            float(np.mean(sign[c0:c1] < 0)), math.log10(colnorm[c0:c1].max() + _TINY),
            math.log10(len(s.rowPattern)), dmed, math.log10(amax),
        ])
    return np.asarray(rows, dtype=np.float64)


def init_params(seed: int) -> np.ndarray:
    """Deterministic uniform (Glorot) initialisation, biases zero."""
    rng = np.random.default_rng(seed)
    h, i = L.MLP_HIDDEN, L.MLP_INPUTS
    W1 = rng.uniform(-1, 1, (h, i)) * math.sqrt(6.0 / (i + h))
    W2 = rng.uniform(-1, 1, (h, h)) * math.sqrt(6.0 / (2 * h))
    w3 = rng.uniform(-1, 1, h) * math.sqrt(6.0 / (h + 1))
    return np.concatenate([W1.ravel(), np.zeros(h), W2.ravel(), np.zeros(h), w3, [0.0]])


class Network:
    """The device-resident network (symla_mlp_*): predict, gradient, train."""

    def __init__(self, params: np.ndarray, device: int = 0):
        self._lib = L.load()
        p = np.ascontiguousarray(params, dtype=np.float64)
        if p.size != L.MLP_PARAMS:
            raise ValueError(f"expected {L.MLP_PARAMS} parameters, got {p.size}")
        h = C.c_void_p()
        rc = self._lib.symla_mlp_create(device, L.ptr_d(p), C.byref(h))
        if rc != L.SYMLA_OK:
            raise RuntimeError(L.last_error())
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self._lib.symla_mlp_destroy(self.h)
            self.h = None

    def params(self) -> np.ndarray:
        out = np.zeros(L.MLP_PARAMS)
        self._check(self._lib.symla_mlp_get_params(self.h, L.ptr_d(out)))
        return out

    def predict(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float64)
        y = np.zeros(X.shape[0])
        self._check(self._lib.symla_mlp_predict(self.h, L.ptr_d(X), X.shape[0], L.ptr_d(y)))
        return y

    def gradient(self, X: np.ndarray, T: np.ndarray):
        X = np.ascontiguousarray(X, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        g = np.zeros(L.MLP_PARAMS)
        loss = C.c_double()
        self._check(self._lib.symla_mlp_gradient(self.h, L.ptr_d(X), L.ptr_d(T), X.shape[0], L.ptr_d(g),
                                                 C.byref(loss)))
        return loss.value, g

    def train(self, X: np.ndarray, T: np.ndarray, epochs: int, lr: float, minibatch: int = 0) -> float:
        X = np.ascontiguousarray(X, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        loss = C.c_double()
        self._check(self._lib.symla_mlp_train(self.h, L.ptr_d(X), L.ptr_d(T), X.shape[0], epochs, minibatch, lr,
                                              C.byref(loss)))
        return loss.value

    @staticmethod
    def _check(rc):
        if rc != L.SYMLA_OK:
            raise RuntimeError(L.last_error())


class DeltaModel:
    """Standardised front features -> first-attempt delta, in decades above
    the base delta.

    A front's delta is its prediction, but never below the median prediction
    over the matrix's fronts, plus a margin in decades: an under-predicted
    delta costs a whole failed factorization, an over-predicted one only a
    larger perturbation for refinement to remove. `fit` chooses the margin
    as the smallest that would have covered `coverage` of the training
    matrices (their median prediction plus margin at or above the delta
    escalation accepted), unless a margin is given."""

    def __init__(self, seed: int = 0, device: int = 0, margin: float | None = None, coverage: float = 0.9):
        self.net = Network(init_params(seed), device)
        self.mean = np.zeros(NFEAT)
        self.std = np.ones(NFEAT)
        self.margin = margin
        self.coverage = coverage

    def fit(self, X: np.ndarray, T: np.ndarray, groups=None, epochs: int = 400, lr: float = 3e-3,
            minibatch: int = 4096) -> float:
        """X: front features, T: log10(accepted delta / base delta) of each
        front's matrix, groups: the matrix index of each row (for the
        margin)."""
        self.mean = X.mean(axis=0)
        self.std = X.std(axis=0)
        self.std[self.std < 1e-12] = 1.0
        loss = self.net.train((X - self.mean) / self.std, T, epochs, lr, minibatch)
        if self.margin is None:
            if groups is None:
                self.margin = 0.5
            else:
                pred = self.predict_log10(X)
                groups = np.asarray(groups)
                short = [float(T[groups == g][0] - np.median(pred[groups == g])) for g in np.unique(groups)]
                self.margin = max(0.0, float(np.quantile(short, self.coverage)))
        return loss

    def update(self, X: np.ndarray, T: np.ndarray, retries: int | None = None, window: int = 20, epochs: int = 20,
               lr: float = 1e-3, minibatch: int = 4096) -> float | None:
        """Online step along a sequence: add one matrix's fronts with the
        delta escalation accepted for it to the last `window` matrices and,
        unless the first attempt passed (`retries` == 0: the model was right
        and nothing new is learned), fine-tune on them (same
        standardisation) and refit the margin. Returns the training loss,
        or None when no training ran."""
        self._buf = getattr(self, "_buf", [])
        self._buf.append((np.asarray(X, dtype=np.float64), np.asarray(T, dtype=np.float64)))
        self._buf = self._buf[-window:]
        if retries == 0:
            return None
        Xb = np.vstack([x for x, _ in self._buf])
        Tb = np.concatenate([t for _, t in self._buf])
        loss = self.net.train((Xb - self.mean) / self.std, Tb, epochs, lr, minibatch)
        pred = self.predict_log10(Xb)
        short, off = [], 0
        for x, t in self._buf:
            short.append(float(t[0] - np.median(pred[off:off + len(t)])))
            off += len(t)
        self.margin = max(0.0, float(np.quantile(short, self.coverage)))
        return loss

    def predict_log10(self, X: np.ndarray) -> np.ndarray:
        return self.net.predict((X - self.mean) / self.std)

    def front_deltas(self, X: np.ndarray, base: float) -> np.ndarray:
        """Per-front first-attempt deltas for a matrix whose plain first
        attempt is `base`: never below it (a smaller delta than plain
        escalation's first one gains nothing)."""
        p = self.predict_log10(X)
        return base * 10.0 ** np.maximum(0.0, np.maximum(p, np.median(p)) + (self.margin or 0.0))
