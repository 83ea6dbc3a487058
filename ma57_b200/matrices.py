"""Seeded, portable generators for the benchmark configurations and the
reference's test fixtures.

Random numbers come from a SplitMix64 counter stream (Steele, Lea & Flood,
"Fast splittable pseudorandom number generators", OOPSLA 2014): output i of
stream `seed` is mix64(seed + (i + 1) * 0x9E3779B97F4A7C15), uniforms take the
top 53 bits, normals use the Box-Muller transform. The stream is defined
independently of platform and library version, and is vectorised over i.
Configuration seeds are 20261203 + configuration index.

Stencil matrices:
  L7(k)   3D 7-point Laplacian on a k x k x k grid, Dirichlet (diag 6, -1)
  L27(k)  3D 27-point stencil (centre 26, all 26 neighbours -1)
  L5(a,b) 2D 5-point Laplacian on an a x b grid (diag 4, -1)
KKT systems K = [[-E, A^T], [A, F]] are stored lower-triangle only, like the
reference's buildKKT (test/correctness/kkt_static_pivoting_test.cpp:98-118).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
SEED_BASE = 20261203


def _mix64(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.uint64, copy=True)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


class Stream:
    """SplitMix64 counter stream with a cursor."""

    def __init__(self, seed: int):
        self.seed = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
        self.pos = 0

    def raw(self, count: int) -> np.ndarray:
        i = np.arange(self.pos + 1, self.pos + count + 1, dtype=np.uint64)
        self.pos += count
        with np.errstate(over="ignore"):
            return _mix64(self.seed + i * GOLDEN)

    def uniform(self, count: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
        u = (self.raw(count) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
        return lo + (hi - lo) * u

    def integers(self, count: int, n: int) -> np.ndarray:
        """Uniform integers in [0, n) (multiply-shift on the top 32 bits)."""
        top = (self.raw(count) >> np.uint64(32)).astype(np.uint64)
        return ((top * np.uint64(n)) >> np.uint64(32)).astype(np.int64)

    def normal(self, count: int) -> np.ndarray:
        m = (count + 1) // 2
        u1 = self.uniform(m)
        u2 = self.uniform(m)
        u1 = np.where(u1 <= 0.0, 1.0 / 9007199254740992.0, u1)
        r = np.sqrt(-2.0 * np.log(u1))
        z = np.empty(2 * m)
        z[0::2] = r * np.cos(2.0 * math.pi * u2)
        z[1::2] = r * np.sin(2.0 * math.pi * u2)
        return z[:count]


# --------------------------------------------------------------------------
# Stencils


def laplacian7(k: int) -> sp.csc_matrix:
    e = np.ones(k)
    T = sp.diags([-e[:-1], 2 * e, -e[:-1]], [-1, 0, 1])
    I = sp.identity(k)
    A = sp.kron(sp.kron(T, I), I) + sp.kron(sp.kron(I, T), I) + sp.kron(sp.kron(I, I), T)
    return sp.csc_matrix(A)


def laplacian27(k: int) -> sp.csc_matrix:
    """Centre 26, each of the 26 neighbours in the 3x3x3 cube -1, Dirichlet."""
    one = sp.diags([np.ones(k - 1), np.ones(k), np.ones(k - 1)], [-1, 0, 1])  # tridiagonal of ones
    J = sp.kron(sp.kron(one, one), one)  # 27-point ones pattern (includes centre)
    A = 27.0 * sp.identity(k ** 3) - J
    A = sp.csc_matrix(A)
    A.eliminate_zeros()
    return A


def laplacian5(a: int, b: int) -> sp.csc_matrix:
    def t(k):
        e = np.ones(k)
        return sp.diags([-e[:-1], 2 * e, -e[:-1]], [-1, 0, 1])
    A = sp.kron(t(a), sp.identity(b)) + sp.kron(sp.identity(a), t(b))
    return sp.csc_matrix(A)


def lower(A) -> sp.csc_matrix:
    L = sp.tril(sp.csc_matrix(A), format="csc")
    L.sort_indices()
    return L


def sym_full(A) -> sp.csc_matrix:
    """Symmetric matrix from its lower triangle (for dense checks)."""
    Lw = sp.tril(sp.csc_matrix(A))
    return sp.csc_matrix(Lw + sp.tril(Lw, -1).T)


def kkt(E, F, A) -> sp.csc_matrix:
    """K = [[-E, A^T], [A, F]], lower triangle stored."""
    n1, n2 = E.shape[0], F.shape[0]
    K = sp.bmat([[-sp.tril(E), None], [sp.csc_matrix(A), sp.tril(F)]], format="csc")
    assert K.shape == (n1 + n2, n1 + n2)
    K.sort_indices()
    return K


# --------------------------------------------------------------------------
# Benchmark configurations


def config1(k: int = 20, shift: float = 2.0):
    """L7(k^3) - shift*I, lower triangle; b ~ N(0,1) nrhs 1."""
    A = lower(laplacian7(k) - shift * sp.identity(k ** 3))
    b = Stream(SEED_BASE + 1).normal(k ** 3)
    return A, b


def random_coupling(n2: int, n1: int, per_row: int, stream: Stream) -> sp.csc_matrix:
    cols = stream.integers(n2 * per_row, n1)
    vals = stream.normal(n2 * per_row)
    rows = np.repeat(np.arange(n2), per_row)
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n2, n1)).tocsc()  # duplicates summed
    A.sum_duplicates()
    return A


def config2(grid: int = 200, n2: int = 20000, per_row: int = 3):
    """KKT: E = L5(grid^2) + 1e-2 I, A random 3/row N(0,1), F = 1e-8 I."""
    st = Stream(SEED_BASE + 2)
    n1 = grid * grid
    E = laplacian5(grid, grid) + 1e-2 * sp.identity(n1)
    A = random_coupling(n2, n1, per_row, st)
    F = 1e-8 * sp.identity(n2)
    K = kkt(E, F, A)
    b = st.normal(n1 + n2)
    return K, b, n1, n2


def config3(k: int = 64, shift: float = 3.0, nrhs: int = 16):
    """L27(k^3) - shift*I, lower triangle; B ~ N(0,1), n x nrhs."""
    n = k ** 3
    A = lower(laplacian27(k) - shift * sp.identity(n))
    B = Stream(SEED_BASE + 3).normal(n * nrhs).reshape(nrhs, n).T.copy(order="F")
    return A, B


def config4_system(i: int, nmin: int = 200, nmax: int = 4000, stream: Stream | None = None):
    """System i of the batched config: L5 on a random rectangle, shifted."""
    st = stream or Stream(SEED_BASE + 4 + 1_000_003 * (i + 1))
    u = st.uniform(3)
    ni = math.exp(math.log(nmin) + (math.log(nmax) - math.log(nmin)) * u[0])
    r = math.exp(math.log(0.25) + (math.log(4.0) - math.log(0.25)) * u[1])
    a = max(2, int(round(math.sqrt(ni * r))))
    b = max(2, int(round(ni / a)))
    sigma = 0.5 + 3.5 * u[2]
    A = lower(laplacian5(a, b) - sigma * sp.identity(a * b))
    return A, a, b, sigma


def config4(count: int = 4096, nrhs: int = 8):
    systems = []
    for i in range(count):
        A, a, b, sigma = config4_system(i)
        st = Stream(SEED_BASE + 4 + 7_000_001 * (i + 1))
        B = st.normal(A.shape[0] * nrhs).reshape(nrhs, A.shape[0]).T.copy(order="F")
        systems.append((A, B))
    return systems


class InteriorPointSequence:
    """Config 5: K_k = [[-E_k, A^T], [A, F_k]], E_k = L7(k^3) + diag(mu_k / x^2),
    F_k = mu_k * 1e-6 I, A: (n1/2) x n1 with 3 N(0,1) entries per row;
    x log-uniform in [1e-8, 1e2] with multiplicative exp(N(0, 0.3)) drift per
    step, mu_k = 10^(-9 k / (steps - 1))."""

    def __init__(self, k: int = 20, steps: int = 500, curvature_shift: float = 0.0):
        """curvature_shift c > 0 gives the nonconvex variant E_k = L7 - c I +
        diag(mu_k / x^2): for small mu_k, E_k has negative curvature, K_k is no
        longer quasi-definite and StaticRegularized must perturb wrongly signed
        pivots (c = 0 is the configuration as specified, which is
        quasi-definite for every k)."""
        self.st = Stream(SEED_BASE + 5)
        self.shift = curvature_shift
        self.n1 = k ** 3
        self.n2 = self.n1 // 2
        self.steps = steps
        self.L = laplacian7(k)
        self.A = random_coupling(self.n2, self.n1, 3, self.st)
        u = self.st.uniform(self.n1)
        self.logx = math.log(1e-8) + (math.log(1e2) - math.log(1e-8)) * u
        self.b = self.st.normal(self.n1 + self.n2)

    def matrix(self, step: int):
        mu = 10.0 ** (-9.0 * step / max(1, self.steps - 1))
        if step > 0:
            self.logx = self.logx + 0.3 * self.st.normal(self.n1)
            self.logx = np.clip(self.logx, math.log(1e-8), math.log(1e2))
        x2 = np.exp(2.0 * self.logx)
        E = self.L + sp.diags(mu / x2 - self.shift)
        F = (mu * 1e-6) * sp.identity(self.n2)
        return kkt(E, F, self.A), mu


# --------------------------------------------------------------------------
# Fixtures in the spirit of the reference's test helpers
# (test/unit/test_helpers.hpp:38-150); values drawn from the stream above.


def random_sparse_spd(n: int, avg_nnz_per_row: int, seed: int) -> sp.csc_matrix:
    st = Stream(seed)
    rows, cols, vals = [], [], []
    rowsum = np.zeros(n)
    for i in range(n):
        ne = 1 + int(st.integers(1, max(1, avg_nnz_per_row))[0]) if avg_nnz_per_row > 0 else 0
        js = st.integers(ne, n)
        vs = st.uniform(ne, 0.1, 1.0)
        for j, v in zip(js, vs):
            if j <= i:
                continue
            rows += [i, j]
            cols += [j, i]
            vals += [v, v]
            rowsum[i] += v
            rowsum[j] += v
    for i in range(n):
        rows.append(i)
        cols.append(i)
        vals.append(rowsum[i] + 1.0 + (i % 5) * 0.1)
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsc()
    A.sum_duplicates()
    return A


def random_sparse_indefinite(n: int, avg_nnz_per_row: int, seed: int) -> sp.csc_matrix:
    A = random_sparse_spd(n, avg_nnz_per_row, seed).tolil()
    flips = Stream(seed ^ 0x9E3779B9).integers(n, 2)
    for i in range(n):
        if flips[i] == 0:
            A[i, i] = -A[i, i]
    return sp.csc_matrix(A)
