"""Shared test helpers: a SymLDLT-shaped adapter over the oracle, fixtures
restated from the reference's test helpers, and the reference's error
measures."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp

from ma57_b200 import matrices as M
from ma57_b200.solver import (Analysis, Inertia, Mode, OrderingType, PivotBlock, RefinedSolve, RefinementOptions,
                              RefinementResult, SupernodeFactor, SymbolicFactorOptions, SymLDLT, as_csc)


class OracleSolver:
    """The oracle behind the same interface as ma57_b200.SymLDLT, so one test
    body exercises both. The symbolic analysis is the shared host analysis."""

    def __init__(self):
        self.mode = Mode.ThresholdPivot
        self.ordering = OrderingType.AMD
        self.settings = {}
        self.kkt = None
        self.signs = None
        self._o = None
        self._an = None

    def setMode(self, m):
        self.mode = Mode(m)

    def setOrdering(self, o):
        self.ordering = OrderingType(o)

    def setPivotThreshold(self, u):
        self.settings["pivot_threshold"] = u

    def setPrecision(self, p):
        pass

    def setKKTBlockSizes(self, n1, n2):
        self.kkt = (n1, n2)
        self.signs = None

    def setExpectedSignPattern(self, s):
        self.signs = np.asarray(s, np.int32)
        self.kkt = None

    def setInitialRegularizationDelta(self, d):
        self.settings["initial_delta"] = d

    def setMaxRegularizationRetries(self, r):
        self.settings["max_retries"] = r

    def setRegularizationGrowth(self, g):
        self.settings["growth"] = g

    def setStaticPivotFloor(self, rel, abs_=1e-300):
        self.settings["static_rel_floor"] = rel
        self.settings["static_abs_floor"] = abs_

    def setParallel(self, p):
        self.settings["parallel"] = 1 if p else 0

    def analyzePattern(self, A, options=None):
        from oracle.pyoracle import OracleSymLDLT
        n, cp, ri, _ = as_csc(A)
        self._an = Analysis(n, cp, ri, self.ordering, options or SymbolicFactorOptions())
        self._o = OracleSymLDLT(self._an.factor())
        self._o.set(mode=int(self.mode), **self.settings)
        if self.kkt is not None:
            self._o.setKKTBlockSizes(*self.kkt)
        if self.signs is not None:
            self._o.setExpectedSignPattern(self.signs)

    def factorize(self, A):
        from ma57_b200.solver import LogicError
        if self._o is None:
            raise LogicError("symla::SymLDLT::factorize: analyzePattern must be called first")
        self._o.factorize(A)

    def compute(self, A):
        self.analyzePattern(A)
        self.factorize(A)

    def refactorize(self, A):
        self.factorize(A)

    def solve(self, B):
        return self._o.solve(B)

    def solveWithRefinement(self, A, B, options=None):
        options = options or RefinementOptions()
        x, d = self._o.solveWithRefinement(A, B, options.max_iterations, options.tolerance)
        return RefinedSolve(x, RefinementResult(d["iterations"], d["initial"], d["final"]))

    def inertia(self):
        return Inertia(*self._o.inertia())

    def isSingular(self):
        return bool(self._o.info()["singular"])

    def singularColumns(self):
        return self._o.singularColumns()

    def factorized(self):
        return bool(self._o.info()["factorized"])

    def regularizationRetriesUsed(self):
        return self._o.info()["retries"]

    def lastRegularizationDelta(self):
        return self._o.info()["last_delta"]

    def totalPerturbation(self):
        return self._o.info()["total_perturbation"]

    def numPerturbedPivots(self):
        return self._o.info()["num_perturbed"]

    def symbolicFactor(self):
        return self._an.factor()

    def numericFactor(self):
        class NF:
            pass
        nf = NF()
        nf.fronts = [SupernodeFactor(f["rowIndices"], f["nPivots"], f["L"], f["Ddiag"], f["Doff"],
                                     [PivotBlock(s, k) for (s, k) in f["pivotBlocks"]]) for f in self._o.fronts()]
        nf.perm = self._an.factor().perm
        nf.inertia = self.inertia()
        nf.singular = self.isSingular()
        nf.n = len(nf.perm)
        return nf


IMPLS = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]


def make_solver(impl):
    return OracleSolver() if impl == "oracle" else SymLDLT()


# ---------------------------------------------------------------------------


def dense_sym(A) -> np.ndarray:
    """Dense symmetric matrix from the lower triangle of A."""
    return M.sym_full(A).toarray()


def dense_stored(A) -> np.ndarray:
    """Ad(i,j) = stored entry, then symmetrized from the stored triangle(s) the
    way the reference's toDense helpers do (both triangles set)."""
    A = sp.coo_matrix(A)
    Ad = np.zeros(A.shape)
    Ad[A.row, A.col] = A.data
    Ad[A.col, A.row] = A.data
    return Ad


def backward_error_inf(A, X, B):
    """refine.hpp:109-114 with ||A|| = max stored-entry row sum (refine.hpp:69-81)."""
    X = np.asarray(X).reshape(A.shape[0], -1)
    B = np.asarray(B).reshape(A.shape[0], -1)
    Af = M.sym_full(A)
    R = B - Af @ X
    normA = np.asarray(abs(sp.csr_matrix(A)).sum(axis=1)).max()
    den = normA * np.abs(X).max() + np.abs(B).max()
    return np.abs(R).max() / den if den > 0 else np.abs(R).max()


def ref_residual(Ad, X, B):
    """(Ad X - B).norm() / (max|Ad| * max(1, ||X||) + ||B||), Frobenius norms, as
    in the reference's correctness tests."""
    return np.linalg.norm(Ad @ X - B) / (np.abs(Ad).max() * max(1.0, np.linalg.norm(X)) + np.linalg.norm(B))


def flatten(sf_perm, nf):
    """Dense L, D and original-index order from per-front factors
    (test/unit/multifrontal_test_helpers.hpp:40-120)."""
    order = []
    for f in nf.fronts:
        order.extend(int(r) for r in f.rowIndices[:f.nPivots])
    n = len(order)
    pos = {g: t for t, g in enumerate(order)}
    Lf = np.eye(n)
    Df = np.zeros((n, n))
    for f in nf.fronts:
        k = f.nPivots
        rows = [pos[int(g)] for g in f.rowIndices]
        two = {b.start for b in f.pivotBlocks if b.kind == 1}
        for j in range(k):
            cj = rows[j]
            for i in range(j + 1, len(rows)):
                if i == j + 1 and j in two:
                    continue
                Lf[rows[i], cj] = f.L[i, j]
        for b in f.pivotBlocks:
            s = b.start
            if b.kind == 0:
                Df[rows[s], rows[s]] = f.Ddiag[s]
            else:
                a, c = rows[s], rows[s + 1]
                Df[a, a] = f.Ddiag[s]
                Df[c, c] = f.Ddiag[s + 1]
                Df[a, c] = Df[c, a] = f.Doff[s]
    orig = np.array([sf_perm[g] for g in order])
    return orig, Lf, Df


def random_symmetric_indefinite_eig(n, seed):
    """Q diag(lambda) Q^T with random signs, |lambda| in [0.5, 10]
    (the shape of dense_kernel_test.cpp's randomSymmetricIndefiniteEig)."""
    st = M.Stream(seed)
    G = st.normal(n * n).reshape(n, n)
    Q, _ = np.linalg.qr(G)
    lam = st.uniform(n, 0.5, 10.0) * np.where(st.uniform(n) < 0.5, -1.0, 1.0)
    return (Q * lam) @ Q.T


def hinge_chain(n_hinges, seed):
    """zero_diagonal_test.cpp:39-67: 2x2 hinges with exact zero diagonals."""
    st = M.Stream(seed)
    n = 2 * n_hinges
    rows, cols, vals = [], [], []
    cs = st.uniform(n_hinges, 0.5, 2.0)
    for h in range(n_hinges):
        a, b = 2 * h, 2 * h + 1
        rows += [a, b, b, a]
        cols += [a, b, a, b]
        vals += [0.0, 0.0, cs[h], cs[h]]
    cv = st.uniform(max(0, n_hinges - 1), -0.05, 0.05)
    for h in range(n_hinges - 1):
        a, bn = 2 * h, 2 * (h + 1)
        rows += [bn, a]
        cols += [a, bn]
        vals += [cv[h], cv[h]]
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsc()
    A.sum_duplicates()
    return A


def spd_block(n, avg, seed):
    return M.random_sparse_spd(n, avg, seed)


def random_rect(n2, n1, avg, seed):
    st = M.Stream(seed)
    rows, cols, vals = [], [], []
    for i in range(n2):
        ne = 1 + int(st.integers(1, avg)[0]) if avg > 0 else 0
        js = st.integers(ne, n1)
        vs = st.uniform(ne, -0.5, 0.5)
        rows += [i] * ne
        cols += list(js)
        vals += list(vs)
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n2, n1)).tocsc()
    A.sum_duplicates()
    return A


def with_diagonal_override(Mx, idx, val):
    Mx = sp.lil_matrix(Mx)
    Mx[idx, idx] = val
    return sp.csc_matrix(Mx)
