"""ORACLE -- test infrastructure only.

Brute-force symbolic factorization of a small symmetric pattern, the
independent check the reference's own symbolic tests use:

* ``dense_symbolic_colcounts`` restates ``denseSymbolicCholeskyColCounts``
  (test/unit/test_helpers.hpp:87-125): symmetric Gaussian elimination on a
  dense boolean copy of the (already permuted) pattern, treating every stored
  entry as structurally nonzero; colCount[j] = number of rows i >= j with
  L(i, j) nonzero.
* ``dense_symbolic_etree`` reads the elimination tree off the same filled
  pattern: parent[j] = the first row i > j with L(i, j) nonzero (Liu's
  definition, which elimination_tree.hpp:78-96 computes by union-find).
* ``total_fill`` is ``totalFill`` of test/unit/ordering_test.cpp:60-76: the
  column-count sum of P A P^T for a pivot order ``perm`` (perm[k] = original
  index of the k-th pivot).

O(n^3) in numpy; for the unit-test sizes (n <= a few hundred) only.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _filled(pattern) -> np.ndarray:
    A = sp.coo_matrix(pattern)
    n = A.shape[0]
    nz = np.zeros((n, n), dtype=bool)
    nz[A.row, A.col] = True
    nz[A.col, A.row] = True
    nz[np.arange(n), np.arange(n)] = True
    for j in range(n):
        below = j + 1 + np.flatnonzero(nz[j + 1:, j])
        if len(below) > 1:
            nz[np.ix_(below, below)] = True
    return nz


def dense_symbolic_colcounts(pattern) -> np.ndarray:
    """test_helpers.hpp:87-125."""
    nz = _filled(pattern)
    return np.tril(nz).sum(axis=0).astype(np.int64)


def dense_symbolic_etree(pattern) -> np.ndarray:
    """parent[j] = min{i > j : L(i, j) != 0}, or -1 for a root."""
    nz = _filled(pattern)
    n = nz.shape[0]
    parent = np.full(n, -1, dtype=np.int64)
    for j in range(n):
        below = np.flatnonzero(nz[j + 1:, j])
        if len(below):
            parent[j] = j + 1 + below[0]
    return parent


def permute_symmetric(pattern, perm) -> sp.coo_matrix:
    """P A P^T with row/column perm[k] of A becoming row/column k."""
    A = sp.coo_matrix(pattern)
    n = A.shape[0]
    new_index = np.empty(n, dtype=np.int64)
    new_index[np.asarray(perm)] = np.arange(n)
    return sp.coo_matrix((np.ones(A.nnz), (new_index[A.row], new_index[A.col])), shape=(n, n))


def total_fill(pattern, perm) -> int:
    """ordering_test.cpp:60-76."""
    return int(dense_symbolic_colcounts(permute_symmetric(pattern, perm)).sum())
