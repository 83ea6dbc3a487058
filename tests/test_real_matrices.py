"""The reference's real-matrix suite (test/correctness/real_matrix_test.cpp:40-197)
and its amalgamation guard (test/stability/supernode_amalgamation_regression_test.cpp:44-83),
over the curated SuiteSparse list of bench/fetch_matrices.py:57-86.

The matrices are not in this repository and cannot be downloaded here; as in
the reference, each test skips (per matrix) when its file is absent. Point
SYMLA_MATRICES at a directory laid out as <group>/<name>/<name>.mtx (the
layout the reference's fetch script produces) to run them. The Matrix Market
reader itself is tested on files written here."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from ma57_b200 import OrderingType, SymLDLT
from ma57_b200 import matrices as M
from ma57_b200.matrix_market import MatrixMarketError, collection_path, load_market, save_market

MATRICES = [
    ("GHS_indef", "sit100"), ("GHS_indef", "tuma2"), ("GHS_indef", "ncvxqp1"), ("GHS_indef", "tuma1"),
    ("GHS_indef", "qpband"), ("GHS_indef", "bratu3d"), ("GHS_indef", "c-55"), ("GHS_indef", "aug3dcqp"),
    ("GHS_indef", "stokes128"), ("GHS_indef", "dawson5"), ("GHS_indef", "blockqp1"), ("GHS_indef", "cont-201"),
    ("GHS_indef", "turon_m"), ("GHS_indef", "helm2d03"), ("Schenk_IBMNA", "c-18"), ("Schenk_IBMNA", "c-22"),
    ("Schenk_IBMNA", "c-26"), ("Schenk_IBMNA", "c-30"), ("Schenk_IBMNA", "c-62"), ("Schenk_IBMNA", "c-67"),
    ("HB", "bcsstk14"), ("HB", "bcsstk16"),
]
ROOT = os.environ.get("SYMLA_MATRICES", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                    "bench", "matrices"))
MAX_N = 25000  # real_matrix_test.cpp:114 caps the gated suite at this size


def _load_or_skip(group, name):
    path = collection_path(ROOT, group, name)
    if not os.path.exists(path):
        pytest.skip(f"{group}/{name} not fetched ({path}); set SYMLA_MATRICES")
    A = load_market(path)
    if A.shape[0] != A.shape[1]:
        pytest.skip(f"{group}/{name} is not square")
    return A


def residual_self_adjoint(A, X, B):
    """real_matrix_test.cpp:55-62: ||A X - B|| / (max|a| max(1, ||X||) + ||B||)
    with A from its stored lower triangle, Frobenius norms."""
    AX = M.sym_full(A) @ X
    amax = abs(A).max() or 1.0
    return np.linalg.norm(AX - B) / (amax * max(1.0, np.linalg.norm(X)) + np.linalg.norm(B))


# --- the reader ------------------------------------------------------------

def test_market_round_trip(tmp_path):
    A, _ = M.config1(5)
    p = tmp_path / "a.mtx"
    save_market(p, A, symmetric=True, comment="lower triangle of L7(5^3) - 2I")
    B = load_market(p)
    assert (B != sp.csc_matrix(A)).nnz == 0
    G = sp.random(7, 5, density=0.4, random_state=2, format="csc")
    save_market(tmp_path / "g.mtx", G)
    np.testing.assert_array_equal(load_market(tmp_path / "g.mtx").toarray(), G.toarray())


def test_market_fields_and_errors(tmp_path):
    p = tmp_path / "p.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n% comment\n\n3 3 4\n1 1\n2 1\n3 3\n2 1\n")
    A = load_market(p)
    assert A.shape == (3, 3) and A[0, 0] == 1.0 and A[1, 0] == 2.0 and A[2, 2] == 1.0  # duplicates summed
    q = tmp_path / "i.mtx"
    q.write_text("%%MatrixMarket matrix coordinate integer general\n2 2 2\n1 2 5\n2 1 -3\n")
    assert load_market(q).toarray().tolist() == [[0.0, 5.0], [-3.0, 0.0]]
    bad = tmp_path / "c.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n")
    with pytest.raises(MatrixMarketError):
        load_market(bad)
    short = tmp_path / "s.mtx"
    short.write_text("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n")
    with pytest.raises(MatrixMarketError):
        load_market(short)


# --- the reference's suite ---------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("group,name", MATRICES, ids=[f"{g}/{n}" for g, n in MATRICES])
def test_real_matrix(group, name):
    """real_matrix_test.cpp:75-190: AMD, compute, inertia self-consistency,
    solve of b = A x_true, residual below 0.05."""
    A = _load_or_skip(group, name)
    n = A.shape[0]
    if n > MAX_N:
        pytest.skip(f"{group}/{name}: n={n} above the suite's cap of {MAX_N}")
    s = SymLDLT()
    s.setOrdering(OrderingType.AMD)
    s.compute(A)
    assert s.factorized()
    inertia = s.inertia()
    nsing = len(s.singularColumns())
    assert inertia.n_pos + inertia.n_neg + inertia.n_zero == n - nsing
    if s.isSingular():
        return
    xtrue = M.Stream(1234567 + n).normal(n)
    B = (M.sym_full(A) @ xtrue).reshape(n, 1)
    X = s.solve(B)
    assert residual_self_adjoint(A, X, B) < 0.05


def test_stokes128_amalgamation():
    """supernode_amalgamation_regression_test.cpp:44-83: with the default
    relaxation, stokes128's supernodes average more than 5 columns."""
    A = _load_or_skip("GHS_indef", "stokes128")
    s = SymLDLT()
    s.setOrdering(OrderingType.AMD)
    s.analyzePattern(A)
    sns = s.symbolicFactor().supernodes
    assert sns and A.shape[0] / len(sns) > 5.0
