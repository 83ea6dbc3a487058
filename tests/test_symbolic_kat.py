"""The reference's own known-answer tests of the host symbolic analysis,
ported onto the C ABI's analysis (symla_analyze / symla_compute_ordering) and
checked against a brute-force dense symbolic factorization
(oracle/symbolic_ref.py, a restatement of test_helpers.hpp:87-125):

* elimination-tree shapes and column counts (test/unit/elimination_tree_test.cpp:48-111);
* supernode-partition invariants (test/unit/symbolic_test.cpp:46-158);
* ordering validity and star-graph fill (test/unit/ordering_test.cpp:85-136);
* the METIS permutation in the reference's convention (ordering.hpp:130-141).

The random SPD matrices follow the recipe of randomSparseSPD
(test_helpers.hpp:38-77) on the project's portable generator (the
reference's std::mt19937 distributions are not portable), so the seeds name
different matrices than the reference's. Runs on the CPU."""
import numpy as np
import pytest
import scipy.sparse as sp

from ma57_b200 import OrderingType, SymLDLT, SymbolicFactorOptions, computeOrdering
from ma57_b200 import matrices as M
from oracle import symbolic_ref as R


def tridiagonal(n):
    """elimination_tree_test.cpp:19-29."""
    A = sp.diags([-np.ones(n - 1), 4 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1], shape=(n, n)) if n > 1 else \
        sp.csc_matrix(4 * np.ones((1, 1)))
    return sp.csc_matrix(A)


def arrow_hub_last(n):
    """elimination_tree_test.cpp:35-45: hub n-1 joined to every other node."""
    A = sp.lil_matrix((n, n))
    for i in range(n):
        A[i, i] = n + 1
    for i in range(n - 1):
        A[i, n - 1] = A[n - 1, i] = 1.0
    return sp.csc_matrix(A)


def arrow_upper_hub_first(n):
    """ordering_test.cpp:44-53: hub 0, only the upper triangle stored."""
    A = sp.lil_matrix((n, n))
    for i in range(n):
        A[i, i] = n + 1
    for i in range(1, n):
        A[0, i] = 1.0
    return sp.csc_matrix(A)


def star_hub_first(n):
    """ordering_test.cpp:55-65: hub 0, both triangles stored."""
    A = sp.lil_matrix((n, n))
    for i in range(n):
        A[i, i] = n + 1
    for i in range(1, n):
        A[0, i] = A[i, 0] = 1.0
    return sp.csc_matrix(A)


def analyze(A, ordering=OrderingType.Natural, opts=None):
    s = SymLDLT()
    s.setOrdering(ordering)
    s.analyzePattern(A, opts or SymbolicFactorOptions())
    return s.symbolicFactor()


def is_valid_permutation(p, n):
    p = np.asarray(p)
    return len(p) == n and np.array_equal(np.sort(p), np.arange(n))


# --- elimination_tree_test.cpp -------------------------------------------

def test_tridiagonal_chain_etree():
    """elimination_tree_test.cpp:48-60: parent[j] = j+1, colCount 2 then 1."""
    n = 5
    sf = analyze(tridiagonal(n))
    assert sf.etree.n == n
    assert list(sf.perm) == list(range(n))
    assert list(sf.etree.parent) == [1, 2, 3, 4, -1]
    assert list(sf.etree.colCount) == [2, 2, 2, 2, 1]


def test_arrow_star_etree():
    """elimination_tree_test.cpp:62-76: every leaf's parent is the hub."""
    n = 5
    sf = analyze(arrow_hub_last(n))
    assert list(sf.perm) == list(range(n))
    assert list(sf.etree.parent) == [n - 1] * (n - 1) + [-1]
    assert list(sf.etree.colCount) == [2] * (n - 1) + [1]


@pytest.mark.parametrize("n", [5, 10, 25, 40])
@pytest.mark.parametrize("ordering", [OrderingType.Natural, OrderingType.AMD])
def test_colcount_and_parent_match_brute_force(n, ordering):
    """elimination_tree_test.cpp:78-91 (colCount against the dense oracle on
    random SPD matrices, three trials per size); the etree parent is checked
    against the same filled pattern. Both are taken on the final permuted
    pattern P A P^T of the analysis."""
    for trial in range(3):
        A = M.random_sparse_spd(n, 3, 12345 + 17 * n + trial)
        sf = analyze(A, ordering)
        PAP = R.permute_symmetric(A, sf.perm)
        np.testing.assert_array_equal(sf.etree.colCount, R.dense_symbolic_colcounts(PAP))
        np.testing.assert_array_equal(sf.etree.parent, R.dense_symbolic_etree(PAP))


def test_etree_edge_sizes():
    """elimination_tree_test.cpp:93-107: n = 0 and n = 1."""
    sf0 = analyze(sp.csc_matrix((0, 0)))
    assert sf0.etree.n == 0 and len(sf0.supernodes) == 0
    sf1 = analyze(sp.csc_matrix(np.ones((1, 1))))
    assert sf1.etree.n == 1
    assert list(sf1.etree.parent) == [-1]
    assert list(sf1.etree.colCount) == [1]


# --- symbolic_test.cpp ----------------------------------------------------

def check_symbolic_factor(A, ordering, opts):
    """checkSymbolicFactor (symbolic_test.cpp:46-104)."""
    n = A.shape[0]
    sf = analyze(A, ordering, opts)
    assert is_valid_permutation(sf.perm, n)
    assert sf.etree.n == n
    total = int(np.sum(sf.etree.colCount, dtype=np.int64))
    funda_total, nxt = 0, 0
    for sn in sf.fundamentalSupernodes:
        assert sn.firstCol == nxt and sn.ncols > 0 and len(sn.rowPattern) >= sn.ncols
        assert list(sn.rowPattern[:sn.ncols]) == list(range(sn.firstCol, sn.firstCol + sn.ncols))
        funda_total += sn.storageNnz()
        nxt = sn.firstCol + sn.ncols
    assert nxt == n
    assert funda_total == total
    firsts = [sn.firstCol for sn in sf.fundamentalSupernodes]
    relaxed_total, nxt = 0, 0
    for sn in sf.supernodes:
        assert sn.firstCol == nxt and sn.ncols > 0 and len(sn.rowPattern) >= sn.ncols
        assert list(sn.rowPattern[:sn.ncols]) == list(range(sn.firstCol, sn.firstCol + sn.ncols))
        assert np.all(np.diff(sn.rowPattern) > 0)
        relaxed_total += sn.storageNnz()
        nxt = sn.firstCol + sn.ncols
        covered = sum(1 for fc in firsts if sn.firstCol <= fc < sn.firstCol + sn.ncols)
        if covered > 1:
            assert sn.ncols <= opts.max_relax_size
    assert nxt == n
    assert relaxed_total >= funda_total
    return sf


@pytest.mark.parametrize("n", [1, 2, 5, 20])
@pytest.mark.parametrize("ordering", [OrderingType.Natural, OrderingType.AMD])
def test_symbolic_tridiagonal(n, ordering):
    """symbolic_test.cpp:110-116."""
    check_symbolic_factor(tridiagonal(n), ordering, SymbolicFactorOptions())


@pytest.mark.parametrize("n", [5, 10, 25, 60])
@pytest.mark.parametrize("ordering", [OrderingType.Natural, OrderingType.AMD, OrderingType.Metis,
                                      OrderingType.MetisIperm])
def test_symbolic_random_spd(n, ordering):
    """symbolic_test.cpp:118-131 (three trials per size)."""
    for trial in range(3):
        check_symbolic_factor(M.random_sparse_spd(n, 4, 777 + 3 * n + trial), ordering, SymbolicFactorOptions())


def test_symbolic_relaxation_sweep():
    """symbolic_test.cpp:133-147: no relaxation and generous relaxation."""
    A = M.random_sparse_spd(80, 5, 999)
    tight = check_symbolic_factor(A, OrderingType.AMD, SymbolicFactorOptions(1, 0.0))
    loose = check_symbolic_factor(A, OrderingType.AMD, SymbolicFactorOptions(128, 1.0))
    # with merging disabled every supernode is a fundamental one
    assert [(s.firstCol, s.ncols) for s in tight.supernodes] == \
        [(s.firstCol, s.ncols) for s in tight.fundamentalSupernodes]
    assert len(loose.supernodes) <= len(tight.supernodes)


@pytest.mark.parametrize("ordering", [OrderingType.AMD, OrderingType.Metis])
def test_symbolic_larger(ordering):
    """symbolic_test.cpp:149-155: one larger random SPD matrix."""
    check_symbolic_factor(M.random_sparse_spd(500, 6, 2024), ordering, SymbolicFactorOptions())


# --- ordering_test.cpp ----------------------------------------------------

@pytest.mark.parametrize("n", [1, 2, 5, 10])
def test_ordering_validity(n):
    """ordering_test.cpp:85-101, including an upper-triangle-only input."""
    for A in (tridiagonal(n), arrow_upper_hub_first(n)):
        for ordering in (OrderingType.Natural, OrderingType.AMD):
            assert is_valid_permutation(computeOrdering(A, ordering), n)
        if n >= 2:
            for ordering in (OrderingType.Metis, OrderingType.MetisIperm):
                assert is_valid_permutation(computeOrdering(A, ordering), n)


def test_natural_ordering_is_identity():
    """ordering_test.cpp:103-107."""
    assert list(computeOrdering(tridiagonal(7), OrderingType.Natural)) == list(range(7))


def test_star_fill_reduction():
    """ordering_test.cpp:109-134: hub-first natural order fills the trailing
    block; AMD and METIS put the hub last (natural fill > 4x theirs)."""
    n = 60
    A = star_hub_first(n)
    natural = R.total_fill(A, np.arange(n))
    for ordering in (OrderingType.AMD, OrderingType.Metis):
        p = computeOrdering(A, ordering)
        assert is_valid_permutation(p, n)
        assert natural > 4 * R.total_fill(A, p), ordering


def test_metis_iperm_is_the_inverse_of_metis():
    """The reference takes METIS's second output array as its pivot order
    (ordering.hpp:130-141); SYMLA_ORDER_METIS takes the first. METIS returns
    the two as mutually inverse permutations."""
    A = M.config1(8)[0]
    p = computeOrdering(A, OrderingType.Metis)
    q = computeOrdering(A, OrderingType.MetisIperm)
    assert is_valid_permutation(p, A.shape[0]) and is_valid_permutation(q, A.shape[0])
    np.testing.assert_array_equal(q[p], np.arange(A.shape[0]))


def test_metis_pivot_order_fills_less_than_its_inverse():
    """Why SYMLA_ORDER_METIS departs from the reference's convention: on a 3D
    stencil the nested-dissection order (METIS's first array) fills far less
    than its inverse (the reference's choice)."""
    A = M.config1(8)[0]
    fill_nd = R.total_fill(A, computeOrdering(A, OrderingType.Metis))
    fill_ref = R.total_fill(A, computeOrdering(A, OrderingType.MetisIperm))
    assert fill_nd < fill_ref


@pytest.mark.parametrize("ordering", [OrderingType.AMD, OrderingType.Metis])
def test_oracle_library_analysis_is_the_same(ordering):
    """The oracle library carries its own build of the host analysis (so the
    CPU baseline runs without the product library); it must give the same
    permutation, elimination tree and supernodes."""
    from oracle.pyoracle import analyze
    A = M.config3(10, nrhs=1)[0]
    a = analyze(A, int(ordering))
    sf = globals()["analyze"](A, ordering)
    np.testing.assert_array_equal(a.perm, sf.perm)
    np.testing.assert_array_equal(a.etree.parent, sf.etree.parent)
    assert len(a.supernodes) == len(sf.supernodes)
    for x, y in zip(a.supernodes, sf.supernodes):
        assert (x.firstCol, x.ncols) == (y.firstCol, y.ncols)
        np.testing.assert_array_equal(x.rowPattern, y.rowPattern)
