"""Dense frontal kernel: the reference's known-answer tests
(test/unit/dense_kernel_test.cpp:207-387) on the oracle, and the same cases on
the GPU kernel through a single dense front (Natural ordering, the whole
matrix is one supernode)."""
import numpy as np
import pytest
import scipy.linalg.lapack as lapack
import scipy.sparse as sp

from ma57_b200 import OrderingType, SymLDLT
from oracle.pyoracle import dense_factor

from helpers import ref_residual, random_symmetric_indefinite_eig


def reconstruct(Af, res, k):
    """P^T A P restricted to the first k pivots: L D L^T (dense_kernel_test.cpp
    reconstructPAPT)."""
    n = Af.shape[0]
    L = np.eye(n)
    D = np.zeros((n, n))
    two = {s for s, kind in res["pivots"] if kind == 1}
    for j in range(k):
        for i in range(j + 1, n):
            if i == j + 1 and j in two:
                continue
            L[i, j] = Af[i, j]
    for s, kind in res["pivots"]:
        D[s, s] = res["Ddiag"][s]
        if kind == 1:
            D[s + 1, s + 1] = res["Ddiag"][s + 1]
            D[s + 1, s] = D[s, s + 1] = res["Doff"][s]
    return (L[:, :k] @ D[:k, :k] @ L[:, :k].T)[:k, :k]


def apply_perm(A0, perm, k):
    p = np.asarray(perm)[:k]
    return A0[np.ix_(p, p)]


def solve_from(Af, res, b):
    n = Af.shape[0]
    p = res["perm"]
    L = np.tril(Af, -1) + np.eye(n)
    D = np.zeros((n, n))
    for s, kind in res["pivots"]:
        D[s, s] = res["Ddiag"][s]
        if kind == 1:
            L[s + 1, s] = 0.0
            D[s + 1, s + 1] = res["Ddiag"][s + 1]
            D[s + 1, s] = D[s, s + 1] = res["Doff"][s]
    y = np.linalg.solve(L @ D @ L.T, b[p])
    x = np.zeros(n)
    x[p] = y
    return x


def test_hand_verified_3x3_diagonal():
    A0 = np.array([[10, 1, 1], [1, 8, 1], [1, 1, 6]], float)
    Af, res = dense_factor(A0)
    assert res["n_factored"] == 3
    assert [k for _, k in res["pivots"]] == [0, 0, 0]
    assert list(res["perm"]) == [0, 1, 2]
    assert np.linalg.norm(reconstruct(Af, res, 3) - apply_perm(A0, res["perm"], 3)) / np.linalg.norm(A0) < 1e-12
    assert res["inertia"][:2] == (3, 0)


def test_hand_verified_forces_2x2():
    A0 = np.array([[0, 1, 0.2], [1, 0, 0.3], [0.2, 0.3, 5.0]])
    Af, res = dense_factor(A0)
    assert res["n_factored"] == 3
    assert res["pivots"][0] == (0, 1)
    assert res["inertia"][:2] == (2, 1)
    assert np.linalg.norm(reconstruct(Af, res, 3) - apply_perm(A0, res["perm"], 3)) / np.linalg.norm(A0) < 1e-10


def test_hand_verified_5x5_mixed():
    A0 = np.array([[20, 1, 0.5, 0.1, 0.1], [1, 15, 0.2, 0.1, 0.1], [0.5, 0.2, 0, 2, 0.1], [0.1, 0.1, 2, 0, 0.2],
                   [0.1, 0.1, 0.1, 0.2, 12]])
    Af, res = dense_factor(A0)
    assert res["n_factored"] == 5
    assert np.linalg.norm(reconstruct(Af, res, 5) - apply_perm(A0, res["perm"], 5)) / np.linalg.norm(A0) < 1e-10
    assert res["inertia"][0] + res["inertia"][1] == 5 and res["inertia"][2] == 0


@pytest.mark.parametrize("n", [10, 50, 200])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_residual_random(n, seed):
    A0 = random_symmetric_indefinite_eig(n, seed * 1000 + n)
    Af, res = dense_factor(A0)
    assert res["n_factored"] == n and not res["delayed_cols"]
    rel = np.linalg.norm(reconstruct(Af, res, n) - apply_perm(A0, res["perm"], n)) / np.linalg.norm(A0)
    assert rel < 1e-10
    b = np.random.default_rng(seed + 777).standard_normal(n)
    x = solve_from(Af, res, b)
    assert np.linalg.norm(A0 @ x - b) / (np.abs(A0).max() * np.linalg.norm(x) + np.linalg.norm(b)) < 1e-8
    assert res["max_growth"] < 1000.0


@pytest.mark.parametrize("panel", [1, 2, 7, 64, 1000])
def test_panel_sizes_agree(panel):
    """The blocked and unblocked paths are the same algorithm (dense_kernel.hpp:386-392)."""
    A0 = random_symmetric_indefinite_eig(120, 99)
    Af, res = dense_factor(A0, panel_size=panel)
    _, ref = dense_factor(A0, panel_size=1)
    assert res["inertia"] == ref["inertia"]
    assert np.linalg.norm(reconstruct(Af, res, 120) - apply_perm(A0, res["perm"], 120)) / np.linalg.norm(A0) < 1e-10


@pytest.mark.parametrize("n", [5, 10, 25, 50, 100])
@pytest.mark.parametrize("seed", [11, 22, 33])
def test_lapack_inertia_cross_check(n, seed):
    """Inertia equal to LAPACK dsytrf's (dense_kernel_test.cpp:305-333)."""
    A0 = random_symmetric_indefinite_eig(n, seed * 1000 + n)
    _, res = dense_factor(A0)
    lu, ipiv, info = lapack.dsytrf(A0, lower=1)
    assert info == 0
    pos = neg = 0
    k = 0
    while k < n:
        if ipiv[k] > 0:
            d = lu[k, k]
            pos += d > 0
            neg += d < 0
            k += 1
        else:
            blk = np.array([[lu[k, k], lu[k + 1, k]], [lu[k + 1, k], lu[k + 1, k + 1]]])
            ev = np.linalg.eigvalsh(blk)
            pos += int((ev > 0).sum())
            neg += int((ev < 0).sum())
            k += 2
    assert res["inertia"][:2] == (pos, neg)


def test_delayed_pivot_all_zero_trailing_block():
    A0 = np.zeros((5, 5))
    A0[0, 0], A0[1, 1], A0[2, 2] = 10, 8, 6
    A0[0, 1] = A0[1, 0] = 1
    A0[0, 2] = A0[2, 0] = 0.5
    A0[1, 2] = A0[2, 1] = 0.2
    Af, res = dense_factor(A0)
    assert res["n_factored"] == 3
    assert res["delayed_cols"] == [3, 4]
    rec = reconstruct(Af, res, 3)
    assert np.linalg.norm(rec - apply_perm(A0, res["perm"], 3)) / np.linalg.norm(A0[:3, :3]) < 1e-10


def test_delayed_pivot_rank_deficient_2x2():
    A0 = np.array([[100, 0, 0], [0, 0, 1e-20], [0, 1e-20, 2e-20]])
    Af, res = dense_factor(A0, zero_tolerance=1e-8)
    assert res["n_factored"] == 1
    assert len(res["delayed_cols"]) == 2
    assert abs(reconstruct(Af, res, 1)[0, 0] - A0[0, 0]) < 1e-8


def test_static_pivoting_perturbs_wrong_sign():
    """factorStatic: fixed order, 1x1 only, sign-matched perturbation
    (dense_kernel.hpp:982-1011)."""
    A0 = np.diag([2.0, -0.5, 3.0])
    _, res = dense_factor(A0, static=True, expected_sign=[1, 1, 1], delta=1.0)
    assert res["n_factored"] == 3
    assert res["num_perturbed"] == 1
    assert abs(res["Ddiag"][1] - 0.5) < 1e-15
    assert res["inertia"] == (3, 0, 0)


# ---------------------------------------------------------------------------
# The same cases on the GPU kernel: one dense front.


def _gpu_dense(A0, **kw):
    n = A0.shape[0]
    A = sp.csc_matrix((np.tril(A0)[np.tril_indices(n)[0], np.tril_indices(n)[1]],
                       (np.tril_indices(n)[0], np.tril_indices(n)[1])), shape=(n, n))
    s = SymLDLT()
    s.setOrdering(OrderingType.Natural)
    s.analyzePattern(A)
    s.factorize(A)
    return A, s


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["3x3", "2x2", "5x5"])
def test_gpu_hand_cases(case):
    A0 = {"3x3": np.array([[10, 1, 1], [1, 8, 1], [1, 1, 6]], float),
          "2x2": np.array([[0, 1, 0.2], [1, 0, 0.3], [0.2, 0.3, 5.0]]),
          "5x5": np.array([[20, 1, 0.5, 0.1, 0.1], [1, 15, 0.2, 0.1, 0.1], [0.5, 0.2, 0, 2, 0.1],
                           [0.1, 0.1, 2, 0, 0.2], [0.1, 0.1, 0.1, 0.2, 12]])}[case]
    A, s = _gpu_dense(A0)
    _, ref = dense_factor(A0)
    assert s.inertia().as_tuple() == ref["inertia"]
    nf = s.numericFactor()
    kinds = [b.kind for f in nf.fronts for b in f.pivotBlocks]
    assert kinds == [k for _, k in ref["pivots"]]
    b = np.arange(1.0, A0.shape[0] + 1)
    x = s.solve(b)
    assert ref_residual(A0, x, b) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("n", [10, 50, 100, 200, 400])
def test_gpu_dense_random_matches_lapack_inertia(n):
    A0 = random_symmetric_indefinite_eig(n, 7000 + n)
    A, s = _gpu_dense(A0)
    _, ref = dense_factor(A0)
    assert s.inertia().as_tuple() == ref["inertia"]
    b = np.random.default_rng(n).standard_normal(n)
    x = s.solve(b)
    assert ref_residual(A0, x, b) < 1e-10


def _dense_lower_csc(A0):
    n = A0.shape[0]
    ii, jj = np.tril_indices(n)
    return sp.csc_matrix((A0[ii, jj], (ii, jj)), shape=(n, n))


@pytest.mark.gpu
@pytest.mark.parametrize("n1,n2", [(120, 60), (400, 200)])
def test_gpu_dense_static_large_front(n1, n2):
    """One large front under Mode::StaticRegularized (the cluster panel's
    static branch): SQD inertia (n2, n1, 0)."""
    from ma57_b200 import Mode
    st = np.random.default_rng(n1)
    E = st.standard_normal((n1, n1))
    E = E @ E.T / n1 + np.eye(n1)
    Fm = st.standard_normal((n2, n2))
    Fm = Fm @ Fm.T / n2 + np.eye(n2)
    Ac = st.standard_normal((n2, n1)) * 0.3
    K = np.block([[-E, Ac.T], [Ac, Fm]])
    A = _dense_lower_csc(K)
    s = SymLDLT()
    s.setOrdering(OrderingType.Natural)
    s.setMode(Mode.StaticRegularized)
    s.setKKTBlockSizes(n1, n2)
    s.analyzePattern(A)
    s.factorize(A)
    assert s.inertia().as_tuple() == (n2, n1, 0)
    b = st.standard_normal(n1 + n2)
    assert ref_residual(K, s.solve(b), b) < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("n,z", [(300, 20), (700, 5)])
def test_gpu_large_front_singular_tail(n, z):
    """A large single front whose last z rows/columns are zero: those columns
    can never pivot (delayed at the root -> singular), the rest factor."""
    A0 = random_symmetric_indefinite_eig(n - z, 90 + n)
    K = np.zeros((n, n))
    K[: n - z, : n - z] = A0
    A = _dense_lower_csc(K + np.diag(np.r_[np.zeros(n - z), np.zeros(z)]))
    s = SymLDLT()
    s.setOrdering(OrderingType.Natural)
    s.analyzePattern(A)
    s.factorize(A)
    assert s.isSingular()
    assert sorted(s.singularColumns()) == list(range(n - z, n))
    _, ref = dense_factor(A0)
    i = s.inertia().as_tuple()
    assert i[:2] == ref["inertia"][:2]
