"""Multifrontal factorize / solve / refine: the reference's unit, correctness
and stability tests (test/unit/multifrontal_test.cpp, test/correctness/*,
test/stability/*), run on the oracle (CPU) and on the GPU path."""
import numpy as np
import pytest
import scipy.sparse as sp

from ma57_b200 import Mode, OrderingType, SymbolicFactorOptions
from ma57_b200 import matrices as M
from ma57_b200.solver import InvalidArgument, LogicError

from helpers import (IMPLS, dense_stored, flatten, hinge_chain, make_solver, random_rect, ref_residual, spd_block,
                     with_diagonal_override)


def from_dense(A):
    return sp.csc_matrix(A)


def check_factorization_correctness(impl, A, ordering=OrderingType.AMD):
    """multifrontal_test.cpp:37-56"""
    n = A.shape[0]
    s = make_solver(impl)
    s.setOrdering(ordering)
    s.analyzePattern(A)
    s.factorize(A)
    assert s.factorized() and not s.isSingular()
    orig, Lf, Df = flatten(s.symbolicFactor().perm, s.numericFactor())
    Ad = dense_stored(A)
    Ap = Ad[np.ix_(orig, orig)]
    rec = Lf @ Df @ Lf.T
    assert np.linalg.norm(rec - Ap) / max(1.0, np.abs(Ap).max()) < 1e-8
    b = np.random.default_rng(12345 + n).standard_normal(n)
    x = s.solve(b)
    assert ref_residual(Ad, x, b) < 1e-8
    return s


@pytest.mark.parametrize("impl", IMPLS)
def test_hand_verified_spd_4x4(impl):
    A = np.array([[10, 1, 0, 1], [1, 8, 1, 0], [0, 1, 6, 1], [1, 0, 1, 9]], float)
    check_factorization_correctness(impl, from_dense(A))
    check_factorization_correctness(impl, from_dense(A), OrderingType.Natural)


@pytest.mark.parametrize("impl", IMPLS)
def test_hand_verified_indefinite_5x5(impl):
    A = np.array([[10, 1, 0, 0, 1], [1, -8, 1, 0, 0], [0, 1, 6, 1, 0], [0, 0, 1, -9, 1], [1, 0, 0, 1, 7]], float)
    s = check_factorization_correctness(impl, from_dense(A))
    i = s.inertia()
    assert i.n_pos + i.n_neg + i.n_zero == 5 and i.n_zero == 0


@pytest.mark.parametrize("impl", IMPLS)
def test_delayed_pivot_arrow(impl):
    """multifrontal_test.cpp:102-164: fronts' nPivots == [0, 0, 5]."""
    A = np.zeros((5, 5))
    A[2, 2], A[3, 3], A[4, 4] = 5.0, 7.0, 20.0
    A[2, 3] = A[3, 2] = 1.1
    A[3, 4] = A[4, 3] = 1.3
    A[2, 4] = A[4, 2] = 0.9
    A[0, 4] = A[4, 0] = 2.0
    A[1, 3] = A[3, 1] = 1.7
    S = from_dense(A)
    s = make_solver(impl)
    s.setOrdering(OrderingType.Natural)
    s.analyzePattern(S, SymbolicFactorOptions(max_relax_size=1, max_relax_fill_fraction=0.0))
    sf = s.symbolicFactor()
    assert [(x.firstCol, x.ncols) for x in sf.supernodes] == [(0, 1), (1, 1), (2, 3)]
    s.factorize(S)
    assert s.factorized() and not s.isSingular()
    nf = s.numericFactor()
    assert [f.nPivots for f in nf.fronts] == [0, 0, 5]
    i = s.inertia()
    assert i.n_pos + i.n_neg + i.n_zero == 5 and i.n_zero == 0
    orig, Lf, Df = flatten(sf.perm, nf)
    Ap = A[np.ix_(orig, orig)]
    assert np.linalg.norm(Lf @ Df @ Lf.T - Ap) / np.abs(Ap).max() < 1e-10
    b = np.array([1, 2, 3, 4, 5.0])
    x = s.solve(b)
    assert np.linalg.norm(A @ x - b) / (np.abs(A).max() * np.linalg.norm(x) + np.linalg.norm(b)) < 1e-10


@pytest.mark.parametrize("impl", IMPLS)
def test_genuinely_singular(impl):
    """multifrontal_test.cpp:171-196: singularColumns() == {1}."""
    A = np.zeros((3, 3))
    A[0, 0], A[2, 2] = 4.0, 3.0
    A[0, 2] = A[2, 0] = 0.5
    s = make_solver(impl)
    s.compute(from_dense(A))
    assert s.factorized() and s.isSingular()
    assert s.singularColumns() == [1]
    nf = s.numericFactor()
    assert sum(f.nPivots for f in nf.fronts) == 2
    i = s.inertia()
    assert i.n_pos + i.n_neg + i.n_zero == 2
    with pytest.raises(LogicError):
        s.solve(np.ones(3))


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("n", [4, 6, 8])
@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_random_small_indefinite(impl, n, seed):
    A = M.random_sparse_indefinite(n, 3, seed * 100 + n)
    check_factorization_correctness(impl, A)
    check_factorization_correctness(impl, A, OrderingType.Natural)


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("n", [20, 100, 500])
def test_multifrontal_correctness_inertia_matches_dense(impl, n):
    """multifrontal_correctness_test.cpp:39-115: inertia equal to a
    whole-matrix dense factorization; SPD gives (n, 0, 0)."""
    A = M.random_sparse_indefinite(n, 4, 4242 + n)
    s = check_factorization_correctness(impl, A)
    ev = np.linalg.eigvalsh(dense_stored(A))
    assert s.inertia().as_tuple() == (int((ev > 0).sum()), int((ev < 0).sum()), 0)
    Aspd = M.random_sparse_spd(n, 4, 777 + n)
    s2 = make_solver(impl)
    s2.compute(Aspd)
    assert s2.inertia().as_tuple() == (n, 0, 0)


@pytest.mark.parametrize("impl", IMPLS)
def test_solve_multi_rhs_equals_single(impl):
    """solve_test.cpp:66-75: multi-RHS equals single-RHS columns to 1e-12."""
    A = M.random_sparse_indefinite(300, 4, 31337)
    s = make_solver(impl)
    s.compute(A)
    B = np.random.default_rng(5).standard_normal((300, 7))
    X = s.solve(B)
    for c in range(7):
        xc = s.solve(B[:, c])
        assert np.abs(X[:, c] - xc).max() <= 1e-12 * max(1.0, np.abs(xc).max())
    assert ref_residual(dense_stored(A), X, B) < 1e-8


@pytest.mark.parametrize("impl", IMPLS)
def test_solve_errors(impl):
    """smoke_test.cpp:46-65 and solver.hpp:198-209."""
    A = from_dense(np.diag([2.0, 3.0]))
    s = make_solver(impl)
    with pytest.raises(LogicError):
        s.factorize(A)
    s.analyzePattern(A)
    if impl == "gpu":
        with pytest.raises(LogicError):
            s.solve(np.ones(2))
    s.factorize(A)
    x = s.solve(np.array([4.0, 9.0]))
    assert np.abs(x - [2, 3]).max() < 1e-12
    assert s.inertia().as_tuple() == (2, 0, 0)
    with pytest.raises(InvalidArgument):
        s.solve(np.ones(3))


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("n_hinges", [2, 10, 50, 200])
@pytest.mark.parametrize("ordering", [OrderingType.AMD, OrderingType.Natural, OrderingType.Metis])
def test_zero_diagonal_hinge_chain(impl, n_hinges, ordering):
    """zero_diagonal_test.cpp:77-111: inertia (h, h, 0), >= h 2x2 pivots."""
    A = hinge_chain(n_hinges, 1000 + n_hinges)
    s = make_solver(impl)
    s.setOrdering(ordering)
    s.compute(A)
    assert s.factorized() and not s.isSingular()
    assert s.inertia().as_tuple() == (n_hinges, n_hinges, 0)
    nf = s.numericFactor()
    assert sum(1 for f in nf.fronts for b in f.pivotBlocks if b.kind == 1) >= n_hinges
    Ad = dense_stored(A)
    xt = np.random.default_rng(n_hinges).standard_normal(2 * n_hinges)
    B = Ad @ xt
    X = s.solve(B)
    assert ref_residual(Ad, X, B) < 1e-8


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("n", [20, 50, 200])
@pytest.mark.parametrize("gap", [1e-4, 1e-8, 1e-12, 1e-16])
def test_near_singular(impl, n, gap):
    """near_singular_test.cpp:48-103"""
    A = M.random_sparse_indefinite(n, 5, n + int(gap * 1e6) + 17).tolil()
    t = n // 2
    A[t, t] = (1.0 if A[t, t] > 0 else -1.0) * gap
    A = sp.csc_matrix(A)
    s = make_solver(impl)
    s.compute(A)
    i = s.inertia()
    assert i.n_pos + i.n_neg + i.n_zero == n
    if s.isSingular():
        with pytest.raises(LogicError):
            s.solve(np.ones(n))
        return
    Ad = dense_stored(A)
    xt = np.random.default_rng(n).standard_normal(n)
    B = Ad @ xt
    X = s.solve(B)
    assert np.all(np.isfinite(X))
    assert ref_residual(Ad, X, B) < 1e-4


@pytest.mark.parametrize("impl", IMPLS)
def test_pivot_threshold_is_a_no_op(impl):
    """pivot_threshold_sweep_test.cpp:7-16, 39-89: u does not change results."""
    A = M.random_sparse_indefinite(150, 5, 2024)
    b = np.random.default_rng(1).standard_normal(150)
    xs, inert = [], []
    for u in [0.001, 0.01, 0.1, 0.5]:
        s = make_solver(impl)
        s.setPivotThreshold(u)
        s.compute(A)
        xs.append(s.solve(b))
        inert.append(s.inertia().as_tuple())
    assert all(x == inert[0] for x in inert)
    for x in xs[1:]:
        assert np.array_equal(x, xs[0])


# ---------------------------------------------------------------------------
# KKT static pivoting (test/correctness/kkt_static_pivoting_test.cpp)


def build_kkt(n1, n2, seed):
    E = spd_block(n1, 4, seed)
    F = spd_block(n2, 4, seed + 17)
    A = random_rect(n2, n1, 3, seed + 31)
    return M.kkt(E, F, A), E, F, A


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("n1,n2", [(30, 10), (120, 60), (400, 150)])
@pytest.mark.parametrize("ordering", [OrderingType.AMD, OrderingType.Natural])
def test_kkt_genuine_sqd(impl, n1, n2, ordering):
    K, *_ = build_kkt(n1, n2, 7 * n1 + n2)
    s = make_solver(impl)
    s.setOrdering(ordering)
    s.setMode(Mode.StaticRegularized)
    s.setKKTBlockSizes(n1, n2)
    s.analyzePattern(K)
    s.factorize(K)
    assert s.factorized() and not s.isSingular()
    assert s.inertia().as_tuple() == (n2, n1, 0)
    assert s.regularizationRetriesUsed() <= 1
    Kd = dense_stored(K)
    xt = np.random.default_rng(n1).standard_normal(n1 + n2)
    B = Kd @ xt
    X = s.solve(B)
    assert ref_residual(Kd, X, B) < 1e-6


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("n1,n2", [(40, 15), (150, 60)])
def test_kkt_near_sqd_regularization_triggers(impl, n1, n2):
    seed = 3 * n1 + n2
    E = spd_block(n1, 4, seed)
    F = spd_block(n2, 4, seed + 17)
    A = random_rect(n2, n1, 3, seed + 31)
    E = with_diagonal_override(E, 0, -0.05)
    K = M.kkt(E, F, A)
    s = make_solver(impl)
    s.setOrdering(OrderingType.AMD)
    s.setMode(Mode.StaticRegularized)
    s.setKKTBlockSizes(n1, n2)
    s.setInitialRegularizationDelta(1e-6)
    s.setRegularizationGrowth(10.0)
    s.setMaxRegularizationRetries(10)
    s.analyzePattern(K)
    s.factorize(K)
    assert s.factorized() and not s.isSingular()
    assert s.inertia().as_tuple() == (n2, n1, 0)
    assert s.regularizationRetriesUsed() >= 1
    f = make_solver(impl)
    f.setOrdering(OrderingType.AMD)
    f.setMode(Mode.StaticRegularized)
    f.setKKTBlockSizes(n1, n2)
    f.setInitialRegularizationDelta(1e-6)
    f.setRegularizationGrowth(10.0)
    f.setMaxRegularizationRetries(0)
    f.analyzePattern(K)
    with pytest.raises(RuntimeError):
        f.factorize(K)
    assert not f.factorized()


@pytest.mark.parametrize("impl", IMPLS)
def test_kkt_refinement_recovers_accuracy(impl):
    """kkt_static_pivoting_test.cpp: large floor forces perturbation; refined
    residual <= 1e-2 * raw and < 1e-8."""
    n1, n2 = 120, 50
    K, *_ = build_kkt(n1, n2, 99)
    s = make_solver(impl)
    s.setMode(Mode.StaticRegularized)
    s.setKKTBlockSizes(n1, n2)
    s.setStaticPivotFloor(100.0)
    s.setInitialRegularizationDelta(0.005)
    s.analyzePattern(K)
    s.factorize(K)
    assert s.inertia().as_tuple() == (n2, n1, 0)
    assert s.numPerturbedPivots() > 0
    Kd = dense_stored(K)
    xt = np.random.default_rng(3).standard_normal(n1 + n2)
    B = Kd @ xt
    raw = ref_residual(Kd, s.solve(B), B)
    r = s.solveWithRefinement(K, B)
    ref = ref_residual(Kd, r.x, B)
    assert ref <= 1e-2 * raw and ref < 1e-8


@pytest.mark.parametrize("impl", IMPLS)
def test_kkt_threshold_pivot_inertia(impl):
    """kkt_test.cpp:104-139: ThresholdPivot on K gives (n2, n1, 0)."""
    n1, n2 = 200, 80
    K, *_ = build_kkt(n1, n2, 5)
    s = make_solver(impl)
    s.compute(K)
    assert s.inertia().as_tuple() == (n2, n1, 0)
    Kd = dense_stored(K)
    b = np.random.default_rng(8).standard_normal(n1 + n2)
    assert ref_residual(Kd, s.solve(b), b) < 1e-8


@pytest.mark.parametrize("impl", IMPLS)
def test_refactorize_reuses_pattern(impl):
    A = M.random_sparse_indefinite(200, 4, 11)
    s = make_solver(impl)
    s.analyzePattern(A)
    for scale in [1.0, 2.0, -1.5]:
        A2 = A * scale
        s.refactorize(A2)
        b = np.ones(200)
        assert ref_residual(dense_stored(A2), s.solve(b), b) < 1e-8


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("kappa_exp", [1, 3, 5, 7, 9])
def test_conditioning_fuzz(impl, kappa_exp):
    """conditioning_fuzz_test.cpp:102-162: residual < 1e5 eps."""
    n = 60
    st = M.Stream(kappa_exp)
    Q, _ = np.linalg.qr(st.normal(n * n).reshape(n, n))
    lam = np.logspace(0, -kappa_exp, n) * np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    Ad = (Q * lam) @ Q.T
    Ad = 0.5 * (Ad + Ad.T)
    A = sp.csc_matrix(np.tril(Ad))
    s = make_solver(impl)
    s.compute(A)
    xt = st.normal(n)
    b = Ad @ xt
    x = s.solve(b)
    resid = np.linalg.norm(Ad @ x - b) / (np.linalg.norm(Ad, 2) * np.linalg.norm(x) + np.linalg.norm(b))
    assert resid < 1e5 * np.finfo(float).eps
