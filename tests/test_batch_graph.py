"""Graph launch of the factorization, the batched solver over many
independent systems (config 4's shape, fewer systems), and the measured
tile schedule: none of them may change a result."""
import numpy as np
import pytest

from ma57_b200 import OrderingType, SymLDLT, autotune
from ma57_b200 import matrices as M
from ma57_b200.batch import BatchedSolver

pytestmark = pytest.mark.gpu


def backward_error(A, X, B):
    Af = M.sym_full(A)
    R = B - Af @ X
    normA = abs(A).sum(axis=1).max()
    return np.abs(R).max() / (normA * np.abs(X).max() + np.abs(B).max())


@pytest.mark.parametrize("k", [12, 20])
def test_graph_launch_matches_stream_launch_bitwise(k):
    A, b = M.config1(k)
    xs = []
    for graph in (False, True):
        s = SymLDLT()
        s.setGraphLaunch(graph)
        s.analyzePattern(A)
        s.factorize(A)
        # a level that ran past its planned iterations raises its count, so
        # the next factorization recaptures once; the one after replays
        s.refactorize(A)
        first = s.graphStats()
        s.refactorize(A)
        xs.append((s.inertia().as_tuple(), s.solve(b), s.graphStats(), first))
    assert xs[0][0] == xs[1][0]
    np.testing.assert_array_equal(xs[0][1], xs[1][1])
    assert 1 <= xs[1][3]["captures"] <= 2
    assert xs[1][2]["captures"] == xs[1][3]["captures"]  # replayed, not recaptured
    assert xs[1][2]["resumes"] == xs[1][3]["resumes"]  # and ran within the graph
    assert xs[0][2]["captures"] == 0


def test_graph_launch_with_delayed_pivots_continues_on_host():
    K, b, n1, n2 = M.config2(grid=30, n2=300)
    ref = SymLDLT()
    ref.analyzePattern(K)
    ref.factorize(K)
    s = SymLDLT()
    s.setGraphLaunch(True)
    s.analyzePattern(K)
    s.factorize(K)
    s.refactorize(K)
    assert s.inertia().as_tuple() == ref.inertia().as_tuple() == (n2, n1, 0)
    np.testing.assert_array_equal(s.solve(b), ref.solve(b))


def test_batched_systems_match_individual_solves():
    systems = [M.config4_system(i) for i in range(24)]
    mats = [A for A, _, _, _ in systems]
    rng = np.random.default_rng(9)
    Bs = [rng.standard_normal((A.shape[0], 8)) for A in mats]
    bs = BatchedSolver(mats)
    bs.factorize()
    bs.factorize()
    Xs = bs.solve(Bs)
    assert bs.solver.graphStats()["captures"] == 1
    for A, B, X in zip(mats, Bs, Xs):
        s = SymLDLT()
        s.analyzePattern(A)
        s.factorize(A)
        Xi = s.solve(B)
        assert backward_error(A, X, B) <= 1e-12
        assert np.abs(X - Xi).max() <= 1e-10 * max(1.0, np.abs(Xi).max())


def test_autotuned_schedule_keeps_results():
    A, B = M.config3(20, nrhs=2)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.analyzePattern(A)
    s.factorize(A)
    inertia, X0 = s.inertia().as_tuple(), s.solve(B)
    schedule, base, best = autotune.tune(s, A, reps=1)
    assert best <= base
    s.factorize(A)
    assert s.inertia().as_tuple() == inertia
    assert backward_error(A, s.solve(B), B) <= 10 * max(backward_error(A, X0, B), 1e-16)
    info = autotune.level_info(s)
    assert any(i["small_threads"] or i["cluster_ctas"] for i in info) or not (schedule["small"] or schedule["large"])


@pytest.mark.parametrize("rows", [64, 128])
def test_update_tile_rows_keep_results(rows):
    """Both Schur-update tile shapes (rows x 64) give the same inertia and a
    backward error as small as the default's (the summation order within a
    tile is the same; only the tiling of the trailing block differs)."""
    import ctypes as C
    from ma57_b200 import _lib as L
    A, B = M.config3(20, nrhs=2)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.analyzePattern(A)
    s.factorize(A)
    inertia, X0 = s.inertia().as_tuple(), s.solve(B)
    lib = L.load()
    nlev = int(s.plan_stats()["levels"])
    for lv in range(nlev):
        assert lib.symla_gpu_set_level_update_rows(s._ctx.h, lv, rows) == L.SYMLA_OK
    out = C.c_int()
    assert lib.symla_gpu_level_update_rows(s._ctx.h, 0, C.byref(out)) == L.SYMLA_OK and out.value == rows
    assert lib.symla_gpu_set_level_update_rows(s._ctx.h, 0, 32) == L.SYMLA_ERR_INVALID
    s.factorize(A)
    assert s.inertia().as_tuple() == inertia
    X = s.solve(B)
    assert backward_error(A, X, B) <= 10 * max(backward_error(A, X0, B), 1e-16)
    np.testing.assert_allclose(X, X0, rtol=0, atol=1e-9 * np.abs(X0).max())


def _set_all_levels(s, small_threads, cluster_ctas):
    from ma57_b200 import _lib as L
    lib = L.load()
    for lv in range(int(s.plan_stats()["levels"])):
        assert lib.symla_gpu_set_level_schedule(s._ctx.h, lv, small_threads, cluster_ctas) == L.SYMLA_OK


def _factor_arrays(s):
    nf = s.numericFactor()
    return [(list(f.rowIndices), f.nPivots, np.asarray(f.L).copy(), np.r_[f.Ddiag, f.Doff]) for f in nf.fronts]


@pytest.mark.parametrize("case", ["batched", "kkt"])
def test_warp_per_front_matches_block_small_kernel_bitwise(case):
    """Fronts of at most 32 rows run one warp per front (eight per CTA) by
    default; forcing the 128-thread block kernel on every level gives the
    same factor bit for bit (same operations, reductions exact), including
    2 x 2 pivots, interchanges and delayed columns of an indefinite KKT
    system."""
    if case == "batched":
        mats = [M.config4_system(i)[0] for i in range(24)]
        A = BatchedSolver(mats).A
        ordering = OrderingType.Natural
    else:
        from helpers import random_rect, spd_block
        A = M.kkt(spd_block(300, 4, 5), spd_block(120, 4, 22), random_rect(120, 300, 3, 36))
        ordering = OrderingType.AMD
    runs = []
    for threads in (0, 128):
        s = SymLDLT()
        s.setOrdering(ordering)
        s.analyzePattern(A)
        s.factorize(A)
        _set_all_levels(s, threads, 0)
        s.factorize(A)
        runs.append((s.inertia().as_tuple(), _factor_arrays(s)))
    assert runs[0][0] == runs[1][0]
    for (r0, p0, l0, d0), (r1, p1, l1, d1) in zip(runs[0][1], runs[1][1]):
        assert r0 == r1 and p0 == p1
        np.testing.assert_array_equal(l0, l1)
        np.testing.assert_array_equal(d0, d1)


def test_single_cta_panel_keeps_results():
    """Panel cluster size 1 (the single-CTA panel kernel on every level)
    gives the inertia of the cluster kernel and a comparable backward
    error."""
    A, b = M.config1(14)
    s = SymLDLT()
    s.analyzePattern(A)
    s.factorize(A)
    inertia, x0 = s.inertia().as_tuple(), s.solve(b)
    _set_all_levels(s, 0, 1)
    s.factorize(A)
    assert s.inertia().as_tuple() == inertia
    x = s.solve(b)
    assert backward_error(A, x, b) <= 10 * max(backward_error(A, x0, b), 1e-16)
