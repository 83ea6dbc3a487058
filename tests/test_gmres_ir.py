"""GMRES-IR (symla_gpu_solve_gmres_refine), the refinement the reference
lists as missing (refine.hpp:52-57, README.md:215): outer refinement on the
FP64 residual with iterativeRefine's measure and acceptance rule, each
correction solved by GMRES preconditioned by the factorization.

Checked: it reaches the same backward error as fixed-precision refinement
with an accurate factor; with the mixed-precision factor it needs no more
outer iterations; and with a deliberately poor factor (static pivots
perturbed by a large delta) it converges where fixed-precision refinement
stalls. The backward error is recomputed here from the returned X."""
import numpy as np
import pytest

from ma57_b200 import (GmresRefinementOptions, Mode, OrderingType, Precision, RefinementOptions, SymLDLT)
from ma57_b200 import matrices as M

pytestmark = pytest.mark.gpu


def backward_error(A, X, B):
    R = B - M.sym_full(A) @ X
    normA = abs(A).sum(axis=1).max()
    return np.abs(R).max() / (normA * np.abs(X).max() + np.abs(B).max())


def test_gmres_ir_fp64_factor():
    A, B = M.config3(20, nrhs=4)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.analyzePattern(A)
    s.factorize(A)
    r = s.solveWithGmresRefinement(A, B, GmresRefinementOptions(tolerance=1e-14))
    assert r.diagnostics.final_relative_residual <= 1e-14 or backward_error(A, r.x, B) <= 1e-14
    assert backward_error(A, r.x, B) <= 1e-13


def test_gmres_ir_mixed_factor_needs_no_more_outer_steps():
    A, B = M.config3(24, nrhs=4)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.setPrecision(Precision.Mixed)
    s.analyzePattern(A)
    s.factorize(A)
    classic = s.solveWithRefinement(A, B, RefinementOptions(max_iterations=10, tolerance=1e-12))
    g = s.solveWithGmresRefinement(A, B, GmresRefinementOptions(max_outer=10, restart=8, tolerance=1e-12))
    assert backward_error(A, g.x, B) <= 1e-12
    assert g.diagnostics.final_relative_residual <= 1e-12
    assert g.diagnostics.outer_iterations <= max(1, classic.diagnostics.iterations)


def test_gmres_ir_converges_where_fixed_precision_refinement_stalls():
    """A KKT system factorized with static pivots perturbed by a delta far
    above the default (1e-3 of max|K|): the factor is only a rough inverse,
    so fixed-precision refinement contracts slowly and stops short of 1e-12
    in 3 iterations, while GMRES-IR with the same factor reaches it."""
    K, b, n1, n2 = M.config2(grid=30, n2=300)
    s = SymLDLT()
    s.setMode(Mode.StaticRegularized)
    s.setOrdering(OrderingType.AMD)
    s.setKKTBlockSizes(n1, n2)
    s.setInitialRegularizationDelta(1e-3 * abs(K.data).max())
    s.analyzePattern(K)
    s.factorize(K)
    classic = s.solveWithRefinement(K, b, RefinementOptions(max_iterations=3, tolerance=1e-12))
    g = s.solveWithGmresRefinement(K, b, GmresRefinementOptions(max_outer=3, restart=20, tolerance=1e-12))
    assert backward_error(K, g.x, b) <= 1e-12
    assert backward_error(K, g.x, b) < backward_error(K, classic.x, b)


def test_gmres_ir_errors_match_the_reference():
    from ma57_b200 import InvalidArgument, LogicError
    A, b = M.config1(6)
    s = SymLDLT()
    s.analyzePattern(A)
    with pytest.raises(LogicError):
        s.solveWithGmresRefinement(A, b)
    s.factorize(A)
    with pytest.raises(InvalidArgument):
        s.solveWithGmresRefinement(A, np.ones(A.shape[0] + 2))
    with pytest.raises(InvalidArgument):
        s.solveWithGmresRefinement(A, b, GmresRefinementOptions(restart=0))
