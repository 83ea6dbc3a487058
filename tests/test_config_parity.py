"""GPU parity with the oracle on the benchmark configurations at their stated
sizes (or, for the 64^3 stencil, the largest size the oracle finishes within
a test's budget):

* the KKT saddle-point system (n = 60000, StaticRegularized,
  setKKTBlockSizes(40000, 20000), refinement to 1e-12) against the oracle's
  results committed in tests/golden/oracle_config2.json (the oracle needs
  about ten minutes for it; tests/golden/make_oracle_golden.py made the file);
* the 27-point stencil L27(k^3) - 3I with METIS and 16 right-hand sides,
  against the oracle run live at k = 32, in FP64 and in mixed precision;
* the 27-point stencil at 64^3 against its exact inertia (261360, 784, 0),
  known in closed form from the stencil's spectrum.

The bar (as for every parity test here): identical inertia, and a backward
error ||B - A X||_inf / (||A||_inf ||X||_inf + ||B||_inf) (refine.hpp:109-114)
within 10x of the oracle's, and at most 1e-12 after refinement."""
import json
import os

import numpy as np
import pytest

from ma57_b200 import Mode, OrderingType, Precision, RefinementOptions, SymLDLT
from ma57_b200 import matrices as M

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "oracle_config2.json")


def backward_error(A, X, B):
    Af = M.sym_full(A)
    R = B - Af @ X
    normA = abs(A).sum(axis=1).max()  # stored-entry row sums (refine.hpp:69-81)
    return float(np.abs(R).max() / (normA * np.abs(X).max() + np.abs(B).max()))


def analytic_inertia_l27(k, shift):
    """Inertia of L27(k^3) - shift I (Dirichlet, centre 26, neighbours -1):
    eigenvalues 27 - prod_i (1 + 2 cos(pi j_i / (k + 1))) - shift."""
    c = 1.0 + 2.0 * np.cos(np.pi * np.arange(1, k + 1) / (k + 1))
    lam = 27.0 - shift - np.einsum("i,j,l->ijl", c, c, c).ravel()
    return (int(np.sum(lam > 0)), int(np.sum(lam < 0)), int(np.sum(lam == 0)))


def _golden():
    with open(GOLDEN) as f:
        return json.load(f)["config2"]


def test_config2_fixture_matches_generator():
    """CPU: the committed oracle results belong to the matrix and symbolic
    analysis the generator makes today, and carry the exact inertia."""
    import importlib.util
    g = _golden()
    spec = importlib.util.spec_from_file_location("mk", os.path.join(HERE, "golden", "make_oracle_golden.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    K, b, n1, n2 = M.config2()
    assert mk.fingerprint(K) == g["matrix"]["sha256"]
    s = SymLDLT()
    s.setOrdering(OrderingType.AMD)
    s.analyzePattern(K)
    assert mk.symbolic_summary(s.symbolicFactor()) == g["symbolic"]
    # E's eigenvalues lie in [1.05e-2, 8.01] and F > 0: K is quasi-definite
    assert g["oracle"]["inertia"] == [n2, n1, 0]
    assert g["oracle"]["backward_error_refined"] <= 1e-12


def test_config3_analytic_inertia_formula():
    """CPU: the closed-form inertia of the 27-point configuration."""
    assert analytic_inertia_l27(64, 3.0) == (261360, 784, 0)
    w = np.linalg.eigvalsh(M.sym_full(M.config3(10, nrhs=1)[0]).toarray())
    assert analytic_inertia_l27(10, 3.0) == (int(np.sum(w > 0)), int(np.sum(w < 0)), 0)
    assert analytic_inertia_l27(10, 3.0)[1] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [Precision.FP64, Precision.Mixed])
def test_config2_full_size_matches_oracle(precision):
    g = _golden()
    K, b, n1, n2 = M.config2()
    s = SymLDLT()
    s.setMode(Mode.StaticRegularized)
    s.setOrdering(OrderingType.AMD)
    s.setKKTBlockSizes(n1, n2)
    s.setPrecision(precision)
    s.analyzePattern(K)
    s.factorize(K)
    assert list(s.inertia().as_tuple()) == g["oracle"]["inertia"] == [n2, n1, 0]
    assert s.regularizationRetriesUsed() == g["oracle"]["retries"]
    if precision == Precision.FP64:
        # static pivots perturbed where a pivot falls below the floor or has
        # the wrong sign; pivots sitting on that boundary may round either way
        assert abs(s.numPerturbedPivots() - g["oracle"]["num_perturbed"]) <= max(5, 0.01 * g["oracle"]["num_perturbed"])
        e0 = backward_error(K, s.solve(b), b)
        assert e0 <= 10 * max(g["oracle"]["backward_error_unrefined"], 1e-15)
    r = s.solveWithRefinement(K, b, RefinementOptions(max_iterations=10, tolerance=1e-12))
    e = backward_error(K, r.x, b)
    assert e <= 1e-12
    assert e <= 10 * max(g["oracle"]["backward_error_refined"], 1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [Precision.FP64, Precision.Mixed])
def test_config3_k32_matches_oracle(precision):
    from oracle.pyoracle import OracleSymLDLT
    k = 32
    A, B = M.config3(k, nrhs=16)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.setPrecision(precision)
    s.analyzePattern(A)
    s.factorize(A)
    o = OracleSymLDLT(s.symbolicFactor())
    o.set(parallel=1, num_threads=os.cpu_count() or 1)
    o.factorize(A)
    assert s.inertia().as_tuple() == o.inertia() == analytic_inertia_l27(k, 3.0)
    Xo = o.solve(B)
    e_ref = backward_error(A, Xo, B)
    if precision == Precision.FP64:
        X = s.solve(B)
        assert backward_error(A, X, B) <= 10 * max(e_ref, 1e-16)
        np.testing.assert_allclose(X, Xo, rtol=0, atol=1e-8 * np.abs(Xo).max())
    r = s.solveWithRefinement(A, B, RefinementOptions(max_iterations=10, tolerance=1e-12))
    e = backward_error(A, r.x, B)
    assert e <= 1e-12
    assert e <= 10 * max(e_ref, 1e-16) or precision == Precision.Mixed and e <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [Precision.FP64, Precision.Mixed])
def test_config3_64_analytic_inertia(precision):
    A, B = M.config3(64, nrhs=16)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.setPrecision(precision)
    s.setGraphLaunch(True)
    s.analyzePattern(A)
    s.factorize(A)
    assert s.inertia().as_tuple() == (261360, 784, 0)
    r = s.solveWithRefinement(A, B, RefinementOptions(max_iterations=10, tolerance=1e-12))
    assert r.diagnostics.final_relative_residual <= 1e-12
    assert backward_error(A, r.x, B) <= 1e-12
