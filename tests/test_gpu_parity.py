"""GPU parity against the oracle (CPU restatement of the reference) on the
same seeded inputs. Inertia must be identical; the GPU backward error must be
within 10x of the oracle's (and below the reference's own test bounds)."""
import numpy as np
import pytest

from ma57_b200 import Mode, OrderingType, SymLDLT
from ma57_b200 import matrices as M
from oracle.pyoracle import OracleSymLDLT

pytestmark = pytest.mark.gpu


def backward_error(A, x, b):
    """||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) (refine.hpp:109-114)."""
    Af = M.sym_full(A)
    r = b - Af @ x
    normA = abs(A).sum(axis=1).max()  # stored-entry row sums (refine.hpp:69-81)
    return np.abs(r).max() / (normA * np.abs(x).max() + np.abs(b).max())


@pytest.mark.parametrize("k", [6, 12, 20])
def test_shifted_laplacian_inertia_and_residual(k):
    A, b = M.config1(k)
    s = SymLDLT()
    s.analyzePattern(A)
    s.factorize(A)
    o = OracleSymLDLT(s.symbolicFactor())
    o.factorize(A)
    assert s.inertia().as_tuple() == o.inertia()
    x = s.solve(b)
    xo = o.solve(b)
    e_gpu, e_ref = backward_error(A, x, b), backward_error(A, xo, b)
    assert e_gpu <= 10 * max(e_ref, 1e-16)
    assert np.allclose(x, xo, rtol=1e-6, atol=1e-8 * np.abs(xo).max())


def test_config1_analytic_inertia():
    A, b = M.config1(20)
    s = SymLDLT()
    s.analyzePattern(A)
    s.factorize(A)
    assert s.inertia().as_tuple() == (7590, 410, 0)
    r = s.solveWithRefinement(A, b)
    assert r.diagnostics.final_relative_residual <= 1e-12
    assert backward_error(A, r.x, b) <= 1e-12
