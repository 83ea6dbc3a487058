"""Mixed-precision factorization (TF32x3 tensor-core far Schur update, FP64
pivots, D and near updates) against the FP64 path on the same inputs.

The reference evaluates every Schur update in FP64 (dense_kernel.hpp:806-821),
so the bar here is: identical inertia, an unrefined solution within a
TF32x3-sized distance of the FP64 one, and iterative refinement
(refine.hpp:96-160) reaching the same 1e-12 backward error as FP64."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from ma57_b200 import OrderingType, Precision, RefinementOptions, SymLDLT
from ma57_b200 import _lib as L
from ma57_b200 import matrices as M

pytestmark = pytest.mark.gpu


def backward_error(A, x, b):
    Af = M.sym_full(A)
    r = b - Af @ x
    normA = abs(A).sum(axis=1).max()
    return np.abs(r).max() / (normA * np.abs(x).max() + np.abs(b).max())


def pair(A, ordering=OrderingType.AMD, kkt=None):
    out = []
    for prec in (Precision.FP64, Precision.Mixed):
        s = SymLDLT()
        s.setOrdering(ordering)
        s.setPrecision(prec)
        if kkt is not None:
            s.setKKTBlockSizes(*kkt)
        s.analyzePattern(A)
        s.factorize(A)
        out.append(s)
    return out


@pytest.mark.parametrize("k", [20, 28])
def test_shifted_laplacian_mixed_matches_fp64(k):
    A, b = M.config1(k)
    s64, smx = pair(A)
    assert smx.inertia().as_tuple() == s64.inertia().as_tuple()
    assert smx.plan_stats()["max_m"] > 128  # large fronts: the tensor-core path ran
    x64, xmx = s64.solve(b), smx.solve(b)
    rel = np.abs(xmx - x64).max() / np.abs(x64).max()
    assert 0.0 < rel < 1e-2  # TF32x3 error is ~1e-7 of |L||LD|, amplified by cond(A)
    r = smx.solveWithRefinement(A, b)
    assert r.diagnostics.final_relative_residual <= 1e-12
    assert r.diagnostics.iterations <= 6
    assert backward_error(A, r.x, b) <= 1e-12


def test_config3_multi_rhs_mixed_refines_to_fp64_accuracy():
    A, B = M.config3(24, nrhs=4)
    s64, smx = pair(A, OrderingType.Metis)
    assert smx.inertia().as_tuple() == s64.inertia().as_tuple()
    X64 = s64.solve(B)
    Xmx = smx.solve(B)
    assert not np.array_equal(X64, Xmx)  # a different (TF32x3) far update ran
    assert np.abs(Xmx - X64).max() / np.abs(X64).max() < 1e-2
    r = smx.solveWithRefinement(A, B)
    assert r.diagnostics.final_relative_residual <= 1e-12
    for j in range(B.shape[1]):
        assert backward_error(A, r.x[:, j], B[:, j]) <= 1e-12


def test_kkt_with_delays_mixed():
    K, b, n1, n2 = M.config2(grid=40, n2=600)
    s64, smx = pair(K, kkt=(n1, n2))
    assert smx.inertia().as_tuple() == s64.inertia().as_tuple() == (n2, n1, 0)
    r = smx.solveWithRefinement(K, b, RefinementOptions(max_iterations=10))
    assert backward_error(K, r.x, b) <= 1e-11


def test_mixed_far_update_is_instrumented():
    A, b = M.config1(20)
    s = SymLDLT()
    s.setPrecision(Precision.Mixed)
    s.analyzePattern(A)
    lib = L.load()
    s.factorize(A)
    lib.symla_gpu_reset_kernel_stats(s._ctx.h)
    lib.symla_gpu_set_profiling(s._ctx.h, 1)
    s.refactorize(A)
    lib.symla_gpu_set_profiling(s._ctx.h, 0)
    buf = (C.c_double * 4)()
    assert lib.symla_gpu_kernel_stats(s._ctx.h, L.KERNEL_KINDS.index("far_update"), buf) == 0
    assert buf[0] > 0  # launches
    assert buf[2] > 0  # counted flops
    assert s.inertia().as_tuple() == (7590, 410, 0)


@pytest.mark.parametrize("n", [300, 700])
def test_dense_front_factor_entries_close_to_fp64(n):
    """One large front (natural order, strongly diagonal, so both paths take
    the same 1x1 pivots): L and D of the mixed factorization agree with FP64
    to the TF32x3 accuracy of the far update, entry by entry."""
    st = np.random.default_rng(n)
    G = st.standard_normal((n, n))
    A0 = (G + G.T) / np.sqrt(n) + np.diag(st.choice([-1.0, 1.0], n) * (6.0 + st.random(n)))
    ii, jj = np.tril_indices(n)
    A = sp.csc_matrix((A0[ii, jj], (ii, jj)), shape=(n, n))
    fs = []
    for prec in (Precision.FP64, Precision.Mixed):
        s = SymLDLT()
        s.setOrdering(OrderingType.Natural)
        s.setPrecision(prec)
        s.analyzePattern(A)
        s.factorize(A)
        fs.append(s.numericFactor())
    assert fs[0].inertia.as_tuple() == fs[1].inertia.as_tuple()
    for f64, fmx in zip(fs[0].fronts, fs[1].fronts):
        assert [b.kind for b in f64.pivotBlocks] == [b.kind for b in fmx.pivotBlocks]
        np.testing.assert_array_equal(f64.rowIndices, fmx.rowIndices)
        assert np.abs(fmx.L - f64.L).max() <= 1e-5 * max(1.0, np.abs(f64.L).max())
        assert np.abs(fmx.Ddiag - f64.Ddiag).max() <= 1e-5 * np.abs(f64.Ddiag).max()
