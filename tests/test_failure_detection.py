"""Failure detection and the reference's error contract, with every failure
made on the host or by a device wait given too little time -- nothing here
faults, traps or hangs a GPU:

* a device-side wait that runs out (the pipelined solves' block flags, the
  tensor-core Schur update's copy/MMA barriers; symla_gpu_set_wait_limit_ns)
  returns SYMLA_ERR_TIMEOUT, and the context stays usable;
* a context whose plan exceeds its device-memory limit fails with
  SYMLA_ERR_OOM (symla_gpu_set_memory_limit), and the next one succeeds;
* NaN / Inf injected into the matrix values: the calls return, and the same
  context factorizes the clean values correctly afterwards;
* size and call-order errors map to the reference's exceptions with its
  messages (solver.hpp:54-55, :140-143, :198-209, :299-315, :403-413).
"""
import ctypes as C

import numpy as np
import pytest

from ma57_b200 import (InvalidArgument, LogicError, Mode, OrderingType, Precision, RefinementOptions, SymLDLT)
from ma57_b200 import _lib as L
from ma57_b200 import matrices as M
from ma57_b200.solver import as_csc


def backward_error(A, X, B):
    R = B - M.sym_full(A) @ X
    normA = abs(A).sum(axis=1).max()
    return np.abs(R).max() / (normA * np.abs(X).max() + np.abs(B).max())


def test_kkt_block_size_errors_on_host():
    """setKKTBlockSizes rejects negative sizes (solver.hpp:54-55)."""
    s = SymLDLT()
    with pytest.raises(InvalidArgument, match="sizes must be nonnegative"):
        s.setKKTBlockSizes(-1, 3)


def test_factorize_before_analyze_is_a_logic_error():
    """solver.hpp:140-143."""
    A, _ = M.config1(4)
    with pytest.raises(LogicError, match="analyzePattern must be called first"):
        SymLDLT().factorize(A)


def test_memory_limit_rejects_negative():
    lib = L.load()
    assert lib.symla_gpu_set_memory_limit(-5) == L.SYMLA_ERR_INVALID
    assert lib.symla_gpu_set_memory_limit(0) == L.SYMLA_OK


@pytest.mark.gpu
def test_solve_wait_timeout_is_reported_and_context_survives():
    """A 1 ns limit cannot cover the forward solve's chain of 64-row blocks
    (each waits for the one before it), so a wait runs out: the solve
    returns SYMLA_ERR_TIMEOUT. With the default limit the same context solves
    again, bit for bit as before."""
    A, B = M.config3(24, nrhs=4)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.analyzePattern(A)
    s.factorize(A)
    assert s.plan_stats()["max_m"] > 256  # fronts with several row blocks
    X0 = s.solve(B)
    lib = L.load()
    assert lib.symla_gpu_set_wait_limit_ns(s._ctx.h, 1) == L.SYMLA_OK
    with pytest.raises(RuntimeError, match="timed out") as ei:
        s.solve(B)
    assert "status 7" in str(ei.value)  # SYMLA_ERR_TIMEOUT
    assert lib.symla_gpu_set_wait_limit_ns(s._ctx.h, 0) == L.SYMLA_OK
    X1 = s.solve(B)
    np.testing.assert_array_equal(X1, X0)
    assert backward_error(A, X1, B) < 1e-12


@pytest.mark.gpu
def test_tensor_core_wait_timeout_is_reported_and_context_survives():
    """The mixed-precision far update waits on TMA copies and MMA groups; a
    1 ns limit makes those waits run out. The CTA abandons its tile, drains
    (within the default limit) what it has in flight and frees its tensor
    memory; the factorization returns SYMLA_ERR_TIMEOUT. With the default
    limit the same context factorizes to the right inertia."""
    A, B = M.config3(24, nrhs=2)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.setPrecision(Precision.Mixed)
    s.analyzePattern(A)
    s.factorize(A)
    good = s.inertia().as_tuple()
    lib = L.load()
    lib.symla_gpu_reset_kernel_stats(s._ctx.h)
    assert lib.symla_gpu_set_wait_limit_ns(s._ctx.h, 1) == L.SYMLA_OK
    with pytest.raises(RuntimeError, match="timed out") as ei:
        s.factorize(A)
    assert "status 7" in str(ei.value)
    assert "no longer usable" not in str(ei.value)
    with pytest.raises(LogicError):  # the failed factorization is not solvable
        s.solve(B)
    assert lib.symla_gpu_set_wait_limit_ns(s._ctx.h, 0) == L.SYMLA_OK
    s.factorize(A)
    assert s.inertia().as_tuple() == good
    r = s.solveWithRefinement(A, B, RefinementOptions(tolerance=1e-12))
    assert r.diagnostics.final_relative_residual <= 1e-12


@pytest.mark.gpu
def test_undersized_memory_limit_gives_oom_then_recovers():
    """A plan that does not fit the device-memory limit fails with
    SYMLA_ERR_OOM at create time (no context is returned); with the limit
    lifted the same analysis creates and factorizes."""
    A, b = M.config1(12)
    s = SymLDLT()
    s.analyzePattern(A)
    lib = L.load()
    _, cp, ri, _ = as_csc(A)
    try:
        assert lib.symla_gpu_set_memory_limit(64 * 1024) == L.SYMLA_OK
        h = C.c_void_p()
        rc = lib.symla_gpu_create(s._analysis.h, A.shape[0], L.ptr_i(cp), L.ptr_i(ri), 0, C.byref(h))
        assert rc == L.SYMLA_ERR_OOM
        assert not h.value
        assert "memory limit" in L.last_error()
        with pytest.raises(RuntimeError, match="memory limit"):
            s.factorize(A)
    finally:
        lib.symla_gpu_set_memory_limit(0)
    s.factorize(A)
    assert s.inertia().as_tuple() == (1720 - 6, 6, 0) or sum(s.inertia().as_tuple()) == A.shape[0]
    x = s.solve(b)
    assert backward_error(A, x, b) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
@pytest.mark.parametrize("precision", [Precision.FP64, Precision.Mixed])
def test_nonfinite_values_then_clean_refactorization(bad, precision):
    """Host-injected NaN / Inf in the values (the reference does not check
    for them either): factorize, solve and refinement return without hanging
    and without reporting a converged solution, and the same context then
    refactorizes the clean values to the right inertia and accuracy."""
    A, B = M.config3(20, nrhs=2)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.setPrecision(precision)
    s.analyzePattern(A)
    s.factorize(A)
    good = s.inertia().as_tuple()
    Abad = A.copy()
    Abad.data[Abad.nnz // 2] = bad
    s.factorize(Abad)
    if not s.isSingular():
        r = s.solveWithRefinement(Abad, B, RefinementOptions(max_iterations=3, tolerance=1e-12))
        assert not (r.diagnostics.final_relative_residual <= 1e-12)
    else:
        with pytest.raises(LogicError, match="numerically singular"):
            s.solve(B)
    s.factorize(A)
    assert s.inertia().as_tuple() == good
    r = s.solveWithRefinement(A, B, RefinementOptions(tolerance=1e-12))
    assert r.diagnostics.final_relative_residual <= 1e-12
    assert backward_error(A, r.x, B) <= 1e-12


@pytest.mark.gpu
def test_size_and_order_errors_match_the_reference():
    A, b = M.config1(6)
    n = A.shape[0]
    s = SymLDLT()
    s.analyzePattern(A)
    with pytest.raises(LogicError, match=r"factorize\(\) must be called before solve\(\)"):
        s.solve(b)
    s.factorize(A)
    with pytest.raises(InvalidArgument, match="B.rows"):
        s.solve(np.ones(n + 1))
    lib = L.load()
    X = np.zeros(n)
    bb = np.ascontiguousarray(b)
    assert lib.symla_gpu_solve(s._ctx.h, L.ptr_d(bb), n, -1, L.ptr_d(X), n, 0) == L.SYMLA_ERR_BAD_SIZE
    assert lib.symla_gpu_solve(s._ctx.h, L.ptr_d(bb), n - 1, 1, L.ptr_d(X), n, 0) == L.SYMLA_ERR_BAD_SIZE
    assert lib.symla_gpu_solve(s._ctx.h, L.ptr_d(bb), n, 1, L.ptr_d(X), n - 1, 0) == L.SYMLA_ERR_BAD_SIZE
    # the context is untouched by rejected calls
    x = s.solve(b)
    assert backward_error(A, x, b) < 1e-12
    # StaticRegularized size checks (solver.hpp:299-315)
    k = SymLDLT()
    k.setMode(Mode.StaticRegularized)
    k.setKKTBlockSizes(n - 1, 2)
    k.analyzePattern(A)
    with pytest.raises(InvalidArgument, match="do not sum to the matrix size"):
        k.factorize(A)
    k.setExpectedSignPattern(np.ones(n - 3, np.int32))
    with pytest.raises(InvalidArgument, match="does not match the matrix size"):
        k.factorize(A)
    # retry budget exhausted (solver.hpp:403-413): the indefinite stencil
    # cannot have the all-positive inertia a one-block KKT expects
    k.setKKTBlockSizes(0, n)
    k.setMaxRegularizationRetries(0)
    with pytest.raises(RuntimeError, match="retry budget"):
        k.factorize(A)
