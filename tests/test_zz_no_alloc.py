"""symla_gpu_relative_residual_noalloc: the refinement residual measure
without any device allocation, for callers whose device memory belongs to
another allocator or whose loop cannot take cudaMalloc's device-wide
synchronisation. Its scratch is a fixed array inside the library, so it is
checked here against symla_gpu_solve_refine's own reported residuals on two
calls in a row (the second call must not see the first one's maxima).

The file name sorts last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from ma57_b200 import SymLDLT
from ma57_b200 import _lib as L
from ma57_b200 import matrices as M

pytestmark = pytest.mark.gpu


def _refine(lib, h, B, iterations):
    n, nrhs = B.shape
    X = np.zeros((n, nrhs), order="F")
    info = L.RefineInfo()
    rc = lib.symla_gpu_solve_refine(h, None, L.ptr_d(B), n, nrhs, L.ptr_d(X), n, 0, iterations, 0.0,
                                    C.byref(info))
    assert rc == L.SYMLA_OK, L.last_error()
    return X, info


def _noalloc(lib, h, dXt, dBt, n=None):
    """dXt, dBt: (nrhs, ld) contiguous device tensors, i.e. column-major
    ld x nrhs with the first n rows used (n defaults to ld)."""
    nrhs, ldx = dXt.shape
    ldb = dBt.shape[1]
    n = ldx if n is None else n
    out = C.c_double(-1.0)
    rc = lib.symla_gpu_relative_residual_noalloc(h, C.c_void_p(dXt.data_ptr()), ldx, C.c_void_p(dBt.data_ptr()), ldb,
                                                  nrhs, C.byref(out))
    assert rc == L.SYMLA_OK, L.last_error()
    return out.value


def test_noalloc_residual_matches_solve_refine_twice():
    import torch
    A, _ = M.config1(12)
    n = A.shape[0]
    nrhs = 3
    rng = np.random.default_rng(5)
    # the second right-hand side is 1000x smaller: stale maxima from the first
    # call would change its residual by orders of magnitude
    Bs = [np.asfortranarray(rng.standard_normal((n, nrhs))),
          np.asfortranarray(1e-3 * rng.standard_normal((n, nrhs)))]
    s = SymLDLT()
    s.analyzePattern(A)
    s.factorize(A)
    lib = L.load()
    h = s._ctx.h
    ref = [_refine(lib, h, B, 0) for B in Bs]  # no refinement: the residual of the returned X

    dev = torch.device("cuda", 0)
    for B, (X, info) in zip(Bs, ref):  # two calls in a row through the same scratch
        dBt = torch.from_numpy(np.ascontiguousarray(B.T)).to(dev)
        dXt = torch.from_numpy(np.ascontiguousarray(X.T)).to(dev)
        value = _noalloc(lib, h, dXt, dBt)
        expected = info.initial_relative_residual
        assert expected > 0.0
        assert abs(value - expected) <= 1e-12 * expected


def test_noalloc_residual_rejects_sizes_beyond_its_scratch():
    import torch
    A, _ = M.config1(6)
    s = SymLDLT()
    s.analyzePattern(A)
    s.factorize(A)
    lib = L.load()
    n = A.shape[0]
    nrhs = L.NOALLOC_RESIDUAL_MAX_ENTRIES // n + 1
    d = torch.zeros(n, dtype=torch.float64, device="cuda")  # never read: the size check comes first
    out = C.c_double(0.0)
    rc = lib.symla_gpu_relative_residual_noalloc(s._ctx.h, C.c_void_p(d.data_ptr()), n, C.c_void_p(d.data_ptr()), n,
                                                  nrhs, C.byref(out))
    assert rc == L.SYMLA_ERR_BAD_SIZE
    assert "exceeds the fixed scratch" in L.last_error()


def test_noalloc_residual_with_leading_dimensions_beyond_n():
    """X and B with leading dimensions larger than n: the rows past n of
    each column are padding filled with huge values, which must not enter
    the residual or the norms."""
    import torch
    A, _ = M.config1(10)
    n = A.shape[0]
    nrhs = 2
    B = np.asfortranarray(np.random.default_rng(11).standard_normal((n, nrhs)))
    s = SymLDLT()
    s.analyzePattern(A)
    s.factorize(A)
    lib = L.load()
    h = s._ctx.h
    X, info = _refine(lib, h, B, 0)
    dev = torch.device("cuda", 0)
    for ldx, ldb in ((n + 5, n + 3), (n + 1, n)):
        Xp = np.full((nrhs, ldx), 1e30)
        Bp = np.full((nrhs, ldb), -1e30)
        Xp[:, :n] = X.T
        Bp[:, :n] = B.T
        value = _noalloc(lib, h, torch.from_numpy(Xp).to(dev), torch.from_numpy(Bp).to(dev), n=n)
        expected = info.initial_relative_residual
        assert abs(value - expected) <= 1e-12 * expected, (ldx, ldb, value, expected)
