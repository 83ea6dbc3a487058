"""The C ABI library: it loads, exports every function include/symla_gpu.h
declares, and the host-only entry points work without a GPU; device entry
points report an error (no CPU fallback) when no CUDA device is present."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from ma57_b200 import _lib as L
from ma57_b200 import matrices as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "symla_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(symla_\w+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    lib = L.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(L.EXPORTED)


def test_analyze_runs_on_host():
    A, _ = M.config1(6)
    from ma57_b200.solver import Analysis, SymbolicFactorOptions, as_csc
    n, cp, ri, _ = as_csc(A)
    sf = Analysis(n, cp, ri, 0, SymbolicFactorOptions()).factor()
    assert sorted(sf.perm) == list(range(n))
    assert sum(s.ncols for s in sf.supernodes) == n


def test_status_codes_and_errors_without_device():
    lib = L.load()
    out = C.c_void_p()
    # bad ordering -> INVALID
    cp = np.array([0, 1], np.int32)
    ri = np.array([0], np.int32)
    assert lib.symla_analyze(1, L.ptr_i(cp), L.ptr_i(ri), 7, 64, 0.25, C.byref(out)) == L.SYMLA_ERR_INVALID
    assert "OrderingType" in L.last_error()
    # no symbolic -> NOT_ANALYZED
    assert lib.symla_gpu_create(None, 1, L.ptr_i(cp), L.ptr_i(ri), 0, C.byref(out)) == L.SYMLA_ERR_NOT_ANALYZED
    # a solve on a NULL context -> NOT_FACTORIZED (logic_error in the C++ / Python wrappers)
    b = np.ones(1)
    assert lib.symla_gpu_solve(None, L.ptr_d(b), 1, 1, L.ptr_d(b), 1, 0) == L.SYMLA_ERR_NOT_FACTORIZED


def test_device_entry_points_fail_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = L.load()
    A, _ = M.config1(4)
    from ma57_b200.solver import as_csc
    n, cp, ri, _ = as_csc(A)
    sym = C.c_void_p()
    assert lib.symla_analyze(n, L.ptr_i(cp), L.ptr_i(ri), 0, 64, 0.25, C.byref(sym)) == 0
    ctx = C.c_void_p()
    rc = lib.symla_gpu_create(sym, n, L.ptr_i(cp), L.ptr_i(ri), 0, C.byref(ctx))
    assert rc in (L.SYMLA_ERR_NO_DEVICE, L.SYMLA_ERR_CUDA)
    assert not ctx.value
    lib.symla_symbolic_destroy(sym)
