"""Runs a fixed set of factorizations and solves through whichever native
library the environment selects (SYMLA_GPU_LIBRARY) and saves the results,
for tests/test_checked_build.py to compare the bounds-checked build with the
ordinary one. Usage: python tests/checked_worker.py OUT.npz"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from ma57_b200 import Mode, OrderingType, Precision, RefinementOptions, SymbolicFactorOptions, SymLDLT  # noqa: E402
from ma57_b200 import _lib as L  # noqa: E402
from ma57_b200 import matrices as M  # noqa: E402


def arrow():
    """The delayed-pivot arrow of multifrontal_test.cpp:102-164 (the
    factorization re-plans its root front)."""
    import scipy.sparse as sp
    A = np.zeros((5, 5))
    A[2, 2], A[3, 3], A[4, 4] = 5.0, 7.0, 20.0
    A[2, 3] = A[3, 2] = 1.1
    A[3, 4] = A[4, 3] = 1.3
    A[2, 4] = A[4, 2] = 0.9
    A[0, 4] = A[4, 0] = 2.0
    A[1, 3] = A[3, 1] = 1.7
    return sp.csc_matrix(np.tril(A)), np.arange(1.0, 6.0).reshape(5, 1)


def status(s):
    cnt, code, where = L.C.c_int(), L.C.c_int(), L.C.c_longlong()
    assert L.load().symla_gpu_check_status(s._ctx.h, L.C.byref(cnt), L.C.byref(code), L.C.byref(where)) == 0
    return [cnt.value, code.value, where.value]


def main(out):
    res = {"checked_build": np.array(L.load().symla_gpu_checked_build())}
    A, B = arrow()
    s = SymLDLT()
    s.setOrdering(OrderingType.Natural)
    s.analyzePattern(A, SymbolicFactorOptions(max_relax_size=1, max_relax_fill_fraction=0.0))
    s.factorize(A)
    res["arrow_npiv"] = np.array([f.nPivots for f in s.numericFactor().fronts])
    res["arrow_x"] = s.solve(B)
    res["arrow_dynamic"] = np.array(s.last_info.used_dynamic_path)
    res["arrow_status"] = np.array(status(s))
    cases = [("c1", *M.config1(12), Precision.FP64, Mode.ThresholdPivot),
             ("c3", *M.config3(24, nrhs=4), Precision.FP64, Mode.ThresholdPivot),
             ("c3m", *M.config3(24, nrhs=4), Precision.Mixed, Mode.ThresholdPivot)]
    K, b, n1, n2 = M.config2(grid=40, n2=600)
    cases += [("kkt", K, b, Precision.FP64, Mode.ThresholdPivot), ("kkts", K, b, Precision.FP64, Mode.StaticRegularized)]
    for name, A, B, prec, mode in cases:
        s = SymLDLT()
        s.setOrdering(OrderingType.Metis if name.startswith("c3") else OrderingType.AMD)
        s.setPrecision(prec)
        s.setMode(mode)
        if mode == Mode.StaticRegularized:
            s.setKKTBlockSizes(n1, n2)
        s.analyzePattern(A)
        s.factorize(A)
        res[name + "_inertia"] = np.array(s.inertia().as_tuple())
        res[name + "_dynamic"] = np.array(s.last_info.used_dynamic_path)
        res[name + "_x"] = s.solve(B)
        r = s.solveWithRefinement(A, B, RefinementOptions(max_iterations=10, tolerance=1e-12))
        res[name + "_xr"] = r.x
        res[name + "_status"] = np.array(status(s))
    np.savez(out, **res)


if __name__ == "__main__":
    main(sys.argv[1])
