"""Writes tests/golden/oracle_config2.json: the oracle's (CPU restatement of
the reference's numeric path) results on the KKT saddle-point system at its
full benchmark size, which the oracle needs about ten minutes of CPU to
produce:

  K = [[-E, A^T], [A, F]], E = L5(200^2) + 1e-2 I (n1 = 40000), A 20000 x 40000
  with 3 N(0,1) entries per row, F = 1e-8 I (n2 = 20000); n = 60000.
  Mode::StaticRegularized with setKKTBlockSizes(40000, 20000), AMD ordering,
  b ~ N(0,1), solveWithRefinement to backward error 1e-12
  (kkt_static_pivoting_test.cpp:128-167 is the reference's test of this mode).

tests/test_config_parity.py compares the GPU path with these numbers:
identical inertia and retry count, backward error within 10x of the
oracle's. A fingerprint of the matrix and of its symbolic analysis is stored
beside them, so a change of the generator or of the analysis shows up as a
fixture mismatch rather than as a parity failure.

Run from the repository root: python tests/golden/make_oracle_golden.py
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ma57_b200 import OrderingType, SymLDLT  # noqa: E402
from ma57_b200 import matrices as M  # noqa: E402
from ma57_b200.solver import as_csc  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "oracle_config2.json")


def fingerprint(A):
    """sha256 of the CSC pattern and values (lower triangle as generated)."""
    n, cp, ri, v = as_csc(A)
    h = hashlib.sha256()
    for a in (np.int64(n), cp, ri, v):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def symbolic_summary(sf):
    ms = [len(s.rowPattern) for s in sf.supernodes]
    return {"num_supernodes": len(ms), "max_front": max(ms), "sum_m": int(sum(ms)),
            "storage_nnz": int(sum(s.storageNnz() for s in sf.supernodes))}


def backward_error(A, x, b):
    """||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf), ||A|| as the
    stored-entry row sums (refine.hpp:69-81, :109-114)."""
    r = b - M.sym_full(A) @ x
    normA = abs(A).sum(axis=1).max()
    return float(np.abs(r).max() / (normA * np.abs(x).max() + np.abs(b).max()))


def config2_case():
    from oracle.pyoracle import OracleSymLDLT
    K, b, n1, n2 = M.config2()
    s = SymLDLT()
    s.setOrdering(OrderingType.AMD)
    s.analyzePattern(K)
    sf = s.symbolicFactor()
    o = OracleSymLDLT(sf)
    o.set(mode=1, parallel=1, num_threads=os.cpu_count() or 1)
    o.setKKTBlockSizes(n1, n2)
    t0 = time.perf_counter()
    o.factorize(K)
    t_factor = time.perf_counter() - t0
    info = o.info()
    x0 = o.solve(b)
    x, d = o.solveWithRefinement(K, b, max_iterations=10, tolerance=1e-12)
    return {
        "matrix": {"n": int(K.shape[0]), "n1": n1, "n2": n2, "nnz_lower": int(K.nnz), "sha256": fingerprint(K)},
        "symbolic": symbolic_summary(sf),
        "oracle": {"inertia": [info["n_pos"], info["n_neg"], info["n_zero"]], "retries": info["retries"],
                   "last_delta": info["last_delta"], "num_perturbed": info["num_perturbed"],
                   "total_perturbation": info["total_perturbation"],
                   "backward_error_unrefined": backward_error(K, x0, b),
                   "backward_error_refined": backward_error(K, x, b), "refine_iterations": d["iterations"],
                   "refine_final": d["final"], "factor_s": t_factor, "threads": os.cpu_count()},
    }


if __name__ == "__main__":
    out = {"config2": config2_case()}
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))
