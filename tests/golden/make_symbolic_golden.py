"""Writes tests/golden/symbolic.npz: the symbolic analysis (ordering, final
elimination tree, fundamental and relaxed supernodes with their row
patterns) of small instances of the benchmark configurations, as computed by
the host analysis at the time the file was made. tests/test_symbolic_golden.py
checks the analysis against it bit for bit, so a rewrite of the analysis for
speed must reproduce it exactly (the analysis is a restatement of the
reference's symbolic.hpp, elimination_tree.hpp and ordering.hpp, whose exact
outputs the GPU factorization's parity depends on).

Run from the repository root: python tests/golden/make_symbolic_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ma57_b200 import OrderingType, SymLDLT  # noqa: E402
from ma57_b200 import matrices as M  # noqa: E402

CASES = {
    "config1_k10_amd": (lambda: M.config1(10)[0], OrderingType.AMD),
    "config1_k10_metis": (lambda: M.config1(10)[0], OrderingType.Metis),
    "config3_k12_metis": (lambda: M.config3(12, nrhs=1)[0], OrderingType.Metis),
    "config3_k12_natural": (lambda: M.config3(12, nrhs=1)[0], OrderingType.Natural),
    "config2_kkt_amd": (lambda: M.config2(grid=12, n2=60)[0], OrderingType.AMD),
}


def analysis_arrays(A, ordering):
    s = SymLDLT()
    s.setOrdering(ordering)
    s.analyzePattern(A)
    sf = s.symbolicFactor()

    def pack(sns):
        first = np.array([x.firstCol for x in sns], np.int32)
        ncols = np.array([x.ncols for x in sns], np.int32)
        ptr = np.zeros(len(sns) + 1, np.int64)
        ptr[1:] = np.cumsum([len(x.rowPattern) for x in sns])
        rows = np.concatenate([np.asarray(x.rowPattern, np.int32) for x in sns]) if sns else np.zeros(0, np.int32)
        return first, ncols, ptr, rows

    out = {"perm": np.asarray(sf.perm, np.int32), "parent": np.asarray(sf.etree.parent, np.int32),
           "colcount": np.asarray(sf.etree.colCount, np.int32)}
    for tag, sns in (("sn", sf.supernodes), ("fsn", sf.fundamentalSupernodes)):
        first, ncols, ptr, rows = pack(sns)
        out[f"{tag}_first"], out[f"{tag}_ncols"], out[f"{tag}_ptr"], out[f"{tag}_rows"] = first, ncols, ptr, rows
    return out


def main():
    arrays = {}
    for name, (make, ordering) in CASES.items():
        for k, v in analysis_arrays(make(), ordering).items():
            arrays[f"{name}/{k}"] = v
    path = os.path.join(ROOT, "tests", "golden", "symbolic.npz")
    np.savez_compressed(path, **arrays)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
