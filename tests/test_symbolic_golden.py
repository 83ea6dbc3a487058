"""The host symbolic analysis against the committed golden fixture
(tests/golden/symbolic.npz, made by tests/golden/make_symbolic_golden.py):
ordering, final elimination tree, fundamental and relaxed supernodes and
their row patterns, bit for bit. Runs on the CPU."""
import importlib.util
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
_spec = importlib.util.spec_from_file_location("make_symbolic_golden",
                                               os.path.join(HERE, "golden", "make_symbolic_golden.py"))
G = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(G)
GOLDEN = np.load(os.path.join(HERE, "golden", "symbolic.npz"))


@pytest.mark.parametrize("name", sorted(G.CASES))
def test_symbolic_analysis_matches_golden(name):
    make, ordering = G.CASES[name]
    got = G.analysis_arrays(make(), ordering)
    keys = sorted(k.split("/", 1)[1] for k in GOLDEN.files if k.startswith(name + "/"))
    assert keys == sorted(got)
    for k in keys:
        np.testing.assert_array_equal(got[k], GOLDEN[f"{name}/{k}"], err_msg=f"{name}: {k}")
