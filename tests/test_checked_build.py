"""The bounds-checked build (libsymla_b200_checked.so, -DSYMLA_GPU_CHECKED):
the library compiled with a check before every table-indexed access and a
validation of the device tables around every factorization and solve, each
failure recorded in a device status word instead of trapping.

CPU: the library is built, exports every declared entry point and reports
itself as checked; the predicates the checks use (ma57_b200/csrc/gpu/
checked.cuh) are compiled for the host and run against planted bad tables.
GPU: the same factorizations and solves (the delayed-pivot arrow, which
re-plans a front; config 1; the 27-point stencil in FP64 and mixed precision;
a KKT system in threshold and StaticRegularized mode) run through both
builds: no check fails, and the results are bit-identical."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from ma57_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORKER = os.path.join(ROOT, "tests", "checked_worker.py")
PRED_SRC = os.path.join(ROOT, "tests", "cpp", "check_predicates_test.cpp")
PRED_OUT = os.path.join(ROOT, "tests", "cpp", "_build", "check_predicates_test")


def _open(path):
    return C.CDLL(str(path), mode=os.RTLD_NOW | os.RTLD_LOCAL)


def test_checked_library_exports_every_entry_point():
    assert L.CHECKED_LIB_PATH.exists(), "run __graft_entry__.build()"
    lib = _open(L.CHECKED_LIB_PATH)
    for name in L.EXPORTED:
        assert hasattr(lib, name), name
    lib.symla_gpu_checked_build.restype = C.c_int
    assert lib.symla_gpu_checked_build() == 1
    prod = _open(L.PRODUCT_LIB_PATH)
    prod.symla_gpu_checked_build.restype = C.c_int
    assert prod.symla_gpu_checked_build() == 0


def test_library_selection_by_environment():
    code = "from ma57_b200 import _lib as L; print(L.LIB_PATH.name, L.load().symla_gpu_checked_build())"
    for choice, want in (("", "libsymla_b200.so 0"), ("checked", "libsymla_b200_checked.so 1")):
        env = dict(os.environ, SYMLA_GPU_LIBRARY=choice)
        r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert r.stdout.split() == want.split()


def test_check_predicates_catch_planted_bad_tables():
    os.makedirs(os.path.dirname(PRED_OUT), exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "ma57_b200", "csrc", "gpu"),
           "-I", "/usr/local/cuda/include", PRED_SRC, "-o", PRED_OUT]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    r = subprocess.run([PRED_OUT], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "check_predicates OK" in r.stdout


def _run_worker(choice, tmp_path):
    out = tmp_path / f"{choice or 'product'}.npz"
    env = dict(os.environ, SYMLA_GPU_LIBRARY=choice)
    r = subprocess.run([sys.executable, WORKER, str(out)], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return dict(np.load(out))


@pytest.mark.gpu
def test_checked_build_passes_and_matches_the_ordinary_build(tmp_path):
    chk = _run_worker("checked", tmp_path)
    prod = _run_worker("", tmp_path)
    assert int(chk["checked_build"]) == 1 and int(prod["checked_build"]) == 0
    assert int(chk["arrow_dynamic"]) == 1  # the re-planned (delayed-pivot) path ran under the checks
    assert chk["arrow_npiv"].tolist() == [0, 0, 5]
    for key in chk:
        if key.endswith("_status"):
            assert chk[key].tolist() == [0, 0, 0], (key, chk[key])
        elif key != "checked_build":
            np.testing.assert_array_equal(chk[key], prod[key], err_msg=key)
