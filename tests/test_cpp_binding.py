"""The C++ binding (include/symla_gpu_backend.hpp) compiled and run the way
symla's SymLDLT<double> would use it: tests/cpp/backend_test.cpp drives
analyzePattern -> import of the reference's SymbolicFactor -> factorize ->
solve -> solveWithRefinement on L7(20^3) - 2I against Eigen-free stand-ins of
the reference's types, and checks the inertia (7590, 410, 0) and the error
mapping onto the reference's exceptions."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "backend_test.cpp")
OUT = os.path.join(ROOT, "tests", "cpp", "_build", "backend_test")
LIBDIR = os.path.join(ROOT, "ma57_b200", "lib")


def build():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-o", OUT, "-L", LIBDIR, "-lsymla_b200", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return OUT


def test_binding_compiles_against_the_reference_shaped_types():
    assert os.path.exists(build())


@pytest.mark.gpu
def test_binding_factorizes_and_solves_config1():
    exe = build()
    r = subprocess.run([exe, "20"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "inertia=(7590,410,0)" in r.stdout
    assert "backend_test OK" in r.stdout
