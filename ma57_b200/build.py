"""Build recipe for the native library ``ma57_b200/lib/libsymla_b200.so``.

Compiles the host symbolic analysis (C++17, g++) and the sm_100a CUDA kernels
plus the C ABI (nvcc, ``-gencode arch=compute_100a,code=sm_100a``), and links
them with the CUDA toolkit's static METIS into one shared library. The built
library stays in-tree so that it travels with the repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libsymla_b200.so"
CHECKED_LIB = LIBDIR / "libsymla_b200_checked.so"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

HOST_SRCS = ["host/symbolic.cpp", "host/amd.cpp", "host/metis_order.cpp"]
CUDA_SRCS = ["gpu/capi.cu", "gpu/factor_kernels.cu", "gpu/solve_kernels.cu", "gpu/panel_cluster.cu", "gpu/schur_tc.cu", "gpu/noalloc.cu", "gpu/mlp.cu"]
# benchmark tooling, its own library (bench.py loads it; not part of the C ABI)
BENCH_SRC = "bench/fp64_peak.cu"
BENCH_LIB = LIBDIR / "libsymla_bench.so"


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _headers() -> list[Path]:
    hs = list(CSRC.rglob("*.h")) + list(CSRC.rglob("*.hpp")) + list(CSRC.rglob("*.cuh"))
    hs.append(PKG.parent / "include" / "symla_gpu.h")
    return hs


def _build_library(lib: Path, objdir: Path, defines: list[str], verbose: bool, force: bool) -> None:
    objdir.mkdir(parents=True, exist_ok=True)
    hdrs = _headers()
    objs: list[Path] = []
    for src in HOST_SRCS:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")  # host code is the same in both builds
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            _run(["g++", "-std=c++17", "-O3", "-fPIC", "-Wall", "-c", str(s), "-o", str(o)])
    for src in CUDA_SRCS:
        s = CSRC / src
        o = objdir / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [NVCC, *ARCH, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", *defines, "-c", str(s), "-o", str(o)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
    metis = CUDA_HOME / "lib64" / "libmetis_static.a"
    if force or _stale(lib, objs):
        # --no-undefined: a missing symbol fails the build, not the first dlopen
        _run([NVCC, *ARCH, "-shared", "-o", str(lib), *map(str, objs), str(metis), "-lcudart_static",
              "-Xlinker", "--no-undefined"])


def build(verbose: bool = False, force: bool = False, checked: bool = True) -> Path:
    """Compile every source that changed and link the shared library, and
    (checked=True) its bounds-checked variant (-DSYMLA_GPU_CHECKED)."""
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    _build_library(LIB, BUILD, [], verbose, force)
    if checked:
        _build_library(CHECKED_LIB, BUILD / "checked", ["-DSYMLA_GPU_CHECKED"], verbose, force)
    bsrc = CSRC / BENCH_SRC
    bobj = BUILD / "fp64_peak.o"
    if force or _stale(bobj, [bsrc]):
        _run([NVCC, *ARCH, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-c", str(bsrc), "-o", str(bobj)])
    if force or _stale(BENCH_LIB, [bobj]):
        _run([NVCC, *ARCH, "-shared", "-o", str(BENCH_LIB), str(bobj), "-lcudart_static", "-Xlinker", "--no-undefined"])
    return LIB


def clean() -> None:
    shutil.rmtree(BUILD, ignore_errors=True)
    for lib in (LIB, CHECKED_LIB):
        if lib.exists():
            lib.unlink()


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
