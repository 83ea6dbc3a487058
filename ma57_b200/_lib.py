"""ctypes binding of ``lib/libsymla_b200.so`` (declared in include/symla_gpu.h).

The library is required: importing this module fails loudly when it is
missing, and every device entry point reports an error (no CPU fallback)
when no CUDA device is present. With SYMLA_GPU_LIBRARY=checked in the
environment the process loads the bounds-checked build,
``lib/libsymla_b200_checked.so`` (same entry points); any other value is
taken as the path of the library to load.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "lib"
PRODUCT_LIB_PATH = LIB_DIR / "libsymla_b200.so"
CHECKED_LIB_PATH = LIB_DIR / "libsymla_b200_checked.so"


def library_path() -> Path:
    """The library this process loads (see the module docstring)."""
    choice = os.environ.get("SYMLA_GPU_LIBRARY", "")
    if not choice:
        return PRODUCT_LIB_PATH
    if choice == "checked":
        return CHECKED_LIB_PATH
    return Path(choice)


LIB_PATH = library_path()

SYMLA_OK = 0
SYMLA_ERR_NOT_ANALYZED = 1
SYMLA_ERR_NOT_FACTORIZED = 2
SYMLA_ERR_SINGULAR = 3
SYMLA_ERR_BAD_SIZE = 4
SYMLA_ERR_RETRY_EXHAUSTED = 5
SYMLA_ERR_OOM = 6
SYMLA_ERR_TIMEOUT = 7
SYMLA_ERR_CUDA = 8
SYMLA_ERR_INVALID = 9
SYMLA_ERR_NO_DEVICE = 10
SYMLA_ERR_INTERNAL = 11

MODE_THRESHOLD = 0
MODE_STATIC = 1
PREC_FP64 = 0
PREC_MIXED = 1

_i = C.c_int
_d = C.c_double
_p = C.c_void_p
_pi = C.POINTER(C.c_int)
_pd = C.POINTER(C.c_double)
_pf = C.POINTER(C.c_float)


class SymbolicInfo(C.Structure):
    _fields_ = [("n", _i), ("num_supernodes", _i), ("num_fundamental", _i), ("pattern_len", C.c_int64),
                ("fundamental_len", C.c_int64), ("storage_nnz", C.c_int64)]


class FactorOpts(C.Structure):
    _fields_ = [("mode", _i), ("precision", _i), ("pivot_threshold", _d), ("zero_tolerance", _d),
                ("relative_pivot_floor", _d), ("static_delta", _d), ("static_rel_floor", _d),
                ("static_abs_floor", _d), ("expected_sign", _pi), ("front_delta", _pd)]


class FactorInfo(C.Structure):
    _fields_ = [("n_pos", _i), ("n_neg", _i), ("n_zero", _i), ("singular", _i), ("n_singular", _i),
                ("num_perturbed", _i), ("total_perturbation", _d), ("num_delayed", _i),
                ("used_dynamic_path", _i), ("max_growth", _d), ("factor_ms", C.c_float)]


class RegularizeOpts(C.Structure):
    _fields_ = [("initial_delta", _d), ("max_retries", _i), ("growth", _d), ("static_rel_floor", _d),
                ("static_abs_floor", _d), ("expected_sign", _pi), ("kkt_n1", _i), ("kkt_n2", _i),
                ("precision", _i), ("front_delta", _pd)]


class RegularizeInfo(C.Structure):
    _fields_ = [("retries_used", _i), ("last_delta", _d), ("attempts", _i), ("attempt_delta", _d * 32),
                ("attempt_ok", _i * 32)]


class RefineInfo(C.Structure):
    _fields_ = [("iterations", _i), ("initial_relative_residual", _d), ("final_relative_residual", _d)]


class GmresInfo(C.Structure):
    _fields_ = [("outer_iterations", _i), ("inner_iterations", _i), ("initial_relative_residual", _d),
                ("final_relative_residual", _d)]


_SIGS = {
    "symla_last_error": (C.c_char_p, []),
    "symla_analyze": (_i, [_i, _pi, _pi, _i, _i, _d, C.POINTER(_p)]),
    "symla_symbolic_destroy": (None, [_p]),
    "symla_compute_ordering": (_i, [_i, _pi, _pi, _i, _pi]),
    "symla_symbolic_get_info": (_i, [_p, C.POINTER(SymbolicInfo)]),
    "symla_symbolic_get": (_i, [_p, _pi, _pi, _pi, _pi, _pi, _pi, _pi]),
    "symla_symbolic_get_fundamental": (_i, [_p, _pi, _pi, _pi, _pi]),
    "symla_symbolic_import": (_i, [_i, _pi, _pi, _i, _pi, _pi, _pi, _pi, C.POINTER(_p)]),
    "symla_gpu_create": (_i, [_p, _i, _pi, _pi, _i, C.POINTER(_p)]),
    "symla_gpu_destroy": (None, [_p]),
    "symla_factor_opts_default": (None, [C.POINTER(FactorOpts)]),
    "symla_gpu_factorize": (_i, [_p, _pd, _i, C.POINTER(FactorOpts), C.POINTER(FactorInfo)]),
    "symla_regularize_opts_default": (None, [C.POINTER(RegularizeOpts)]),
    "symla_gpu_factorize_regularized": (_i, [_p, _pd, _i, C.POINTER(RegularizeOpts), C.POINTER(FactorInfo),
                                             C.POINTER(RegularizeInfo)]),
    "symla_gpu_solve": (_i, [_p, _pd, _i, _i, _pd, _i, _i]),
    "symla_gpu_solve_refine": (_i, [_p, _pd, _pd, _i, _i, _pd, _i, _i, _i, _d, C.POINTER(RefineInfo)]),
    "symla_gpu_solve_gmres_refine": (_i, [_p, _pd, _pd, _i, _i, _pd, _i, _i, _i, _i, _d, C.POINTER(GmresInfo)]),
    "symla_gpu_singular_cols": (_i, [_p, _pi, _i]),
    "symla_gpu_num_fronts": (_i, [_p]),
    "symla_gpu_front_size": (_i, [_p, _i, _pi, _pi]),
    "symla_gpu_front_get": (_i, [_p, _i, _pi, _pd, _pd, _pd, _pi, _pi]),
    "symla_gpu_stream": (_p, [_p]),
    "symla_gpu_phase_ms": (_i, [_p, _pf, _i]),
    "symla_gpu_plan_stats": (_i, [_p, _pd, _i]),
    "symla_gpu_set_profiling": (_i, [_p, _i]),
    "symla_gpu_set_graph": (_i, [_p, _i]),
    "symla_gpu_level_info": (_i, [_p, _i, _pi]),
    "symla_gpu_set_level_schedule": (_i, [_p, _i, _i, _i]),
    "symla_gpu_set_level_update_rows": (_i, [_p, _i, _i]),
    "symla_gpu_level_update_rows": (_i, [_p, _i, _pi]),
    "symla_gpu_graph_stats": (_i, [_p, _pi, _pi]),
    "symla_gpu_kernel_stats": (_i, [_p, _i, _pd]),
    "symla_gpu_level_kernel_stats": (_i, [_p, _i, _i, _pd]),
    "symla_gpu_level_panel_stats": (_i, [_p, _i, C.POINTER(C.c_longlong)]),
    "symla_gpu_reset_kernel_stats": (None, [_p]),
    "symla_gpu_launch_count": (C.c_longlong, [_p]),
    "symla_gpu_set_wait_limit_ns": (_i, [_p, C.c_ulonglong]),
    "symla_gpu_set_memory_limit": (_i, [C.c_longlong]),
    "symla_gpu_relative_residual_noalloc": (_i, [_p, _p, _i, _p, _i, _i, _pd]),
    "symla_gpu_checked_build": (_i, []),
    "symla_gpu_check_status": (_i, [_p, _pi, _pi, C.POINTER(C.c_longlong)]),
    "symla_mlp_create": (_i, [_i, _pd, C.POINTER(_p)]),
    "symla_mlp_destroy": (None, [_p]),
    "symla_mlp_get_params": (_i, [_p, _pd]),
    "symla_mlp_predict": (_i, [_p, _pd, _i, _pd]),
    "symla_mlp_gradient": (_i, [_p, _pd, _pd, _i, _pd, _pd]),
    "symla_mlp_train": (_i, [_p, _pd, _pd, _i, _i, _i, _d, _pd]),
}

MLP_INPUTS = 8
MLP_HIDDEN = 32
MLP_PARAMS = MLP_HIDDEN * MLP_INPUTS + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_HIDDEN + 1

NOALLOC_RESIDUAL_MAX_ENTRIES = 1 << 20

KERNEL_KINDS = ["far_update", "panel", "small", "assemble", "forward", "backward", "residual", "near_update"]

# Every symbol declared in include/symla_gpu.h that is a function.
EXPORTED = tuple(_SIGS.keys())

_lib = None


def load() -> C.CDLL:
    """Load the native library (raises ImportError when it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"ma57_b200 native library not built: {LIB_PATH} (run __graft_entry__.build())")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    msg = load().symla_last_error()
    return msg.decode() if msg else ""


def ptr_i(a):
    return a.ctypes.data_as(_pi) if a is not None else None


def ptr_d(a):
    return a.ctypes.data_as(_pd) if a is not None else None
