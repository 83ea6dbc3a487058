"""ORACLE -- test infrastructure only.

ctypes wrapper over ``oracle/_build/liboracle.so`` exposing the reference's
``SymLDLT`` API (solver.hpp:29-418) on top of the CPU restatement. The
symbolic analysis it consumes is the host analysis shared with the GPU path
(the permutation and supernodes must be identical for both).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
_lib = None
_i, _d, _p = C.c_int, C.c_double, C.c_void_p
_pi, _pd = C.POINTER(C.c_int), C.POINTER(C.c_double)


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        lib = C.CDLL(str(LIB_PATH))
        sigs = {
            "oracle_solver_create": (_p, [_i, _pi, _pi, _i, _pi, _pi, _pi, _pi]),
            "oracle_solver_destroy": (None, [_p]),
            "oracle_set": (_i, [_p, C.c_char_p, _d]),
            "oracle_set_kkt": (_i, [_p, _i, _i]),
            "oracle_set_signs": (_i, [_p, _i, _pi]),
            "oracle_factorize": (_i, [_p, _i, _pi, _pi, _pd, C.c_char_p, _i]),
            "oracle_info": (None, [_p, _pi, _pd]),
            "oracle_singular_cols": (_i, [_p, _pi]),
            "oracle_attempts": (_i, [_p, _pd, _pi, _i]),
            "oracle_solve": (_i, [_p, _pd, _i, _i, _pd, C.c_char_p, _i]),
            "oracle_refine": (_i, [_p, _i, _pi, _pi, _pd, _pd, _i, _pd, _i, _d, _pi, _pd, _pd, C.c_char_p, _i]),
            "oracle_front_sizes": (None, [_p, _pi, _pi]),
            "oracle_front_get": (_i, [_p, _i, _pi, _pd, _pd, _pd, _pi, _pi]),
            "oracle_dense_factor": (_i, [_i, _pd, _i, _i, _i, _d, _d, _i, _d, _d, _d, _pi, _i, _pi, _pd, _pd, _pi,
                                         _pi, _pi, _pd, C.c_char_p, _i]),
            "oracle_analyze": (_p, [_i, _pi, _pi, _i, _i, _d, C.c_char_p, _i]),
            "oracle_analysis_sizes": (None, [_p, _pi, _pi, C.POINTER(C.c_longlong)]),
            "oracle_analysis_get": (None, [_p, _pi, _pi, _pi, _pi, _pi, _pi]),
            "oracle_analysis_destroy": (None, [_p]),
        }
        for k, (r, a) in sigs.items():
            f = getattr(lib, k)
            f.restype = r
            f.argtypes = a
        _lib = lib
    return _lib


def _pi_(a):
    return a.ctypes.data_as(_pi)


def _pd_(a):
    return a.ctypes.data_as(_pd)


class OracleError(Exception):
    pass


class _Supernode:
    def __init__(self, first, ncols, rows):
        self.firstCol, self.ncols, self.rowPattern = first, ncols, rows


class _Etree:
    def __init__(self, parent):
        self.parent = parent
        self.n = len(parent)


class OracleAnalysis:
    """The host symbolic analysis as compiled into the oracle library (same
    sources as the GPU path's host side): perm, etree.parent and the
    supernodes, in the shape OracleSymLDLT takes."""

    def __init__(self, perm, parent, supernodes):
        self.perm = perm
        self.etree = _Etree(parent)
        self.supernodes = supernodes


def analyze(A, ordering=0, max_relax_size=64, max_relax_fill_fraction=0.25) -> OracleAnalysis:
    """SymbolicFactor::analyze (symbolic.hpp:195-399) without the product
    library: ordering 0 AMD, 1 METIS, 2 natural, 3 METIS in the reference's
    convention."""
    from ma57_b200.solver import as_csc
    n, cp, ri, _ = as_csc(A)
    lib = load()
    err = C.create_string_buffer(512)
    h = lib.oracle_analyze(n, _pi_(cp), _pi_(ri), int(ordering), max_relax_size, max_relax_fill_fraction, err, 512)
    if not h:
        raise RuntimeError(err.value.decode())
    try:
        nn, ns, pl = C.c_int(), C.c_int(), C.c_longlong()
        lib.oracle_analysis_sizes(h, C.byref(nn), C.byref(ns), C.byref(pl))
        perm = np.zeros(max(1, nn.value), np.int32)
        par = np.zeros(max(1, nn.value), np.int32)
        first = np.zeros(max(1, ns.value), np.int32)
        ncols = np.zeros(max(1, ns.value), np.int32)
        ptr = np.zeros(ns.value + 1, np.int32)
        rows = np.zeros(max(1, pl.value), np.int32)
        lib.oracle_analysis_get(h, _pi_(perm), _pi_(par), _pi_(first), _pi_(ncols), _pi_(ptr), _pi_(rows))
    finally:
        lib.oracle_analysis_destroy(h)
    sns = [_Supernode(int(first[i]), int(ncols[i]), rows[ptr[i]:ptr[i + 1]].copy()) for i in range(ns.value)]
    return OracleAnalysis(perm[:nn.value].copy(), par[:nn.value].copy(), sns)


def _raise(code, msg):
    from ma57_b200.solver import InvalidArgument, LogicError
    if code == 1:
        raise LogicError(msg)
    if code == 2:
        raise InvalidArgument(msg)
    if code == 3:
        raise RuntimeError(msg)
    raise OracleError(msg)


def dense_factor(A, n_eligible=-1, static=False, zero_tolerance=1e-300, relative_pivot_floor=1e-12, panel_size=64,
                 delta=0.0, static_rel_floor=1e-8, static_abs_floor=1e-300, expected_sign=None):
    """DenseLDLT::factor / factorStatic on a dense copy of A (lower read).
    Returns (A_factored, result dict)."""
    lib = load()
    A = np.array(A, dtype=np.float64, order="F", copy=True)
    n = A.shape[0]
    perm = np.zeros(max(1, n), np.int32)
    dd = np.zeros(max(1, n))
    do = np.zeros(max(1, n))
    ps = np.zeros(max(1, n), np.int32)
    pk = np.zeros(max(1, n), np.int32)
    ints = np.zeros(6, np.int32)
    dbls = np.zeros(2)
    sg = np.ascontiguousarray(expected_sign if expected_sign is not None else np.zeros(1), dtype=np.int32)
    nsg = 0 if expected_sign is None else len(sg)
    err = C.create_string_buffer(512)
    rc = lib.oracle_dense_factor(n, _pd_(A), n, n_eligible, 1 if static else 0, zero_tolerance, relative_pivot_floor,
                                 panel_size, delta, static_rel_floor, static_abs_floor, _pi_(sg), nsg, _pi_(perm),
                                 _pd_(dd), _pd_(do), _pi_(ps), _pi_(pk), _pi_(ints), _pd_(dbls), err, 512)
    if rc:
        _raise(rc, err.value.decode())
    nb = int(ints[4])
    res = dict(n_factored=int(ints[0]), inertia=(int(ints[1]), int(ints[2]), int(ints[3])), perm=perm[:n].copy(),
               Ddiag=dd[:n].copy(), Doff=do[:n].copy(), pivots=[(int(ps[b]), int(pk[b])) for b in range(nb)],
               num_perturbed=int(ints[5]), max_growth=float(dbls[0]), total_perturbation=float(dbls[1]))
    res["delayed_cols"] = list(range(res["n_factored"], n if n_eligible < 0 else n_eligible))
    return A, res


class OracleSymLDLT:
    """Reference SymLDLT semantics on the CPU (factorize, solve, refine, retry loop)."""

    def __init__(self, symbolic):
        lib = load()
        sf = symbolic
        n = len(sf.perm)
        first = np.array([s.firstCol for s in sf.supernodes], np.int32)
        ncol = np.array([s.ncols for s in sf.supernodes], np.int32)
        lens = [len(s.rowPattern) for s in sf.supernodes]
        ptr = np.zeros(len(lens) + 1, np.int32)
        ptr[1:] = np.cumsum(lens)
        rows = (np.concatenate([s.rowPattern for s in sf.supernodes]).astype(np.int32) if lens
                else np.zeros(1, np.int32))
        perm = np.ascontiguousarray(sf.perm, np.int32)
        par = np.ascontiguousarray(sf.etree.parent, np.int32)
        if n == 0:
            perm = par = np.zeros(1, np.int32)
        if len(first) == 0:
            first = ncol = np.zeros(1, np.int32)
        self.h = lib.oracle_solver_create(n, _pi_(perm), _pi_(par), len(lens), _pi_(first), _pi_(ncol), _pi_(ptr),
                                          _pi_(rows))
        self.n = n
        self.perm = np.asarray(sf.perm)

    def __del__(self):
        try:
            load().oracle_solver_destroy(self.h)
        except Exception:
            pass

    def set(self, **kw):
        for k, v in kw.items():
            if load().oracle_set(self.h, k.encode(), float(v)) != 0:
                raise KeyError(k)

    def setKKTBlockSizes(self, n1, n2):
        load().oracle_set_kkt(self.h, n1, n2)

    def setExpectedSignPattern(self, signs):
        s = np.ascontiguousarray(signs, np.int32)
        load().oracle_set_signs(self.h, len(s), _pi_(s))

    def factorize(self, A):
        from ma57_b200.solver import as_csc
        n, cp, ri, v = as_csc(A)
        err = C.create_string_buffer(1024)
        rc = load().oracle_factorize(self.h, n, _pi_(cp), _pi_(ri), _pd_(v), err, 1024)
        if rc:
            _raise(rc, err.value.decode())

    def info(self):
        ints = np.zeros(10, np.int32)
        dbls = np.zeros(2)
        load().oracle_info(self.h, _pi_(ints), _pd_(dbls))
        keys = ["n_pos", "n_neg", "n_zero", "singular", "n_singular", "retries", "num_perturbed", "num_delayed",
                "factorized", "num_fronts"]
        d = {k: int(x) for k, x in zip(keys, ints)}
        d["last_delta"] = float(dbls[0])
        d["total_perturbation"] = float(dbls[1])
        return d

    def inertia(self):
        i = self.info()
        return (i["n_pos"], i["n_neg"], i["n_zero"])

    def singularColumns(self):
        i = self.info()
        out = np.zeros(max(1, i["n_singular"]), np.int32)
        k = load().oracle_singular_cols(self.h, _pi_(out))
        return [int(self.perm[c]) for c in out[:k]]

    def attempts(self):
        d = np.zeros(64)
        ok = np.zeros(64, np.int32)
        k = load().oracle_attempts(self.h, _pd_(d), _pi_(ok), 64)
        return list(d[:k]), list(ok[:k])

    def solve(self, B):
        B = np.asarray(B, np.float64)
        vec = B.ndim == 1
        Bf = np.asfortranarray(B.reshape(-1, 1) if vec else B)
        X = np.zeros_like(Bf, order="F")
        err = C.create_string_buffer(1024)
        rc = load().oracle_solve(self.h, _pd_(Bf), Bf.shape[0], Bf.shape[1], _pd_(X), err, 1024)
        if rc:
            _raise(rc, err.value.decode())
        return X[:, 0] if vec else X

    def solveWithRefinement(self, A, B, max_iterations=10, tolerance=1e-14):
        from ma57_b200.solver import as_csc
        n, cp, ri, v = as_csc(A)
        B = np.asarray(B, np.float64)
        vec = B.ndim == 1
        Bf = np.asfortranarray(B.reshape(-1, 1) if vec else B)
        X = np.zeros_like(Bf, order="F")
        it = C.c_int()
        r0 = C.c_double()
        r1 = C.c_double()
        err = C.create_string_buffer(1024)
        rc = load().oracle_refine(self.h, n, _pi_(cp), _pi_(ri), _pd_(v), _pd_(Bf), Bf.shape[1], _pd_(X),
                                  max_iterations, tolerance, C.byref(it), C.byref(r0), C.byref(r1), err, 1024)
        if rc:
            _raise(rc, err.value.decode())
        return (X[:, 0] if vec else X), dict(iterations=it.value, initial=r0.value, final=r1.value)

    def fronts(self):
        i = self.info()
        nf = i["num_fronts"]
        m = np.zeros(max(1, nf), np.int32)
        npv = np.zeros(max(1, nf), np.int32)
        load().oracle_front_sizes(self.h, _pi_(m), _pi_(npv))
        out = []
        for si in range(nf):
            mm, kk = int(m[si]), int(npv[si])
            rows = np.zeros(max(1, mm), np.int32)
            Lm = np.zeros((mm, kk), order="F")
            dd = np.zeros(max(1, kk))
            do = np.zeros(max(1, kk))
            ps = np.zeros(max(1, kk), np.int32)
            pk = np.zeros(max(1, kk), np.int32)
            nb = load().oracle_front_get(self.h, si, _pi_(rows), _pd_(Lm) if kk else _pd_(dd), _pd_(dd), _pd_(do),
                                         _pi_(ps), _pi_(pk))
            out.append(dict(rowIndices=rows[:mm].copy(), nPivots=kk, L=Lm, Ddiag=dd[:kk].copy(), Doff=do[:kk].copy(),
                            pivotBlocks=[(int(ps[b]), int(pk[b])) for b in range(nb)]))
        return out
