"""Python mirror of ``symla::SymLDLT<double>`` (include/symla/solver.hpp:29-418)
over the B200 C ABI.

Same method names, argument meaning and error behaviour as the reference:
``analyzePattern`` / ``factorize`` / ``compute`` / ``refactorize`` / ``solve``
/ ``solveWithRefinement`` / ``inertia`` / ``isSingular`` /
``singularColumns``, ``Mode.StaticRegularized`` with ``setKKTBlockSizes``,
and the same exception classes (``LogicError`` for call-order violations,
``InvalidArgument`` for size mismatches, ``RuntimeError`` when the
regularization retry budget is exhausted).

Matrices are ``scipy.sparse`` matrices (converted to CSC with int32 indices,
the layout of ``Eigen::SparseMatrix<double, ColMajor, int>``); only the lower
triangle of the values is read.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


class LogicError(RuntimeError):
    """Mirror of std::logic_error."""


class InvalidArgument(ValueError):
    """Mirror of std::invalid_argument."""


class Mode(enum.IntEnum):
    ThresholdPivot = 0
    StaticRegularized = 1


class OrderingType(enum.IntEnum):
    """OrderingType (ordering.hpp:31-35). ``Metis`` is nested dissection in
    METIS's pivot order; ``MetisIperm`` takes METIS's inverse array, as the
    reference does (ordering.hpp:130-141), for bit-identical permutations."""
    AMD = 0
    Metis = 1
    Natural = 2
    MetisIperm = 3


class Precision(enum.IntEnum):
    """Arithmetic of the large fronts' Schur-complement updates."""
    FP64 = 0
    Mixed = 1


@dataclass
class Inertia:
    n_pos: int = 0
    n_neg: int = 0
    n_zero: int = 0

    def as_tuple(self):
        return (self.n_pos, self.n_neg, self.n_zero)


@dataclass
class SymbolicFactorOptions:
    max_relax_size: int = 64
    max_relax_fill_fraction: float = 0.25


@dataclass
class RefinementOptions:
    max_iterations: int = 10
    tolerance: float = 1e-14


@dataclass
class RefinementResult:
    iterations: int = 0
    initial_relative_residual: float = 0.0
    final_relative_residual: float = 0.0


@dataclass
class GmresRefinementOptions:
    """GMRES-IR (a B200 extension; the reference refines in fixed precision
    only, refine.hpp:52-57): outer iterations on the FP64 residual, each
    correction by GMRES with `restart` Krylov vectors preconditioned by the
    factorization."""
    max_outer: int = 10
    restart: int = 8
    tolerance: float = 1e-14


@dataclass
class GmresResult:
    outer_iterations: int = 0
    inner_iterations: int = 0
    initial_relative_residual: float = 0.0
    final_relative_residual: float = 0.0


@dataclass
class RefinedSolve:
    x: np.ndarray
    diagnostics: RefinementResult


@dataclass
class Supernode:
    firstCol: int
    ncols: int
    rowPattern: np.ndarray

    def storageNnz(self) -> int:
        m, k = len(self.rowPattern), self.ncols
        return k * m - k * (k - 1) // 2


@dataclass
class EliminationTree:
    parent: np.ndarray
    colCount: np.ndarray
    n: int


@dataclass
class SymbolicFactor:
    perm: np.ndarray
    etree: EliminationTree
    supernodes: list
    fundamentalSupernodes: list


@dataclass
class PivotBlock:
    start: int
    kind: int  # 0 = 1x1, 1 = 2x2


@dataclass
class SupernodeFactor:
    rowIndices: np.ndarray
    nPivots: int
    L: np.ndarray
    Ddiag: np.ndarray
    Doff: np.ndarray
    pivotBlocks: list


@dataclass
class NumericFactor:
    fronts: list
    perm: np.ndarray
    inertia: Inertia
    singular: bool
    singularCols: list
    n: int
    totalPerturbation: float = 0.0
    numPerturbed: int = 0


def as_csc(A):
    """CSC, sorted, int32 indices, float64 values (Eigen compressed layout)."""
    import scipy.sparse as sp
    A = sp.csc_matrix(A)
    A.sum_duplicates()
    A.sort_indices()
    if A.shape[0] != A.shape[1]:
        raise InvalidArgument("symla::ordering: matrix must be square")
    return (A.shape[0], np.ascontiguousarray(A.indptr, dtype=np.int32),
            np.ascontiguousarray(A.indices, dtype=np.int32), np.ascontiguousarray(A.data, dtype=np.float64))


def _check(rc: int):
    if rc == L.SYMLA_OK:
        return
    msg = L.last_error()
    if rc in (L.SYMLA_ERR_NOT_ANALYZED, L.SYMLA_ERR_NOT_FACTORIZED, L.SYMLA_ERR_SINGULAR):
        raise LogicError(msg)
    if rc in (L.SYMLA_ERR_BAD_SIZE, L.SYMLA_ERR_INVALID):
        raise InvalidArgument(msg)
    raise RuntimeError(f"{msg} (status {rc})")


def computeOrdering(A, ordering) -> np.ndarray:
    """symla::computeOrdering (ordering.hpp:84-149): perm[k] = original index
    of the k-th pivot, without the postorder that analyzePattern applies."""
    n, cp, ri, _ = as_csc(A)
    perm = np.zeros(max(1, n), np.int32)
    _check(L.load().symla_compute_ordering(n, L.ptr_i(cp), L.ptr_i(ri), int(OrderingType(ordering)), L.ptr_i(perm)))
    return perm[:n]


class Analysis:
    """Owns a host symbolic analysis handle (symla_analyze)."""

    def __init__(self, n, colptr, rowind, ordering, options: SymbolicFactorOptions):
        lib = L.load()
        h = C.c_void_p()
        _check(lib.symla_analyze(n, L.ptr_i(colptr), L.ptr_i(rowind), int(ordering), int(options.max_relax_size),
                                 float(options.max_relax_fill_fraction), C.byref(h)))
        self.h = h
        self.n = n
        self._sf = None

    def __del__(self):
        try:
            if self.h:
                L.load().symla_symbolic_destroy(self.h)
        except Exception:
            pass

    def perm(self) -> np.ndarray:
        """The final ordering alone (new -> original index), without
        building the supernode lists."""
        if self._sf is not None:
            return self._sf.perm
        lib = L.load()
        p = np.zeros(self.n, np.int32)
        _check(lib.symla_symbolic_get(self.h, L.ptr_i(p), None, None, None, None, None, None))
        return p

    def factor(self) -> SymbolicFactor:
        if self._sf is not None:
            return self._sf
        lib = L.load()
        info = L.SymbolicInfo()
        _check(lib.symla_symbolic_get_info(self.h, C.byref(info)))
        n, ns, nf = info.n, info.num_supernodes, info.num_fundamental
        perm = np.zeros(n, np.int32)
        par = np.zeros(n, np.int32)
        cc = np.zeros(n, np.int32)
        first = np.zeros(ns, np.int32)
        ncol = np.zeros(ns, np.int32)
        ptr = np.zeros(ns + 1, np.int32)
        rows = np.zeros(max(1, info.pattern_len), np.int32)
        _check(lib.symla_symbolic_get(self.h, L.ptr_i(perm), L.ptr_i(par), L.ptr_i(cc), L.ptr_i(first),
                                      L.ptr_i(ncol), L.ptr_i(ptr), L.ptr_i(rows)))
        sns = [Supernode(int(first[i]), int(ncol[i]), rows[ptr[i]:ptr[i + 1]].copy()) for i in range(ns)]
        f1 = np.zeros(nf, np.int32)
        f2 = np.zeros(nf, np.int32)
        fp = np.zeros(nf + 1, np.int32)
        fr = np.zeros(max(1, info.fundamental_len), np.int32)
        _check(lib.symla_symbolic_get_fundamental(self.h, L.ptr_i(f1), L.ptr_i(f2), L.ptr_i(fp), L.ptr_i(fr)))
        funda = [Supernode(int(f1[i]), int(f2[i]), fr[fp[i]:fp[i + 1]].copy()) for i in range(nf)]
        self._sf = SymbolicFactor(perm, EliminationTree(par, cc, n), sns, funda)
        return self._sf


class Context:
    """Owns a device context (symla_gpu_create) for one analysis + pattern."""

    def __init__(self, analysis: Analysis, colptr, rowind, device: int = 0):
        lib = L.load()
        h = C.c_void_p()
        self._colptr = colptr
        self._rowind = rowind
        _check(lib.symla_gpu_create(analysis.h, analysis.n, L.ptr_i(colptr), L.ptr_i(rowind), device, C.byref(h)))
        self.h = h
        self.n = analysis.n

    def __del__(self):
        try:
            if self.h:
                L.load().symla_gpu_destroy(self.h)
        except Exception:
            pass

    def same_pattern(self, colptr, rowind) -> bool:
        return (len(colptr) == len(self._colptr) and len(rowind) == len(self._rowind)
                and np.array_equal(colptr, self._colptr) and np.array_equal(rowind, self._rowind))


class SymLDLT:
    """B200 ``SymLDLT<double>``; see the module docstring."""

    def __init__(self, device: int = 0):
        self.device = device
        self.mode_ = Mode.ThresholdPivot
        self.pivot_threshold_ = 0.01
        self.ordering_ = OrderingType.AMD
        self.precision_ = Precision.FP64
        self.parallel_ = True
        self.num_threads_ = 0
        self.pattern_analyzed_ = False
        self.factorized_ = False
        self.inertia_ = Inertia()
        self.use_kkt_blocks_ = False
        self.kkt_n1_ = 0
        self.kkt_n2_ = 0
        self.use_explicit_signs_ = False
        self.expected_signs_orig_ = None
        self.initial_regularization_delta_ = 0.0
        self.max_regularization_retries_ = 10
        self.regularization_growth_ = 10.0
        self.static_pivot_relative_floor_ = 1e-8
        self.static_pivot_absolute_floor_ = 1e-300
        self.zero_tolerance_ = 1e-300
        self.relative_pivot_floor_ = 1e-12
        self.last_regularization_delta_ = 0.0
        self.regularization_retries_used_ = 0
        self.last_info = L.FactorInfo()
        self.last_reg_info = L.RegularizeInfo()
        self.front_delta_ = None
        self.graph_launch_ = False
        self._analysis = None
        self._ctx = None
        self._singular_cols = []
        self._numeric = None

    # --- configuration (solver.hpp:36-126) ---
    def setMode(self, mode):
        self.mode_ = Mode(mode)

    def setPivotThreshold(self, u):
        self.pivot_threshold_ = float(u)

    def setOrdering(self, ordering):
        self.ordering_ = OrderingType(ordering)

    def setPrecision(self, precision):
        self.precision_ = Precision(precision)

    def setKKTBlockSizes(self, n1, n2):
        if n1 < 0 or n2 < 0:
            raise InvalidArgument("symla::SymLDLT::setKKTBlockSizes: sizes must be nonnegative")
        self.kkt_n1_, self.kkt_n2_ = int(n1), int(n2)
        self.use_kkt_blocks_ = True
        self.use_explicit_signs_ = False

    def setExpectedSignPattern(self, signs):
        self.expected_signs_orig_ = np.ascontiguousarray(signs, dtype=np.int32)
        self.use_explicit_signs_ = True
        self.use_kkt_blocks_ = False

    def setInitialRegularizationDelta(self, delta):
        self.initial_regularization_delta_ = float(delta)

    def setMaxRegularizationRetries(self, retries):
        self.max_regularization_retries_ = int(retries)

    def setRegularizationGrowth(self, growth):
        self.regularization_growth_ = float(growth)

    def setStaticPivotFloor(self, relativeFloor, absoluteFloor=1e-300):
        self.static_pivot_relative_floor_ = float(relativeFloor)
        self.static_pivot_absolute_floor_ = float(absoluteFloor)

    def setParallel(self, parallel):
        """Accepted for API parity; the device path is always parallel."""
        self.parallel_ = bool(parallel)

    def setNumThreads(self, n):
        """Accepted for API parity (host thread count of the CPU path)."""
        self.num_threads_ = int(n)

    def setFrontDeltas(self, deltas):
        """Per-supernode first-attempt static-pivot deltas (learned predictor)."""
        self.front_delta_ = None if deltas is None else np.ascontiguousarray(deltas, dtype=np.float64)

    # --- diagnostics (solver.hpp:106-111) ---
    def lastRegularizationDelta(self):
        return self.last_regularization_delta_

    def regularizationRetriesUsed(self):
        return self.regularization_retries_used_

    def totalPerturbation(self):
        return self.last_info.total_perturbation

    def numPerturbedPivots(self):
        return self.last_info.num_perturbed

    # --- staged API ---
    def analyzePattern(self, A, options: SymbolicFactorOptions = None):
        n, cp, ri, _ = as_csc(A)
        self._analysis = Analysis(n, cp, ri, self.ordering_, options or SymbolicFactorOptions())
        self._pattern = (cp, ri)
        self._ctx = None
        self.pattern_analyzed_ = True
        self.factorized_ = False
        self._numeric = None

    def _context(self, cp, ri):
        if self._ctx is None or not self._ctx.same_pattern(cp, ri):
            self._ctx = Context(self._analysis, cp, ri, self.device)
            L.load().symla_gpu_set_graph(self._ctx.h, int(self.graph_launch_))
        return self._ctx

    # --- B200 extension: graph launch of the factorization (no reference
    # counterpart; results are those of the ordinary launch path) ---
    def setGraphLaunch(self, enable: bool):
        self.graph_launch_ = bool(enable)
        if self._ctx is not None:
            L.load().symla_gpu_set_graph(self._ctx.h, int(self.graph_launch_))

    def graphStats(self):
        cap, res = C.c_int(), C.c_int()
        if self._ctx is not None:
            L.load().symla_gpu_graph_stats(self._ctx.h, C.byref(cap), C.byref(res))
        return {"captures": cap.value, "resumes": res.value}

    def factorize(self, A):
        if not self.pattern_analyzed_:
            raise LogicError("symla::SymLDLT::factorize: analyzePattern must be called first")
        n, cp, ri, vals = as_csc(A)
        if n != self._analysis.n:
            raise InvalidArgument("symla::SymLDLT::factorize: matrix size differs from the analyzed pattern")
        ctx = self._context(cp, ri)
        self._numeric = None
        lib = L.load()
        info = L.FactorInfo()
        if self.mode_ == Mode.StaticRegularized:
            self._factorize_static(ctx, vals, info)
            return
        o = L.FactorOpts()
        lib.symla_factor_opts_default(C.byref(o))
        o.mode = L.MODE_THRESHOLD
        o.precision = int(self.precision_)
        o.pivot_threshold = self.pivot_threshold_
        o.zero_tolerance = self.zero_tolerance_
        o.relative_pivot_floor = self.relative_pivot_floor_
        _check(lib.symla_gpu_factorize(ctx.h, L.ptr_d(vals), 0, C.byref(o), C.byref(info)))
        self._after_factor(ctx, info)
        self.last_regularization_delta_ = 0.0
        self.regularization_retries_used_ = 0

    def _factorize_static(self, ctx, vals, info):
        lib = L.load()
        n = ctx.n
        ro = L.RegularizeOpts()
        lib.symla_regularize_opts_default(C.byref(ro))
        ro.initial_delta = self.initial_regularization_delta_
        ro.max_retries = self.max_regularization_retries_
        ro.growth = self.regularization_growth_
        ro.static_rel_floor = self.static_pivot_relative_floor_
        ro.static_abs_floor = self.static_pivot_absolute_floor_
        ro.precision = int(self.precision_)
        signs = None
        if self.use_explicit_signs_:
            if len(self.expected_signs_orig_) != n:
                raise InvalidArgument("symla::SymLDLT::factorize: setExpectedSignPattern's vector size does not "
                                      "match the matrix size")
            signs = self.expected_signs_orig_
            ro.expected_sign = L.ptr_i(signs)
        elif self.use_kkt_blocks_:
            ro.kkt_n1, ro.kkt_n2 = self.kkt_n1_, self.kkt_n2_
        fd = self.front_delta_
        if fd is not None:
            ro.front_delta = L.ptr_d(fd)
        rinfo = L.RegularizeInfo()
        rc = lib.symla_gpu_factorize_regularized(ctx.h, L.ptr_d(vals), 0, C.byref(ro), C.byref(info), C.byref(rinfo))
        self.last_reg_info = rinfo
        if rc != L.SYMLA_OK:
            if rc == L.SYMLA_ERR_RETRY_EXHAUSTED:
                self.last_regularization_delta_ = rinfo.last_delta
                self.regularization_retries_used_ = rinfo.retries_used
            _check(rc)
        self.last_regularization_delta_ = rinfo.last_delta
        self.regularization_retries_used_ = rinfo.retries_used
        self._after_factor(ctx, info)

    def _after_factor(self, ctx, info):
        lib = L.load()
        self.last_info = info
        self.inertia_ = Inertia(info.n_pos, info.n_neg, info.n_zero)
        cols = np.zeros(max(1, info.n_singular), np.int32)
        k = lib.symla_gpu_singular_cols(ctx.h, L.ptr_i(cols), len(cols))
        self._singular_cols = [int(x) for x in cols[:k]]
        self.factorized_ = True

    def compute(self, A):
        self.analyzePattern(A)
        self.factorize(A)

    def refactorize(self, A):
        self.factorize(A)

    def _rhs(self, B):
        B = np.asarray(B, dtype=np.float64)
        vec = B.ndim == 1
        B2 = B.reshape(-1, 1) if vec else B
        return np.asfortranarray(B2), vec

    def solve(self, B):
        if not self.factorized_:
            raise LogicError("symla::SymLDLT::solve: factorize() must be called before solve()")
        if self.isSingular():
            raise LogicError("symla::SymLDLT::solve: factorization is numerically singular (see isSingular()/"
                             "singularColumns()); refusing to solve")
        Bf, vec = self._rhs(B)
        n = self._ctx.n
        if Bf.shape[0] != n:
            raise InvalidArgument("symla::SymLDLT::solve: B.rows() must match the factorized matrix size")
        nrhs = Bf.shape[1]
        X = np.zeros((n, nrhs), dtype=np.float64, order="F")
        if nrhs > 0 and n > 0:
            _check(L.load().symla_gpu_solve(self._ctx.h, L.ptr_d(Bf), n, nrhs, L.ptr_d(X), n, 0))
        return X[:, 0] if vec else X

    def solveWithRefinement(self, A, B, options: RefinementOptions = None) -> RefinedSolve:
        options = options or RefinementOptions()
        if not self.factorized_:
            raise LogicError("symla::SymLDLT::solve: factorize() must be called before solve()")
        if self.isSingular():
            raise LogicError("symla::SymLDLT::solve: factorization is numerically singular; refusing to solve")
        n, cp, ri, vals = as_csc(A)
        if not self._ctx.same_pattern(cp, ri):
            raise InvalidArgument("symla::SymLDLT::solveWithRefinement: A's pattern differs from the factorized one")
        Bf, vec = self._rhs(B)
        if Bf.shape[0] != n:
            raise InvalidArgument("symla::SymLDLT::solve: B.rows() must match the factorized matrix size")
        nrhs = Bf.shape[1]
        X = np.zeros((n, nrhs), dtype=np.float64, order="F")
        ri_ = L.RefineInfo()
        if nrhs > 0 and n > 0:
            _check(L.load().symla_gpu_solve_refine(self._ctx.h, L.ptr_d(vals), L.ptr_d(Bf), n, nrhs, L.ptr_d(X), n,
                                                   0, int(options.max_iterations), float(options.tolerance),
                                                   C.byref(ri_)))
        diag = RefinementResult(ri_.iterations, ri_.initial_relative_residual, ri_.final_relative_residual)
        return RefinedSolve(X[:, 0] if vec else X, diag)

    def solveWithGmresRefinement(self, A, B, options: GmresRefinementOptions = None) -> RefinedSolve:
        """GMRES-IR: like solveWithRefinement (same errors, same backward
        error measure and acceptance rule) with every correction solved by
        preconditioned GMRES; diagnostics is a GmresResult."""
        options = options or GmresRefinementOptions()
        if not self.factorized_:
            raise LogicError("symla::SymLDLT::solve: factorize() must be called before solve()")
        if self.isSingular():
            raise LogicError("symla::SymLDLT::solve: factorization is numerically singular; refusing to solve")
        n, cp, ri, vals = as_csc(A)
        if not self._ctx.same_pattern(cp, ri):
            raise InvalidArgument("symla::SymLDLT::solveWithRefinement: A's pattern differs from the factorized one")
        Bf, vec = self._rhs(B)
        if Bf.shape[0] != n:
            raise InvalidArgument("symla::SymLDLT::solve: B.rows() must match the factorized matrix size")
        nrhs = Bf.shape[1]
        X = np.zeros((n, nrhs), dtype=np.float64, order="F")
        gi = L.GmresInfo()
        if nrhs > 0 and n > 0:
            _check(L.load().symla_gpu_solve_gmres_refine(self._ctx.h, L.ptr_d(vals), L.ptr_d(Bf), n, nrhs,
                                                         L.ptr_d(X), n, 0, int(options.max_outer),
                                                         int(options.restart), float(options.tolerance),
                                                         C.byref(gi)))
        diag = GmresResult(gi.outer_iterations, gi.inner_iterations, gi.initial_relative_residual,
                           gi.final_relative_residual)
        return RefinedSolve(X[:, 0] if vec else X, diag)

    # --- results (solver.hpp:242-262) ---
    def inertia(self) -> Inertia:
        return self.inertia_

    def patternAnalyzed(self):
        return self.pattern_analyzed_

    def factorized(self):
        return self.factorized_

    def isSingular(self):
        return bool(self.last_info.singular) if self.factorized_ else False

    def singularColumns(self):
        perm = self.symbolicFactor().perm
        return [int(perm[c]) for c in self._singular_cols]

    def symbolicFactor(self) -> SymbolicFactor:
        if self._analysis is None:
            raise LogicError("symla::SymLDLT: analyzePattern must be called first")
        return self._analysis.factor()

    def numericFactor(self) -> NumericFactor:
        if not self.factorized_:
            raise LogicError("symla::SymLDLT: factorize() must be called first")
        if self._numeric is not None:
            return self._numeric
        lib = L.load()
        h = self._ctx.h
        nf = lib.symla_gpu_num_fronts(h)
        fronts = []
        for si in range(nf):
            m = C.c_int()
            npv = C.c_int()
            _check(lib.symla_gpu_front_size(h, si, C.byref(m), C.byref(npv)))
            m, npv = m.value, npv.value
            rows = np.zeros(max(1, m), np.int32)
            Lm = np.zeros((m, npv), dtype=np.float64, order="F")
            dd = np.zeros(max(1, npv))
            do = np.zeros(max(1, npv))
            ps = np.zeros(max(1, npv), np.int32)
            pk = np.zeros(max(1, npv), np.int32)
            nb = lib.symla_gpu_front_get(h, si, L.ptr_i(rows), L.ptr_d(Lm) if npv > 0 else None, L.ptr_d(dd),
                                         L.ptr_d(do), L.ptr_i(ps), L.ptr_i(pk))
            if nb < 0:
                _check(-nb)
            blocks = [PivotBlock(int(ps[b]), int(pk[b])) for b in range(nb)]
            fronts.append(SupernodeFactor(rows[:m].copy(), npv, Lm, dd[:npv].copy(), do[:npv].copy(), blocks))
        self._numeric = NumericFactor(fronts, self.symbolicFactor().perm, self.inertia_, self.isSingular(),
                                      list(self._singular_cols), self._ctx.n, self.last_info.total_perturbation,
                                      self.last_info.num_perturbed)
        return self._numeric

    # --- measurement helpers ---
    def phase_ms(self):
        buf = (C.c_float * 8)()
        L.load().symla_gpu_phase_ms(self._ctx.h, buf, 8)
        return list(buf)

    def plan_stats(self):
        buf = (C.c_double * 15)()
        L.load().symla_gpu_plan_stats(self._ctx.h, buf, 15)
        keys = ["fronts", "levels", "max_m", "sum_m2", "factor_flops", "nnz_L", "arena_doubles",
                "panels_spec_full", "panels_spec_prefix", "panels_spec_failed", "panels_sequential",
                "seq_1x1_first_test", "seq_1x1_sigma_test", "seq_interchange", "seq_2x2"]
        return dict(zip(keys, list(buf)))
