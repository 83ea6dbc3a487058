"""B200-native numeric factorize / solve for symla (alecjacobson/ma57).

The public entry point is :class:`SymLDLT`, a mirror of the reference's
``symla::SymLDLT<double>`` whose numeric work runs in hand-written sm_100a
kernels behind the C ABI declared in ``include/symla_gpu.h``.
"""
from .solver import (GmresRefinementOptions, GmresResult, Inertia, InvalidArgument, LogicError, Mode, NumericFactor, OrderingType, Precision,
                     RefinedSolve, RefinementOptions, RefinementResult, SymbolicFactor, SymbolicFactorOptions,
                     SymLDLT, as_csc, computeOrdering)

__all__ = ["SymLDLT", "Mode", "OrderingType", "Precision", "Inertia", "SymbolicFactorOptions",
           "RefinementOptions", "RefinementResult", "RefinedSolve", "SymbolicFactor", "NumericFactor",
           "LogicError", "InvalidArgument", "as_csc", "computeOrdering", "GmresRefinementOptions", "GmresResult"]
