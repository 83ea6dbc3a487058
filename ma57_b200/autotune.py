"""Front-size-to-tile-shape schedule chosen by measurement.

Three launch shapes depend on front size and have no single best value:
the width of the small-front kernel (a warp per front for fronts of at most
32 rows, or 128 or 256 threads per front), the
number of CTAs in the panel cluster of the large fronts (2, 4, 8 or 16; more
CTAs hold fewer rows each but occupy more SMs; or 1, the single-CTA panel
kernel, whose pivot-by-pivot decisions need no cluster barriers) and the
tile shape of their
Schur-complement update (128 x 64 or 64 x 64: the smaller tile wastes less
of small fronts' trailing blocks, the larger reuses operands more). The tree
levels are bucketed by
the largest front they hold, and a coordinate search times the actual
factorization (CUDA events around the numeric factorization) for each
candidate shape of one bucket at a time, keeping the fastest. The result is
installed per level through symla_gpu_set_level_schedule; it changes launch
shapes only, never results.
"""
from __future__ import annotations

import ctypes as C
import math

from . import _lib as L

SMALL_BUCKETS = (48, 128)                    # small-front kernel, by the level's largest small front
LARGE_BUCKETS = (512, 2048, 8192, 1 << 30)  # panel cluster, by the level's largest large front


def level_info(solver):
    """Per level: small/large front counts and largest sizes, and the
    installed shapes."""
    lib = L.load()
    h = solver._ctx.h
    nlev = int(solver.plan_stats()["levels"])
    out = []
    buf = (C.c_int * 6)()
    for lv in range(nlev):
        if lib.symla_gpu_level_info(h, lv, buf) != L.SYMLA_OK:
            raise RuntimeError(L.last_error())
        out.append({"small": buf[0], "small_max_m": buf[1], "large": buf[2], "large_max_m": buf[3],
                    "small_threads": buf[4], "cluster_ctas": buf[5]})
    return out


def _bucket(value, edges):
    for i, e in enumerate(edges):
        if value <= e:
            return i
    return len(edges) - 1


def apply(solver, schedule):
    """schedule: {"small": {bucket: threads}, "large": {bucket: ctas},
    "update": {bucket: tile rows}} (missing entries: the default shape)."""
    lib = L.load()
    for lv, info in enumerate(level_info(solver)):
        st = schedule["small"].get(_bucket(info["small_max_m"], SMALL_BUCKETS), 0) if info["small"] else 0
        lb = _bucket(info["large_max_m"], LARGE_BUCKETS)
        cl = schedule["large"].get(lb, 0) if info["large"] else 0
        ur = schedule.get("update", {}).get(lb, 0) if info["large"] else 0
        if lib.symla_gpu_set_level_schedule(solver._ctx.h, lv, st, cl) != L.SYMLA_OK:
            raise RuntimeError(L.last_error())
        if lib.symla_gpu_set_level_update_rows(solver._ctx.h, lv, ur) != L.SYMLA_OK:
            raise RuntimeError(L.last_error())


def _factor_ms(solver, A, reps):
    best = math.inf
    for _ in range(reps):
        solver.factorize(A)
        best = min(best, solver.phase_ms()[6])
    return best


def tune(solver, A, reps: int = 2):
    """Coordinate search over the buckets present in `solver`'s plan (the
    pattern of A must be analyzed and factorized once). Returns the chosen
    schedule (installed) and the measured default / tuned factorization ms."""
    info = level_info(solver)
    small_b = sorted({_bucket(i["small_max_m"], SMALL_BUCKETS) for i in info if i["small"]})
    large_b = sorted({_bucket(i["large_max_m"], LARGE_BUCKETS) for i in info if i["large"]})
    schedule = {"small": {}, "large": {}, "update": {}}
    apply(solver, schedule)
    base = _factor_ms(solver, A, reps)
    best = base
    for kind, buckets, cands in (("small", small_b, (32, 128, 256)), ("large", large_b, (1, 2, 4, 8, 16)),
                                 ("update", large_b, (64, 128))):
        for b in buckets:
            for cand in cands:
                trial = {k: dict(v) for k, v in schedule.items()}
                trial[kind][b] = cand
                apply(solver, trial)
                t = _factor_ms(solver, A, reps)
                if t < best:
                    best, schedule = t, trial
    apply(solver, schedule)
    return schedule, base, best
