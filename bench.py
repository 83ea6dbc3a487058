#!/usr/bin/env python
"""Benchmark: factorize + solve time to backward error <= 1e-12 on the 27-point
3D shifted stencil A = L27(64^3) - 3 I (n = 262144, METIS nested dissection,
nrhs = 16, B ~ N(0,1)), on B200.

One step = numeric factorization + multi-RHS solve with FP64 iterative
refinement until the backward error ||R||/(||A|| ||X|| + ||B||) <= 1e-12
(refine.hpp:109-114), with A's values and B already in device memory. The
symbolic analysis and the device plan are built once, outside the timed
region (as in the reference, analyzePattern is separate from factorize).

Output: one JSON line (see the "metric" field). value = seconds per step
(max over ranks; each rank factors its own replica -- the factorization does
not shard, so N GPUs run N independent replicas). e2e = the same step through
the C ABI with host buffers, host<->device copies included.

--impl reference times the project's CPU restatement of the reference
(oracle/) on the host cores: the reference itself needs Eigen, SuiteSparse AMD
and LAPACK, none of which are installed, so it cannot be built here.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "factorize+solve s at backward error ≤1e-12: mixed/learned vs plain FP64 B200"
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")


def load_peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def clocks_start(index):
    f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                              "-lms", "200"], stdout=f, stderr=subprocess.DEVNULL)
    except Exception:
        p = None
    return p, f.name


def clocks_stop(handle):
    p, path = handle
    if p is not None:
        p.terminate()
        try:
            p.wait(timeout=5)
        except Exception:
            p.kill()
    sms, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        with open(path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sms.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(path)
    except Exception:
        pass
    return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sms)}


def build_problem(k, nrhs):
    from ma57_b200 import matrices as M
    A, B = M.config3(k, nrhs=nrhs)
    return A, B


def cpu_reference(k_sample: int, nrhs: int, reps: int, flop_ratio_to: int | None):
    """Oracle (CPU restatement) factorize + solve + refine on cfg3 at k_sample."""
    import numpy as np
    from ma57_b200 import OrderingType, SymLDLT
    from ma57_b200.solver import as_csc
    from oracle.pyoracle import OracleSymLDLT
    A, B = build_problem(k_sample, nrhs)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.analyzePattern(A)
    o = OracleSymLDLT(s.symbolicFactor())
    threads = os.cpu_count() or 1
    o.set(parallel=1, num_threads=threads)
    times = []
    err = None
    for _ in range(reps):
        t0 = time.perf_counter()
        o.factorize(A)
        x, d = o.solveWithRefinement(A, B, tolerance=1e-12)
        times.append(time.perf_counter() - t0)
        err = d["final"]
    return min(times), threads, err


def algorithmic_flops(k):
    """Algorithmic factorization flops of cfg3 at grid k, from the symbolic
    structure (all pivots 1x1, lower-triangle convention)."""
    from ma57_b200 import OrderingType, SymLDLT
    A, _ = build_problem(k, 1)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.analyzePattern(A)
    f = 0.0
    for sn in s.symbolicFactor().supernodes:
        m = len(sn.rowPattern)
        for kk in range(sn.ncols):
            r = m - kk - 1
            f += r + r * (r + 1)
    return f


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    k_sample = args.cpu_k
    best, threads, err = cpu_reference(k_sample, args.nrhs, max(1, args.steps), None)
    ratio = algorithmic_flops(args.k) / algorithmic_flops(k_sample)
    value = best * ratio
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"L27({args.k}^3)-3I, METIS ND, nrhs={args.nrhs}, refine to 1e-12",
                   "parallelism": "cpu-openmp-task-dag"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port",
                         "sample": f"oracle (CPU restatement; the reference needs Eigen/SuiteSparse/LAPACK, absent) "
                                   f"factorize+solve+refine on L27({k_sample}^3)-3I, best of {max(1, args.steps)}, "
                                   f"{best:.3f} s, scaled by the algorithmic flop ratio {ratio:.1f} to {args.k}^3; "
                                   f"final backward error {err:.2e}"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch

    from ma57_b200 import OrderingType, Precision, SymLDLT
    from ma57_b200 import _lib as L
    from ma57_b200.solver import as_csc

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    lib = L.load()
    A, B = build_problem(args.k, args.nrhs)
    n = A.shape[0]
    nrhs = args.nrhs
    s = SymLDLT(device=local)
    s.setOrdering(OrderingType.Metis)
    t0 = time.perf_counter()
    s.analyzePattern(A)
    t_analyze = time.perf_counter() - t0
    _, cp, ri, vals = as_csc(A)
    ctx = s._context(cp, ri)
    h = ctx.h
    prec = L.PREC_MIXED if args.precision == "mixed" else L.PREC_FP64
    opts = L.FactorOpts()
    lib.symla_factor_opts_default(C.byref(opts))
    opts.precision = prec
    info = L.FactorInfo()
    rinfo = L.RefineInfo()

    dev = torch.device("cuda", local)
    d_vals = torch.from_numpy(vals).to(dev)
    d_B = torch.from_numpy(np.asfortranarray(B).T.copy()).to(dev)  # row c = rhs column c (n x nrhs col-major)
    d_X = torch.zeros((nrhs, n), dtype=torch.float64, device=dev)
    pv = C.cast(C.c_void_p(d_vals.data_ptr()), L._pd)
    pB = C.cast(C.c_void_p(d_B.data_ptr()), L._pd)
    pX = C.cast(C.c_void_p(d_X.data_ptr()), L._pd)
    stream = torch.cuda.ExternalStream(lib.symla_gpu_stream(h), device=dev)

    def check(rc):
        if rc != 0:
            raise RuntimeError(f"{L.last_error()} (status {rc})")

    def step():
        check(lib.symla_gpu_factorize(h, pv, 1, C.byref(opts), C.byref(info)))
        check(lib.symla_gpu_solve_refine(h, pv, pB, n, nrhs, pX, n, 1, 10, 1e-12, C.byref(rinfo)))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    lib.symla_gpu_reset_kernel_stats(h)
    lib.symla_gpu_set_profiling(h, 1)
    clk = clocks_start(local)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    errs = []
    for _ in range(args.steps):
        step()
        errs.append(rinfo.final_relative_residual)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = clocks_stop(clk)
    lib.symla_gpu_set_profiling(h, 0)
    ms = ev0.elapsed_time(ev1) / args.steps
    if dist:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    launches = int(lib.symla_gpu_launch_count(h)) // max(1, args.steps)
    kstats = {}
    buf = (C.c_double * 4)()
    for kind, name in enumerate(L.KERNEL_KINDS):
        lib.symla_gpu_kernel_stats(h, kind, buf)
        kstats[name] = list(buf)
    stats = s.plan_stats()

    # e2e through the C ABI with host buffers
    Bh = np.asfortranarray(B)
    Xh = np.zeros((n, nrhs), order="F")
    e2e_times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(lib.symla_gpu_factorize(h, L.ptr_d(vals), 0, C.byref(opts), C.byref(info)))
        check(lib.symla_gpu_solve_refine(h, L.ptr_d(vals), L.ptr_d(Bh), n, nrhs, L.ptr_d(Xh), n, 0, 10, 1e-12,
                                         C.byref(rinfo)))
        e2e_times.append(time.perf_counter() - t0)
    e2e = statistics.median(e2e_times)
    if dist:
        t = torch.tensor([e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = float(t.item())

    # independent check of the backward error of the host-path result
    import scipy.sparse as sp
    from ma57_b200 import matrices as M
    Af = M.sym_full(A)
    R = Bh - Af @ Xh
    normA = float(np.asarray(abs(sp.csr_matrix(A)).sum(axis=1)).max())
    bw = float(np.abs(R).max() / (normA * np.abs(Xh).max() + np.abs(Bh).max()))

    peaks, peak_kind = load_peaks()
    tr = kstats["far_update"]
    achieved = (tr[2] / (tr[1] * 1e-3)) / 1e12 if tr[1] > 0 else 0.0
    if prec == L.PREC_MIXED:
        peak = peaks.get("bf16_tflops")
        peak_note = f"dense bf16 tensor, {peak_kind}"
    else:
        peak = peaks.get("bf16_tflops")
        peak_note = f"dense bf16 tensor, {peak_kind} (FP64 kernel timed against the tensor peak)"
    roofline = {"bound": "tensor", "kernel": "far (outer-block) Schur-complement update", "achieved": achieved,
                "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                "traffic": None, "peak_source": peak_note,
                "launches_per_step": tr[0] / max(1, args.steps), "ms_per_step": tr[1] / max(1, args.steps),
                "algorithmic_flops_per_step": tr[2] / max(1, args.steps)}

    line = {
        "metric": METRIC, "value": ms / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == L.PREC_FP64 else "f64+mixed-schur", "data": "synthetic",
        "config": {"workload": f"L27({args.k}^3)-3I (n={n}), METIS ND, nrhs={nrhs}, factorize+solve+refine to 1e-12",
                   "precision": args.precision, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (fronts 11 GB)", "inertia": list(s.inertia().as_tuple()),
                   "backward_error": bw, "refine_iterations": rinfo.iterations,
                   "analyze_s": t_analyze, "factor_flops": stats.get("factor_flops"),
                   "kernel_ms_per_step": {k: v[1] / max(1, args.steps) for k, v in kstats.items()}},
        "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": int(8 * (2 * len(vals) + n * nrhs)),
                "d2h_bytes_per_step": int(8 * n * nrhs)},
        "gpu_launches": launches,
        "roofline": roofline,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        best, threads, err = cpu_reference(args.cpu_k, nrhs, 2, None)
        ratio = algorithmic_flops(args.k) / algorithmic_flops(args.cpu_k)
        line["cpu_baseline"] = {"value": best * ratio, "unit": "s", "cores": threads, "kind": "port",
                                "sample": f"oracle factorize+solve+refine on L27({args.cpu_k}^3)-3I, best of 2 = "
                                          f"{best:.3f} s, scaled by the algorithmic flop ratio {ratio:.1f}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--k", type=int, default=64)
    ap.add_argument("--nrhs", type=int, default=16)
    ap.add_argument("--cpu-k", type=int, default=32)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
