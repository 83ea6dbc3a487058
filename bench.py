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
(oracle/: the reference's dense kernel, multifrontal driver, OpenMP task DAG,
solve and refinement) on the host cores, on the same 64^3 workload, one
whole factorize + solve + refinement per timed step: the reference itself
needs Eigen, SuiteSparse AMD and LAPACK, none of which are installed, so it
cannot be built here. Its host analysis is compiled into the oracle library
from the same sources, so that arm does not load the product library.
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


# Bytes of DRAM traffic per algorithmic flop of the FP64 Schur update,
# measured by ncu on config 3 at k = 40 (see roofline below).
UPDATE_DRAM_BYTES_PER_FLOP = 1.2578e9 / 25.8151e9


def replica_group(world: int, backend: str = "nccl"):
    """torch.distributed for N > 1 replicas launched by torchrun (RANK,
    WORLD_SIZE, MASTER_* from the environment), or None for one process. The
    replicas exchange nothing on the data path: only barriers around the
    timed region and the max-over-ranks reductions below. The short timeout
    ends a wait for a rank that died with an error instead of a hang."""
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return dist


def max_over_ranks(value: float, dist, device) -> float:
    """The slowest replica's figure; every rank calls this in the same order."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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


def shared_config(k, nrhs):
    """The workload keys both arms report (identical in the two lines)."""
    return {"workload": f"L27({k}^3)-3I (n={k ** 3}), METIS ND, nrhs={nrhs}, factorize+solve+refine to 1e-12",
            "n": k ** 3, "nrhs": nrhs, "ordering": "metis", "target_backward_error": 1e-12}


def build_problem(k, nrhs):
    from ma57_b200 import matrices as M
    A, B = M.config3(k, nrhs=nrhs)
    return A, B


def cpu_reference(k_sample: int, nrhs: int, reps: int, flop_ratio_to: int | None):
    """Oracle (CPU restatement) factorize + solve + refine on cfg3 at k_sample."""
    from oracle.pyoracle import OracleSymLDLT, analyze
    A, B = build_problem(k_sample, nrhs)
    o = OracleSymLDLT(analyze(A, 1))
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


def panel_bytes(k):
    """Algorithmic bytes of the large-front panel factorization of cfg3 at
    grid k: every pivot column of a front with m > 128 is read and its L
    written once below the pivot (16 bytes per entry)."""
    from ma57_b200 import OrderingType, SymLDLT
    A, _ = build_problem(k, 1)
    s = SymLDLT()
    s.setOrdering(OrderingType.Metis)
    s.analyzePattern(A)
    b = 0.0
    for sn in s.symbolicFactor().supernodes:
        m, p = len(sn.rowPattern), sn.ncols
        if m > 128:
            b += 16.0 * (m * p - p * (p - 1) / 2.0)
    return b


def run_dense(args):
    """One dense front (the profiling case of the large-front kernels): a
    random symmetric indefinite matrix with a dominant diagonal of random
    sign, natural order, factorized `steps` times after `warmup`."""
    import numpy as np
    import scipy.sparse as sp
    import torch
    from ma57_b200 import OrderingType, Precision, SymLDLT
    from ma57_b200 import _lib as L
    n = args.n
    rng = np.random.default_rng(n)
    G = rng.standard_normal((n, n))
    A0 = (G + G.T) / 2 + np.diag(rng.choice([-1.0, 1.0], n) * n / 51.2)
    ii, jj = np.tril_indices(n)
    A = sp.csc_matrix((A0[ii, jj], (ii, jj)), shape=(n, n))
    s = SymLDLT()
    s.setOrdering(OrderingType.Natural)
    s.setPrecision(Precision.Mixed if args.precision == "mixed" else Precision.FP64)
    s.analyzePattern(A)
    for _ in range(max(1, args.warmup)):
        s.factorize(A)
    lib = L.load()
    lib.symla_gpu_reset_kernel_stats(s._ctx.h)
    lib.symla_gpu_set_profiling(s._ctx.h, 1)
    times = []
    for _ in range(max(1, args.steps)):
        s.factorize(A)
        times.append(s.phase_ms()[6])
    lib.symla_gpu_set_profiling(s._ctx.h, 0)
    buf = (C.c_double * 4)()
    ks = {}
    for kind, name in enumerate(L.KERNEL_KINDS):
        lib.symla_gpu_kernel_stats(s._ctx.h, kind, buf)
        if buf[0]:
            ks[name] = {"launches": buf[0] / len(times), "ms": buf[1] / len(times)}
    print(json.dumps({"workload": f"dense front n={n} (natural order, one front)", "precision": args.precision,
                      "factor_ms": min(times), "inertia": list(s.inertia().as_tuple()), "kernels": ks,
                      "panels": {k: v for k, v in s.plan_stats().items() if k.startswith("panels_")}}), flush=True)


def run_batched(args):
    """Config 4: independent L5-minus-shift systems of uneven size, factorized
    and solved together (ma57_b200.batch: one block-diagonal plan, level
    launches shared by all systems, graph launch of the factorization).
    value = systems per second of factorize + 8-RHS solve with the matrices
    and right-hand sides resident on the device; the per-system latency
    percentiles come from factorizing + solving a sample of the systems one
    at a time through the same library."""
    import numpy as np
    import torch
    from ma57_b200 import SymLDLT
    from ma57_b200 import _lib as L
    from ma57_b200 import autotune
    from ma57_b200 import matrices as M
    from ma57_b200.batch import BatchedSolver
    from ma57_b200.solver import as_csc
    count, nrhs = args.systems, 8
    systems = [M.config4_system(i) for i in range(count)]
    mats = [A for A, _, _, _ in systems]
    Bs = []
    for i, A in enumerate(mats):
        st = M.Stream(M.SEED_BASE + 4 + 7_000_001 * (i + 1))
        Bs.append(st.normal(A.shape[0] * nrhs).reshape(nrhs, A.shape[0]).T.copy(order="F"))
    t0 = time.perf_counter()
    bs = BatchedSolver(mats, graph=bool(args.graph))
    t_setup = time.perf_counter() - t0
    lib = L.load()
    s = bs.solver
    bs.factorize()
    schedule, t_default, t_tuned = autotune.tune(s, bs.A, reps=2)
    n = bs.n
    _, cp, ri, vals = as_csc(bs.A)
    h = s._ctx.h
    dev = torch.device("cuda", 0)
    d_vals = torch.from_numpy(vals).to(dev)
    d_B = torch.from_numpy(np.ascontiguousarray(bs.stack(Bs).T)).to(dev)
    d_X = torch.zeros((nrhs, n), dtype=torch.float64, device=dev)
    pv = C.cast(C.c_void_p(d_vals.data_ptr()), L._pd)
    pB = C.cast(C.c_void_p(d_B.data_ptr()), L._pd)
    pX = C.cast(C.c_void_p(d_X.data_ptr()), L._pd)
    opts = L.FactorOpts()
    lib.symla_factor_opts_default(C.byref(opts))
    info = L.FactorInfo()
    stream = torch.cuda.ExternalStream(lib.symla_gpu_stream(h), device=dev)

    def step():
        if lib.symla_gpu_factorize(h, pv, 1, C.byref(opts), C.byref(info)) != 0:
            raise RuntimeError(L.last_error())
        if lib.symla_gpu_solve(h, pB, n, nrhs, pX, n, 1) != 0:
            raise RuntimeError(L.last_error())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clk = clocks_start(0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clocks_stop(clk)
    ms = e0.elapsed_time(e1) / args.steps
    X = d_X.cpu().numpy().T
    Xs = bs.unstack(np.asfortranarray(X))
    worst = 0.0
    for A, B, Xi in zip(mats[:256], Bs[:256], Xs[:256]):
        Af = M.sym_full(A)
        R = B - Af @ Xi
        worst = max(worst, np.abs(R).max() / (abs(A).sum(axis=1).max() * np.abs(Xi).max() + np.abs(B).max()))

    # per-system latency when the systems are served in batches of
    # --batch-size (arrival order): a system's result is ready when its
    # batch's factorize + solve ends, so its latency is its batch's time
    # (device events, after a warm-up of the batch's own graph)
    batch_lat, per_system = [], []
    for b0 in range(0, count, args.batch_size):
        sub = mats[b0:b0 + args.batch_size]
        bb = BatchedSolver(sub, graph=bool(args.graph))
        Bb = bb.stack(Bs[b0:b0 + args.batch_size])
        for _ in range(2):
            bb.factorize()
            bb.solver.solve(Bb)
        ts = []
        for _ in range(3):
            bb.factorize()
            bb.solver.solve(Bb)
            ph = bb.solver.phase_ms()
            ts.append(ph[6] + ph[7])
        t = min(ts)
        batch_lat.append(t)
        per_system += [t] * len(sub)
        del bb
    # single systems, one at a time (factorize + solve, device timing)
    lat = []
    for idx in np.linspace(0, count - 1, 64).astype(int):
        A, B = mats[idx], Bs[idx]
        si = SymLDLT()
        si.analyzePattern(A)
        si.factorize(A)
        si.solve(B)
        si.factorize(A)
        si.solve(B)
        ph = si.phase_ms()
        lat.append(ph[6] + ph[7])

    # CPU baseline on a bounded sample of the systems: the oracle (the
    # reference's algorithm) in a sequential loop over systems, as the
    # reference, which has no batch API, would run them; and, labelled as not
    # the reference, the same per-system work in a thread pool over systems
    cpu = None
    if not args.no_cpu:
        from concurrent.futures import ThreadPoolExecutor
        from oracle.pyoracle import OracleSymLDLT, analyze
        sample = list(range(min(count, args.cpu_systems)))
        solvers = []
        for i in sample:
            o = OracleSymLDLT(analyze(mats[i], 0))
            o.set(parallel=0)
            solvers.append(o)

        def one(i):
            solvers[i].factorize(mats[sample[i]])
            solvers[i].solve(Bs[sample[i]])

        t0 = time.perf_counter()
        for i in range(len(sample)):
            one(i)
        t_seq = time.perf_counter() - t0
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(one, range(len(sample))))
        t_par = time.perf_counter() - t0
        cpu = {"value": len(sample) / t_seq, "unit": "systems/s", "cores": 1, "kind": "port",
               "sample": f"oracle factorize + 8-RHS solve of the first {len(sample)} systems, sequential loop "
                         f"over systems (analysis excluded)",
               "harness_thread_pool": {"value": len(sample) / t_par, "threads": threads,
                                       "note": "project harness, not the reference: systems in a thread pool"}}
    line = {"metric": "batched factorize+solve throughput", "value": count / (ms * 1e-3), "unit": "systems/s",
            "higher_is_better": True, "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
            "n_gpus": 1, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"config 4: {count} systems L5(a x b) - sigma I, n in [200, 4000], nrhs={nrhs}",
                       "total_n": n, "graph": bool(args.graph), "setup_s": t_setup,
                       "autotune": {"schedule": {k: {str(b): v for b, v in d.items()} for k, d in schedule.items()},
                                    "default_factor_ms": t_default, "tuned_factor_ms": t_tuned},
                       "graph_stats": s.graphStats(), "max_backward_error_first_256": worst},
            "per_system_ms": {"p50": float(np.percentile(per_system, 50)),
                              "p99": float(np.percentile(per_system, 99)),
                              "how": f"systems served in batches of {args.batch_size} in arrival order; a "
                                     f"system's latency is its batch's factorize + solve device time",
                              "batches": len(batch_lat)},
            "single_system_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                                 "sample": "64 systems spread over the sizes, factorize + solve each alone"},
            "cpu_baseline": cpu,
            "clocks": clocks}
    print(json.dumps(line), flush=True)


def run_learned(args):
    """Config 5: an interior-point sequence of KKT refactorizations in
    StaticRegularized mode. Plain escalation (first delta 1e-14 max|K|, x10
    per failed inertia check) runs the first `ip_train` matrices and its
    accepted deltas train the network on the GPU; the remaining matrices are
    then run twice from the same state of the sequence, with plain
    escalation and with the network's first-attempt deltas (the network
    fine-tuned, after every matrix whose first attempt failed, on the deltas
    accepted for the last 20, its training time included). Reported: mean
    retries and total time (factorize + refinement towards 1e-10, GMRES-IR by
    default: the perturbed static-pivot factors are rough inverses), over all
    matrices and over those both arms refined to 1e-10. The sequence as
    specified (quasi-definite, c = 0) is run beside the nonconvex variant."""
    shifts = [0.0] if args.curvature_shift == 0.0 else [0.0, args.curvature_shift]
    results = {}
    for c in shifts:
        results["as_specified" if c == 0.0 else f"curvature_shift_{c:g}"] = learned_experiment(args, c)
    line = {"metric": "interior-point sequence: mean retries and total time, learned vs plain escalation",
            "config": {"workload": f"config 5: K_k = [[-E_k, A^T], [A, F_k]] from L7(20^3), {args.ip_steps} "
                                   f"matrices (train {args.ip_train})", "refinement": args.ip_refine,
                       "target_backward_error": 1e-10},
            "results": results, "data": "synthetic"}
    print(json.dumps(line), flush=True)


def learned_experiment(args, curvature_shift):
    import math
    import numpy as np
    from ma57_b200 import GmresRefinementOptions, Mode, OrderingType, RefinementOptions, SymLDLT, learned
    from ma57_b200 import matrices as M
    seq = M.InteriorPointSequence(k=20, steps=args.ip_steps, curvature_shift=curvature_shift)
    signs = np.r_[-np.ones(seq.n1), np.ones(seq.n2)]

    def run(steps, model, online=False):
        s = SymLDLT()
        s.setMode(Mode.StaticRegularized)
        s.setOrdering(OrderingType.AMD)
        s.setKKTBlockSizes(seq.n1, seq.n2)
        s.setMaxRegularizationRetries(40)
        sym = None
        out = {"retries": [], "resid": [], "ms": [], "feats": [], "targets": []}
        for step in steps:
            K, _ = seq.matrix(step)
            if sym is None:
                s.analyzePattern(K)
                sym = s.symbolicFactor()
            F = learned.front_features(sym, K, signs)
            t0 = time.perf_counter()
            base = 1e-14 * abs(K.data).max()
            s.setInitialRegularizationDelta(base)
            s.setFrontDeltas(None if model is None else model.front_deltas(F, base))
            s.factorize(K)
            if args.ip_refine == "gmres":
                r = s.solveWithGmresRefinement(K, seq.b, GmresRefinementOptions(max_outer=10, restart=20,
                                                                                   tolerance=1e-10))
            else:
                r = s.solveWithRefinement(K, seq.b, RefinementOptions(max_iterations=30, tolerance=1e-10))
            T = np.full(F.shape[0], math.log10(s.lastRegularizationDelta() / base))
            if online:  # the sequence's own retry history keeps the model current
                model.update(F, T, retries=s.regularizationRetriesUsed())
            out["ms"].append(1e3 * (time.perf_counter() - t0))
            out["retries"].append(s.regularizationRetriesUsed())
            out["resid"].append(r.diagnostics.final_relative_residual)
            out["feats"].append(F)
            out["targets"].append(T)
        return out

    train = run(range(args.ip_train), None)
    model = learned.DeltaModel(seed=3)
    t0 = time.perf_counter()
    groups = np.concatenate([np.full(len(t), i) for i, t in enumerate(train["targets"])])
    loss = model.fit(np.vstack(train["feats"]), np.concatenate(train["targets"]), groups, epochs=300, lr=3e-3,
                     minibatch=4096)
    t_train = time.perf_counter() - t0
    state = (seq.logx.copy(), seq.st.pos)
    plain = run(range(args.ip_train, args.ip_steps), None)
    seq.logx, seq.st.pos = state
    lrn = run(range(args.ip_train, args.ip_steps), model, online=True)
    both = (np.asarray(plain["resid"]) <= 1e-10) & (np.asarray(lrn["resid"]) <= 1e-10)

    def summ(o, sel=None):
        sel = np.ones(len(o["retries"]), bool) if sel is None else sel
        ms = np.asarray(o["ms"])[sel]
        return {"mean_retries": float(np.mean(np.asarray(o["retries"])[sel])) if sel.any() else None,
                "total_s": float(np.sum(ms) / 1e3), "matrices": int(sel.sum()),
                "refined_to_1e-10": int(np.sum(np.asarray(o["resid"])[sel] <= 1e-10)),
                "median_residual": float(np.median(np.asarray(o["resid"])[sel])) if sel.any() else None}

    return {"curvature_shift": curvature_shift, "n1": seq.n1, "n2": seq.n2,
            "train_samples": int(sum(len(t) for t in train["targets"])), "train_loss": loss, "train_s": t_train,
            "margin_decades": model.margin, "plain": summ(plain), "learned": summ(lrn),
            "both_refined_to_1e-10": {"matrices": int(both.sum()), "plain": summ(plain, both),
                                      "learned": summ(lrn, both)}}


def run_configs(args):
    """Configs 1 and 2 at their stated sizes, GPU and CPU side by side, one
    JSON line each. Config 1: L7(20^3) - 2I, AMD, one right-hand side,
    factorize + solve. Config 2: the KKT system (n = 60000),
    StaticRegularized with setKKTBlockSizes(40000, 20000), AMD, factorize +
    refinement to 1e-12. GPU: best of --steps after --warmup, device time of
    factorize and of solve (+ refinement), and the same step end to end
    through the Python API with host arrays. CPU: the oracle (the reference's
    algorithm, C++ with its OpenMP task DAG) with every host thread and with
    setParallel(false), best of --cpu-reps for config 1 and one run for
    config 2 (minutes long; --no-cpu skips it); analysis excluded."""
    import numpy as np
    from ma57_b200 import Mode, OrderingType, RefinementOptions, SymLDLT
    from ma57_b200 import matrices as M
    from oracle.pyoracle import OracleSymLDLT, analyze

    def backward_error(A, X, B):
        R = B - M.sym_full(A) @ X
        return float(np.abs(R).max() / (abs(A).sum(axis=1).max() * np.abs(X).max() + np.abs(B).max()))

    A1, b1 = M.config1(20)
    K, b2, n1, n2 = M.config2()
    cases = [("config 1: L7(20^3) - 2I, AMD, nrhs 1", A1, b1, None),
             ("config 2: KKT [[-E, A^T], [A, F]], n = 60000, StaticRegularized (40000, 20000), AMD", K, b2, (n1, n2))]
    for name, A, B, kkt in cases:
        clk = clocks_start(0)
        s = SymLDLT()
        s.setOrdering(OrderingType.AMD)
        s.setGraphLaunch(bool(args.graph))
        if kkt:
            s.setMode(Mode.StaticRegularized)
            s.setKKTBlockSizes(*kkt)
        t0 = time.perf_counter()
        s.analyzePattern(A)
        t_an = time.perf_counter() - t0
        ropt = RefinementOptions(max_iterations=10, tolerance=1e-12)

        def step():
            s.factorize(A)
            fac = s.phase_ms()[6]
            t1 = time.perf_counter()
            if kkt:
                r = s.solveWithRefinement(A, B, ropt)
                x, it = r.x, r.diagnostics.iterations
            else:
                x, it = s.solve(B), 0
            return fac, 1e3 * (time.perf_counter() - t1), x, it

        for _ in range(max(3, args.warmup)):
            step()
        fac_ms, sol_ms, e2e_ms = [], [], []
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            f, so, x, it = step()
            e2e_ms.append(1e3 * (time.perf_counter() - t0))
            fac_ms.append(f)
            sol_ms.append(so)
        clocks = clocks_stop(clk)
        line = {"metric": "factorize + solve time", "value": (min(fac_ms) + min(sol_ms)) / 1e3, "unit": "s",
                "higher_is_better": False, "steps": len(fac_ms), "warmup": max(3, args.warmup), "n_gpus": 1,
                "dtype": "f64", "data": "synthetic", "config": {"workload": name, "n": int(A.shape[0])},
                "gpu": {"factorize_ms": min(fac_ms), "solve_ms": min(sol_ms),
                        "solve_what": "solveWithRefinement to 1e-12" if kkt else "solve",
                        "e2e_ms": min(e2e_ms), "e2e_note": "host values and right-hand side through the Python API",
                        "analyze_s": t_an, "inertia": list(s.inertia().as_tuple()),
                        "retries": s.regularizationRetriesUsed() if kkt else 0, "refine_iterations": it,
                        "backward_error": backward_error(A, x, B)},
                "clocks": clocks}
        if not args.no_cpu:
            sf = analyze(A, 0)
            o = OracleSymLDLT(sf)
            if kkt:
                o.set(mode=1)
                o.setKKTBlockSizes(*kkt)
            threads = os.cpu_count() or 1
            cpu = {}
            for label, par in (("openmp", 1), ("sequential", 0)):
                if kkt and par == 0:
                    continue  # tens of minutes: the parallel run alone
                o.set(parallel=par, num_threads=threads)
                reps = 1 if kkt else max(1, args.cpu_reps)
                fs, ss = [], []
                for _ in range(reps):
                    t0 = time.perf_counter()
                    o.factorize(A)
                    t1 = time.perf_counter()
                    if kkt:
                        xo, d = o.solveWithRefinement(A, B, max_iterations=10, tolerance=1e-12)
                    else:
                        xo = o.solve(B)
                    t2 = time.perf_counter()
                    fs.append(t1 - t0)
                    ss.append(t2 - t1)
                cpu[label] = {"factorize_s": min(fs), "solve_s": min(ss), "reps": reps,
                              "threads": threads if par else 1, "inertia": list(o.inertia()),
                              "backward_error": backward_error(A, xo, B)}
            line["cpu_baseline"] = {"value": cpu["openmp"]["factorize_s"] + cpu["openmp"]["solve_s"], "unit": "s",
                                    "cores": threads, "kind": "port",
                                    "sample": "oracle on the full configuration, best of reps (analysis excluded)",
                                    "runs": cpu}
        print(json.dumps(line), flush=True)
        del s


def run_reference(args):
    """The reference's CPU path (the oracle restatement, OpenMP task DAG on
    every host core) on the same workload: each timed step is one whole
    factorize + multi-RHS solve + refinement to 1e-12 of L27(k^3) - 3I. The
    analysis (METIS ordering, elimination tree, supernodes) is outside the
    timed region, as in the GPU arm. One step takes minutes on the host, so
    the arm times as many of the requested steps as fit in --ref-budget
    seconds (at least one) and reports the count it ran."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import numpy as np
    from oracle.pyoracle import OracleSymLDLT, analyze
    threads = os.cpu_count() or 1
    # warm-up: thread pool and code paths on a small instance (untimed)
    for _ in range(max(0, args.warmup)):
        As, Bs = build_problem(12, args.nrhs)
        o = OracleSymLDLT(analyze(As, 1))
        o.set(parallel=1, num_threads=threads)
        o.factorize(As)
        o.solveWithRefinement(As, Bs, tolerance=1e-12)
    A, B = build_problem(args.k, args.nrhs)
    t0 = time.perf_counter()
    sf = analyze(A, 1)
    t_analyze = time.perf_counter() - t0
    o = OracleSymLDLT(sf)
    o.set(parallel=1, num_threads=threads)
    times, fac, sol = [], [], []
    info = d = None
    t_start = time.perf_counter()
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        o.factorize(A)
        t1 = time.perf_counter()
        x, d = o.solveWithRefinement(A, B, tolerance=1e-12)
        t2 = time.perf_counter()
        times.append(t2 - t0)
        fac.append(t1 - t0)
        sol.append(t2 - t1)
        info = o.info()
        if time.perf_counter() - t_start + times[-1] > args.ref_budget:
            break
    value = statistics.mean(times)
    inertia = [info["n_pos"], info["n_neg"], info["n_zero"]]
    sample = (f"oracle (CPU restatement of the reference; Eigen/SuiteSparse/LAPACK absent) on the full workload, "
              f"{len(times)} of {args.steps} requested steps (each step minutes long), {threads} OpenMP threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
        "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": shared_config(args.k, args.nrhs),
        "details": {"parallelism": f"cpu openmp task dag x{threads}", "analyze_s": t_analyze,
                    "factorize_s": statistics.mean(fac), "solve_refine_s": statistics.mean(sol),
                    "inertia": inertia, "backward_error": d["final"], "refine_iterations": d["iterations"],
                    "warmup": "small instance L27(12^3), untimed"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port", "sample": sample},
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
    dist = replica_group(world)

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

    lib.symla_gpu_set_graph(h, int(args.graph))

    def timed_steps(count):
        """count steps between CUDA events on the library's stream."""
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(count):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / count

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    lib.symla_gpu_reset_kernel_stats(h)
    clk = clocks_start(local)
    ms = timed_steps(args.steps)
    if dist:
        dist.barrier()
    clocks = clocks_stop(clk)
    launches = int(lib.symla_gpu_launch_count(h)) // max(1, args.steps)
    inertia = [info.n_pos, info.n_neg, info.n_zero]
    refine_iters = rinfo.iterations
    # the metric's comparison: the same steps with the mixed-precision Schur
    # update (TF32x3 tensor cores, FP64 pivots and refinement), timed alike
    comparison = None
    if not args.no_mixed:
        other = L.PREC_MIXED if prec == L.PREC_FP64 else L.PREC_FP64
        opts.precision = other
        for _ in range(args.warmup):
            step()
        ms_other = max_over_ranks(timed_steps(args.steps), dist, dev)
        name = "mixed" if other == L.PREC_MIXED else "fp64"
        comparison = {f"{name}_s": ms_other / 1e3, f"{args.precision}_s": ms / 1e3,
                      "mixed_over_fp64": (ms_other / ms) if other == L.PREC_MIXED else (ms / ms_other),
                      f"{name}_inertia": [info.n_pos, info.n_neg, info.n_zero],
                      f"{name}_refine_iterations": rinfo.iterations,
                      f"{name}_backward_error": rinfo.final_relative_residual,
                      "target": "mixed at least 3x faster than fp64 (mixed_over_fp64 <= 1/3)"}
        opts.precision = prec
        for _ in range(max(1, args.warmup)):
            step()
        torch.cuda.synchronize()

    # per-kernel breakdown from extra, instrumented steps (CUDA events around
    # every launch), kept out of the timed region above
    lib.symla_gpu_reset_kernel_stats(h)
    lib.symla_gpu_set_profiling(h, 1)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    lib.symla_gpu_set_profiling(h, 0)
    ms = max_over_ranks(ms, dist, dev)
    kstats = {}
    buf = (C.c_double * 4)()
    for kind, name in enumerate(L.KERNEL_KINDS):
        lib.symla_gpu_kernel_stats(h, kind, buf)
        kstats[name] = list(buf)
    stats = s.plan_stats()

    # e2e through the C ABI with host buffers in pinned (page-locked) memory:
    # the values, the right-hand sides and the solution cross PCIe inside the
    # timed region every step
    def pinned(count):
        t = torch.empty(count, dtype=torch.float64, pin_memory=True)
        return t, t.numpy()

    vals_t, vals_h = pinned(len(vals))
    vals_h[:] = vals
    B_t, B_flat = pinned(n * nrhs)
    Bh = B_flat.reshape(nrhs, n).T  # n x nrhs, column-major view
    Bh[:] = B
    X_t, X_flat = pinned(n * nrhs)
    Xh = X_flat.reshape(nrhs, n).T
    e2e_times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(lib.symla_gpu_factorize(h, L.ptr_d(vals_h), 0, C.byref(opts), C.byref(info)))
        check(lib.symla_gpu_solve_refine(h, L.ptr_d(vals_h), L.ptr_d(Bh), n, nrhs, L.ptr_d(Xh), n, 0, 10, 1e-12,
                                         C.byref(rinfo)))
        e2e_times.append(time.perf_counter() - t0)
    e2e = max_over_ranks(statistics.median(e2e_times), dist, dev)

    # independent check of the backward error of the host-path result
    import scipy.sparse as sp
    from ma57_b200 import matrices as M
    Af = M.sym_full(A)
    R = Bh - Af @ Xh
    normA = float(np.asarray(abs(sp.csr_matrix(A)).sum(axis=1)).max())
    bw = float(np.abs(R).max() / (normA * np.abs(Xh).max() + np.abs(Bh).max()))

    peaks, peak_kind = load_peaks()
    steps = max(1, args.steps)
    # the dominant kernel kind by device time, with the roofline that bounds it
    pbytes = panel_bytes(args.k) * steps
    kstats["panel"][3] = pbytes
    dom = max(kstats, key=lambda kk: kstats[kk][1])
    launches_k, ms_k, flops_k, bytes_k = kstats[dom]
    if dom in ("far_update", "near_update", "small"):
        achieved = (flops_k / (ms_k * 1e-3)) / 1e12 if ms_k > 0 else 0.0
        bf16 = peaks.get("bf16_tflops")
        if prec == L.PREC_FP64 and dom != "small":
            # FP64 on the DMMA tensor path: the bf16 figure is no denominator
            # for it; measure the FP64 tensor peak of this GPU the same way
            # (register-only MMA loop), and give the bf16 fraction beside it
            fp64 = C.c_double()
            blib = C.CDLL(os.path.join(ROOT, "ma57_b200", "lib", "libsymla_bench.so"))
            blib.symla_bench_fp64_tensor_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
            if blib.symla_bench_fp64_tensor_peak(local, C.byref(fp64)) != 0:
                raise RuntimeError("FP64 tensor peak probe failed")
            peak = fp64.value
            roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "peak_source": "FP64 DMMA (mma.sync .f64) register-only loop, measured live on this GPU "
                                       "(bench tooling, libsymla_bench.so); no FP64 figure in MEASURED_PEAKS.json",
                        "frac_of_bf16_peak": achieved / bf16 if bf16 else None,
                        "algorithmic_flops_per_launch": flops_k / max(1, launches_k)}
        else:
            peak = bf16
            roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "peak_source": f"dense bf16 tensor, {peak_kind}",
                        "algorithmic_flops_per_launch": flops_k / max(1, launches_k)}
    else:
        achieved = (bytes_k / (ms_k * 1e-3)) / 1e9 if ms_k > 0 else 0.0
        peak = peaks.get("hbm_gbs")
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "peak_source": f"HBM copy, {peak_kind}",
                    "algorithmic_bytes_per_launch": bytes_k / max(1, launches_k)}
    # DRAM traffic per launch: ncu's dram__bytes_read.sum + dram__bytes_write.sum
    # of every FP64 update launch of config 3 at k = 40 (1.257 GB per
    # factorization for 25.8 GFLOP: 0.0487 bytes per flop), scaled to this
    # run's average launch by its flops; those metrics take several replay
    # passes, so the 64^3 workload itself is not captured with them
    traffic = None
    if dom == "far_update" and prec == L.PREC_FP64:
        traffic = {"bytes_per_launch": UPDATE_DRAM_BYTES_PER_FLOP * flops_k / max(1, launches_k),
                   "source": "ncu DRAM bytes of all update launches at k=40 (0.0487 B/flop), scaled by flops"}
    roofline.update({"frac": achieved / peak if peak else None,
                     "traffic": traffic["bytes_per_launch"] if traffic else None,
                     "traffic_source": traffic["source"] if traffic else None, "kernel": dom,
                     "launches_per_step": launches_k / steps, "ms_per_step": ms_k / steps,
                     "avg_launch_us": 1e3 * ms_k / max(1, launches_k)})

    line = {
        "metric": METRIC, "value": ms / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == L.PREC_FP64 else "f64+mixed-schur", "data": "synthetic",
        "config": shared_config(args.k, nrhs),
        "details": {"precision": args.precision, "parallelism": f"replicas x{world}",
                    "l2": "inputs larger than L2 (fronts 11 GB)", "inertia": inertia,
                    "backward_error": bw, "refine_iterations": refine_iters,
                    "analyze_s": t_analyze, "factor_flops": stats.get("factor_flops"),
                    "kernel_ms_per_step": {k: v[1] / max(1, args.steps) for k, v in kstats.items()},
                    "kernel_flops_per_step": {k: v[2] / max(1, args.steps) for k, v in kstats.items() if v[2]},
                    "kernel_launches_per_step": {k: v[0] / max(1, args.steps) for k, v in kstats.items() if v[0]},
                    "panels": {k: v for k, v in stats.items() if k.startswith("panels_") or k.startswith("seq_")}},
        "precision_comparison": comparison,
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
                                "sample": f"bounded sample: oracle factorize+solve+refine on L27({args.cpu_k}^3)-3I, "
                                          f"best of 2 = {best:.3f} s, scaled by the algorithmic flop ratio {ratio:.1f} "
                                          f"(the reference arm, --impl reference, times the full 64^3 workload)"}
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
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision comparison run")
    ap.add_argument("--ref-budget", type=float, default=240.0,
                    help="reference arm: seconds of timed steps (at least one full step runs)")
    ap.add_argument("--graph", type=int, default=1, help="graph launch of the factorization's static pass")
    ap.add_argument("--workload", default="config3", choices=["config3", "dense", "batched", "learned", "configs"])
    ap.add_argument("--cpu-reps", type=int, default=5, help="configs workload: best-of repetitions on the CPU")
    ap.add_argument("--curvature-shift", type=float, default=0.0,
                    help="learned workload: 0 = config 5 as specified; c > 0 = E_k - c I (nonconvex variant)")
    ap.add_argument("--ip-steps", type=int, default=500)
    ap.add_argument("--ip-train", type=int, default=100)
    ap.add_argument("--ip-refine", default="gmres", choices=["gmres", "classic"],
                    help="learned workload: refinement towards 1e-10 (GMRES-IR or fixed-precision)")
    ap.add_argument("--n", type=int, default=4096, help="dense workload: front size")
    ap.add_argument("--systems", type=int, default=4096, help="batched workload: number of systems")
    ap.add_argument("--batch-size", type=int, default=256, help="batched workload: systems per served batch")
    ap.add_argument("--cpu-systems", type=int, default=256, help="batched workload: systems in the CPU sample")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "dense":
        run_dense(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "learned":
        run_learned(args)
    elif args.workload == "configs":
        run_configs(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
