"""Benchmark of the FP64 Cg/Bicg drop-in on one synthetic workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--size 200]

Workload (a "step"): one Cg solve of the pressure-correction Poisson system
and one Bicg solve of a momentum system, both FP64 with Jacobi
preconditioning, on a 200^3 hexahedral grid (8.0 M cells) stretched
geometrically (ratio 1.02) toward both y walls.  Seeded synthetic inputs;
the reference ships no benchmark meshes.  See the DESIGN notes for the
momentum system's Peclet number.

Metric: Mcell-iters/s = sum over solves of (cells x iterations) / time.

* value   -- solves through the library with val/x/b already in device
             memory (tf_solve_device), timed with CUDA events on the
             library's stream, max over ranks.
* e2e     -- the same solves through tf_solve with pinned host buffers:
             every step copies val, x, b host->device and back.
* roofline-- the dominant kernel (the tiled SpMV) timed alone on the same
             matrix with CUDA events; algorithmic bytes per launch
             12*nnz + 4*(n+1) + 16*n; peak = measured HBM copy bandwidth.
* cpu_baseline -- the oracle (C++ restatement of the reference, all host
             threads) on a bounded number of iterations of the same system.

`--impl reference` runs the oracle instead, on rank 0 only.
Multi-GPU runs are replicas (independent systems per rank, weak scaling).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "t-flows_b200"))

def SPMV_BYTES(n, nnz, row_patterns=False):
    """Bytes one SpMV launch must move: values, row pointers, column data,
    p once and q once.  CSR columns: 4 bytes per entry; row-pattern layout:
    one pattern byte per row."""
    cols = n if row_patterns else 4 * nnz
    return 8 * nnz + cols + 4 * (n + 1) + 16 * n


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=200)
    ap.add_argument("--peclet", type=float, default=1.0)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--batched-count", type=int, default=512,
                    help="default mode: systems of the batched leg (0: skip it)")
    ap.add_argument("--parts", default="all",
                    help="batched: comma list of mixed, fp64_batched, mixed_two_phase, drop_in, "
                         "streams, pool; served: pool, mixed (default all)")
    ap.add_argument("--rate", type=float, default=200.0, help="served: arrivals per second")
    ap.add_argument("--max-running", default="96",
                    help="served: comma list of the mixed server's system slots to run "
                         "(0: as many as requests outstanding); the first is the headline")
    ap.add_argument("--seconds", type=float, default=60.0, help="served: window length")
    ap.add_argument("--iters", type=int, default=30, help="iters: Cg iterations per solve")
    ap.add_argument("--mesh", default="hex", choices=["hex", "poly-lattice", "poly-delaunay"],
                    help="spmv: hex (--size^3 cells) or a polyhedral mesh of --cells cells")
    ap.add_argument("--cells", type=int, default=2000000)
    ap.add_argument("--tile-cfgs", default="auto",
                    help="spmv: comma list of SpMV layouts to time (tf_matrix_tile_config "
                         "ids, or auto for the tuner's choice)")
    ap.add_argument("--rcm", action="store_true",
                    help="spmv: renumber the cells by reverse Cuthill-McKee first")
    ap.add_argument("--mode", default="solve",
                    choices=["solve", "spmv", "iters", "multi", "poly", "single", "batched",
                             "served", "icc"],
                    help="spmv: only the pressure matrix and `--steps` SpMV launches "
                         "(the small case profiled with ncu); iters: `--steps` Cg solves "
                         "of exactly `--iters` iterations on the pressure matrix (launch "
                         "lists: run with TF_NO_GRAPH=1)")
    return ap.parse_args()


def _drop_in_solve_times(ctx, sysl, rel):
    """The plain FP64 drop-in, one solve at a time with inputs resident in HBM.
    tol = rel * NRMS(b): the reference's own residual measure reduced by
    `rel` from x = 0.  Returns per-solve ms (CUDA events), iterations and
    the true relative residuals."""
    import torch
    import scipy.sparse as sps
    from tflows_b200 import native, workloads
    stream = torch.cuda.ExternalStream(ctx.stream)
    out = []
    for s in sysl:
        m = native.Matrix(ctx, s.csr.row, s.csr.col, s.csr.dia)
        dval = torch.from_numpy(s.val).cuda()
        db = torch.from_numpy(s.b).cuda()
        dx = torch.zeros(s.n, dtype=torch.float64, device="cuda")
        tol = rel * workloads.nrms_b(s)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        it, res = native.solve_device(ctx, m, s.solver, "jacobi", dval.data_ptr(),
                                      dx.data_ptr(), db.data_ptr(), 100000, tol, 1.0)
        e1.record(stream)
        e1.synchronize()
        A = sps.csr_matrix((s.val, s.csr.col - 1, s.csr.row - 1), shape=(s.n, s.n))
        x = dx.cpu().numpy()
        rr = float(np.linalg.norm(s.b - A @ x) / np.linalg.norm(s.b))
        out.append((e0.elapsed_time(e1), it, rr))
        m.close()
        del dval, db, dx
    return out


def _drop_in_stream_pool(sysl, workers, rel):
    """The FP64 drop-in run from `workers` host threads, each owning a context
    (one CUDA stream), so independent solves overlap on the GPU.  Systems are
    dealt to the workers in decreasing size order; matrices are registered
    and inputs uploaded before timing.  Returns wall seconds and
    per-system (ms, iterations)."""
    import torch
    from tflows_b200 import native, workloads
    ctxs = [native.Context(0) for _ in range(workers)]
    order = sorted(range(len(sysl)), key=lambda k: -sysl[k].n)
    jobs = [[] for _ in range(workers)]
    for r, k in enumerate(order):
        w = r % workers
        s = sysl[k]
        m = native.Matrix(ctxs[w], s.csr.row, s.csr.col, s.csr.dia)
        jobs[w].append((k, s, m, torch.from_numpy(s.val).cuda(), torch.from_numpy(s.b).cuda(),
                        torch.zeros(s.n, dtype=torch.float64, device="cuda"),
                        rel * workloads.nrms_b(s)))
    torch.cuda.synchronize()
    out = [None] * len(sysl)

    def worker(w):
        for k, s, m, dval, db, dx, tol in jobs[w]:
            t0 = time.perf_counter()
            it, _ = native.solve_device(ctxs[w], m, s.solver, "jacobi", dval.data_ptr(),
                                        dx.data_ptr(), db.data_ptr(), 100000, tol, 1.0)
            out[k] = ((time.perf_counter() - t0) * 1e3, it)

    t0 = time.perf_counter()
    th = [threading.Thread(target=worker, args=(w,)) for w in range(workers)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    wall = time.perf_counter() - t0
    for jl in jobs:
        for j in jl:
            j[2].close()
    for c in ctxs:
        c.close()
    return wall, out


def _batch_solve(ctx, sysl, **opts):
    import scipy.sparse as sps
    from tflows_b200 import batch
    need = sum(12 * s.nnz + 8 * (3 * s.n) + 8 * 8 * s.n + 4096 * 4 for s in sysl)
    b = batch.Batch(ctx, mem_budget=int(need * 1.3) + (256 << 20),
                    max_systems=len(sysl) + 8, **opts)
    try:
        t0 = time.perf_counter()
        ids = b.add_many(sysl, tol=1e-10, maxit=100000)   # host preparation on all cores
        t_add = time.perf_counter() - t0
        t1 = time.perf_counter()
        b.run()
        t_run = time.perf_counter() - t1
        res = []
        for s, i in zip(sysl, ids):
            r = b.result(i)
            A = sps.csr_matrix((s.val, s.csr.col - 1, s.csr.row - 1), shape=(s.n, s.n))
            rr = float(np.linalg.norm(s.b - A @ r["x"]) / np.linalg.norm(s.b))
            res.append(dict(iters=r["iters"], status=r["status"], rel=rr, done_ms=r["done_ms"],
                            n_updates=r["n_updates"]))
        info = b.info()
        info["trace"] = b.trace()
        info["upload_ms"] = {k: round(v, 1) for k, v in b.upload_ms().items()}
        if os.environ.get("TF_BATCH_PROFILE"):
            info["kernel_ms"] = b.kernel_ms()
    finally:
        b.close()
    return t_add, t_run, res, info


def _trace_deciles(trace, vec_bytes, sweep_iters=8):
    """The sweep timeline in ten slices of equal wall time, at each slice's
    first sweep: running systems, work items, their rows and entries, the
    sweep's wall ms, and the HBM rate the sweep would reach if every listed
    system ran all its iterations (the engine's algorithmic bytes of an
    inner iteration: matrix with CSR columns or row patterns, row pointers,
    13 iterate vectors) -- an upper bound, since systems that finish inside
    the sweep stop.  When the batch was profiled, the SpMV kernel's rate
    over the CSR bytes model (entries, row pointers, p and q) is added."""
    if not trace:
        return []
    total = sum(t["ms"] for t in trace)
    out, acc, nxt = [], 0.0, 0.0
    for t in trace:
        if acc >= nxt:
            it_bytes = t["iter_bytes"]
            d = {"at_ms": round(acc, 1), "running": t["active"], "work_items": t["items"],
                 "rows": t["rows"], "nnz": t["nnz"], "sweep_ms": round(t["ms"], 3),
                 "gbs_if_all_iterate": round(sweep_iters * it_bytes / t["ms"] / 1e6, 1)}
            k = t["kernel_ms"]
            if k["spmv"] > 0:
                sp_bytes = 12 * t["nnz"] + 4 * (t["rows"] + 1) + 2 * vec_bytes * t["rows"]
                d["kernel_ms"] = {n: round(v, 3) for n, v in k.items()}
                d["spmv_gbs_if_all_iterate"] = round(sweep_iters * sp_bytes / k["spmv"] / 1e6, 1)
            out.append(d)
            nxt += total / 10
        acc += t["ms"]
    return out


def run_batched(args):
    """Many independent systems: mixed-precision batch vs the FP64 drop-in
    solving the same systems one at a time."""
    from tflows_b200 import native
    ctx = native.Context(0)
    out = batched_comparison(ctx, args.count, args.parts)
    print(json.dumps(out), flush=True)
    ctx.close()


def batched_comparison(ctx, count, parts_arg):
    """The batched workload (`count` systems): the engines named in
    parts_arg, each on the same systems, as one dict."""
    from tflows_b200 import workloads
    t0 = time.perf_counter()
    sysl = workloads.batched(count=count, seed=4)
    t_gen = time.perf_counter() - t0
    cells = sum(s.n for s in sysl)
    out = {"mode": "batched", "systems": len(sysl), "cells": cells,
           "nnz": sum(s.nnz for s in sysl), "gen_s": t_gen,
           "workload": f"{len(sysl)} systems, n log-uniform [1e3,1e6]: hex Poisson (Cg) and "
                       "polyhedral upwind convection-diffusion (Bicg, Pe U[1,50], CFL 0.1); "
                       "Jacobi; target ||b-Ax||/||b|| <= 1e-10"}
    smallest = sorted(sysl, key=lambda s: s.n)[:4]
    # A quarter of the batch first: the GPU leaves its idle clocks (after
    # the host-only legs before it) before the first timed part.
    _batch_solve(ctx, sysl[: max(1, len(sysl) // 4)], vec_fp32=True)
    parts = set(("mixed,fp64_batched,mixed_two_phase,drop_in,streams,pool"
                 if parts_arg == "all"
                 else parts_arg).split(","))
    for label, opts in (("mixed", dict(vec_fp32=True)), ("fp64_batched", dict(vec_fp32=False)),
                        ("mixed_two_phase", dict(vec_fp32=True, two_phase_rows=1))):
        if label not in parts:
            continue
        _drop = _batch_solve(ctx, smallest, **opts)   # warm-up (module load, graphs)
        t_add, t_run, res, info = _batch_solve(ctx, sysl, **opts)
        ok = sum(r["status"] == "converged" and r["rel"] <= 1.01e-10 for r in res)
        done = np.array([r["done_ms"] for r in res])
        out[label] = {"run_s": t_run, "upload_s": t_add, "solves_per_s": len(sysl) / t_run,
                      "solves_per_s_incl_upload": len(sysl) / (t_run + t_add),
                      "mcell_iters_per_s": sum(s.n * r["iters"] for s, r in zip(sysl, res))
                      / t_run / 1e6,
                      "converged_to_1e-10": ok, "max_true_rel": max(r["rel"] for r in res),
                      "done_ms_p50": float(np.percentile(done, 50)),
                      "done_ms_p99": float(np.percentile(done, 99)),
                      "sweeps": info["sweeps"],
                      "iters_total": int(sum(r["iters"] for r in res)),
                      "trace_deciles": _trace_deciles(info["trace"], 4 if opts["vec_fp32"] else 8),
                      "kernel_ms": info.get("kernel_ms"),
                      "upload_ms": info["upload_ms"]}
    if "drop_in" in parts:
        _drop_in_solve_times(ctx, smallest[:2], 1e-10)   # warm-up
        t = _drop_in_solve_times(ctx, sysl, 1e-10)
        ms = np.array([a for a, _, _ in t])
        out["fp64_drop_in"] = {"run_s": float(ms.sum() / 1e3),
            "solves_per_s": len(sysl) / float(ms.sum() / 1e3),
            "mcell_iters_per_s": sum(s.n * it for s, (_, it, _) in zip(sysl, t))
            / float(ms.sum() / 1e3) / 1e6,
            "tol": "1e-10 x NRMS(b) (reference normalisation, norm=1)",
            "max_true_rel": max(r for _, _, r in t),
            "solve_ms_p50": float(np.percentile(ms, 50)),
            "solve_ms_p99": float(np.percentile(ms, 99)),
            "iters_total": int(sum(it for _, it, _ in t))}
    for workers in ((8, 32) if "streams" in parts else ()):
        _drop_in_stream_pool(smallest, workers, 1e-10)   # warm-up
        wall, res = _drop_in_stream_pool(sysl, workers, 1e-10)
        out[f"fp64_drop_in_{workers}streams"] = {
            "run_s": wall, "solves_per_s": len(sysl) / wall,
            "mcell_iters_per_s": sum(s.n * it for s, (_, it) in zip(sysl, res)) / wall / 1e6,
            "iters_total": int(sum(it for _, it in res))}
    from tflows_b200 import pool as tpool
    for workers in ((8, 16) if "pool" in parts else ()):
        for rep in range(2):             # first pass warms the memory pool and graphs
            pl = tpool.Pool(workers=workers, mem_budget=40 << 30)
            t0 = time.perf_counter()
            rids = [pl.submit(s, miter=100000, tol=1e-10 * workloads.nrms_b(s), norm=1.0)
                    for s in sysl]
            got = [pl.wait(r) for r in rids]
            wall = time.perf_counter() - t0
            pl.close()
        lat = np.array([g["latency_ms"] for g in got])
        out[f"fp64_pool_{workers}"] = {
            "run_s_incl_upload_and_registration": wall, "solves_per_s": len(sysl) / wall,
            "mcell_iters_per_s": sum(s.n * g["niter"] for s, g in zip(sysl, got)) / wall / 1e6,
            "latency_ms_p50": float(np.percentile(lat, 50)),
            "latency_ms_p99": float(np.percentile(lat, 99)),
            "iters_total": int(sum(g["niter"] for g in got))}
    def ratio(a, b):
        if a in out and b in out:
            out[f"speedup_{a}_vs_{b}"] = out[a]["solves_per_s"] / out[b]["solves_per_s"]
    ratio("fp64_pool_16", "fp64_drop_in")
    ratio("fp64_drop_in_8streams", "fp64_drop_in")
    ratio("mixed", "fp64_drop_in")
    ratio("mixed", "fp64_batched")
    ratio("mixed", "mixed_two_phase")
    ratio("mixed", "fp64_drop_in_8streams")
    return out


def _serve_stream(req_sys, rhs, rate, seconds, workers, budget, seed, max_outstanding=256):
    """Poisson arrivals at `rate`/s for `seconds` into a request pool of
    `workers` streams.  A request that arrives while `max_outstanding` are
    queued or running is shed at the front door (counted, not submitted).
    Completion times come from the library's own latency (submit to x copied
    back); a request counts toward throughput when it completed inside the
    window.  Everything still outstanding at the end is drained before the
    pool closes."""
    import math
    from tflows_b200 import pool as tpool
    rng = np.random.default_rng(seed)
    sizes = np.array([s.n for s in req_sys])
    kinds = np.array([s.solver for s in req_sys])
    pl = tpool.Pool(workers=workers, mem_budget=budget)
    pending, results = [], []
    cv = threading.Condition()
    state = {"submitting": True, "outstanding": 0}

    def waiter():
        while True:
            with cv:
                while not pending and state["submitting"]:
                    cv.wait(0.05)
                if not pending:
                    return
                rid, t_sub, idx = pending.pop(0)
            r = pl.wait(rid)
            with cv:
                state["outstanding"] -= 1
            results.append((t_sub, r["latency_ms"], r["queue_ms"], req_sys[idx].n * r["niter"]))

    wt = threading.Thread(target=waiter)
    wt.start()
    t_start = time.perf_counter()
    stop_at = t_start + seconds
    t_next, offered, shed = t_start, 0, 0
    while True:
        t_next += rng.exponential(1.0 / rate)
        if t_next > stop_at:
            break
        delay = t_next - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        kind = "cg" if rng.random() < 0.5 else "bicg"
        n = math.exp(rng.uniform(math.log(1e4), math.log(4e6)))
        cand = np.nonzero(kinds == kind)[0]
        idx = int(cand[np.argmin(np.abs(np.log(sizes[cand]) - math.log(n)))])
        offered += 1
        with cv:
            if state["outstanding"] >= max_outstanding:
                shed += 1
                continue
            state["outstanding"] += 1
        v = offered % len(rhs[idx])
        s = req_sys[idx]
        t_sub = time.perf_counter()
        rid = pl.submit(s, b=rhs[idx][v][0], x0=np.zeros(s.n), miter=100000,
                        tol=1e-10 * rhs[idx][v][1], norm=1.0)
        with cv:
            pending.append((rid, t_sub, idx))
            cv.notify()
    with cv:
        state["submitting"] = False
        cv.notify()
    wt.join()
    stats = pl.stats()
    pl.close()
    inwin = [r for r in results if r[0] + r[1] * 1e-3 <= stop_at]
    lat = np.array([r[1] for r in inwin]) if inwin else np.zeros(1)
    qms = np.array([r[2] for r in inwin]) if inwin else np.zeros(1)
    return {"rate_per_s": rate, "seconds": seconds, "workers": workers,
            "offered": offered, "shed": shed, "admitted": offered - shed,
            "completed_in_window": len(inwin),
            "solves_per_s": len(inwin) / seconds,
            "mcell_iters_per_s": sum(r[3] for r in inwin) / seconds / 1e6,
            "latency_ms_p50": float(np.percentile(lat, 50)),
            "latency_ms_p99": float(np.percentile(lat, 99)),
            "queue_ms_p50": float(np.percentile(qms, 50)),
            "peak_device_bytes": stats["peak_bytes"]}


def _serve_stream_mixed(req_sys, rhs, rate, seconds, budget, seed, max_outstanding=256,
                        submit_threads=8, max_running=0):
    """The same Poisson stream into the continuous-batching server
    (tf_server_*: the mixed-precision engine, requests admitted into free
    slots between sweeps, Krylov state resident).  Submission copies and
    prepares each system on the caller's thread, so arrivals are handed to
    `submit_threads` submitter threads.  Latency is counted from arrival:
    time until the submit call returned plus the server's own latency
    (submit to result)."""
    import concurrent.futures as cf
    import copy
    import math
    from tflows_b200 import batch, native
    rng = np.random.default_rng(seed)
    sizes = np.array([s.n for s in req_sys])
    kinds = np.array([s.solver for s in req_sys])
    ctx = native.Context(0)
    # max_running: the server's system slots (0: every outstanding request
    # can be admitted); fewer slots keep large requests from being spread
    # over a crowded sweep, at the price of waits in the queue.
    srv = batch.Server(ctx, mem_budget=budget,
                       max_systems=max_running if max_running > 0 else max_outstanding + 8,
                       sweep_iters=8)
    results, lock = [], threading.Lock()
    state = {"outstanding": 0}

    def handle(t_arr, idx, v):
        s = copy.copy(req_sys[idx])
        s.b = rhs[idx][v][0]
        s.x0 = np.zeros(s.n)
        try:
            rid = srv.submit(s, tol=1e-10, maxit=100000)
            t_ret = time.perf_counter()
            r = srv.wait(rid)
            ok = r["status"] == "converged"
            lat = (t_ret - t_arr) * 1e3 + r["latency_ms"]
            with lock:
                results.append((t_arr, lat, r["queue_ms"], s.n * r["iters"], ok))
        finally:
            with lock:
                state["outstanding"] -= 1

    ex = cf.ThreadPoolExecutor(max_outstanding + submit_threads)
    t_start = time.perf_counter()
    stop_at = t_start + seconds
    t_next, offered, shed = t_start, 0, 0
    futs = []
    while True:
        t_next += rng.exponential(1.0 / rate)
        if t_next > stop_at:
            break
        delay = t_next - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        kind = "cg" if rng.random() < 0.5 else "bicg"
        n = math.exp(rng.uniform(math.log(1e4), math.log(4e6)))
        cand = np.nonzero(kinds == kind)[0]
        idx = int(cand[np.argmin(np.abs(np.log(sizes[cand]) - math.log(n)))])
        offered += 1
        with lock:
            if state["outstanding"] >= max_outstanding:
                shed += 1
                continue
            state["outstanding"] += 1
        futs.append(ex.submit(handle, time.perf_counter(), idx, offered % len(rhs[idx])))
    for f in futs:
        f.result()
    ex.shutdown()
    st = srv.stats()
    timing = srv.timing()
    srv.close()
    ctx.close()
    inwin = [r for r in results if r[0] + r[1] * 1e-3 <= stop_at]
    lat = np.array([r[1] for r in inwin]) if inwin else np.zeros(1)
    qms = np.array([r[2] for r in inwin]) if inwin else np.zeros(1)
    return {"rate_per_s": rate, "seconds": seconds, "submit_threads": submit_threads,
            "offered": offered, "shed": shed, "admitted": offered - shed,
            "completed_in_window": len(inwin),
            "converged_to_1e-10": int(sum(r[4] for r in inwin)),
            "solves_per_s": len(inwin) / seconds,
            "mcell_iters_per_s": sum(r[3] for r in inwin) / seconds / 1e6,
            "latency_ms_p50": float(np.percentile(lat, 50)),
            "latency_ms_p99": float(np.percentile(lat, 99)),
            "queue_ms_p50": float(np.percentile(qms, 50)),
            "peak_running": st["peak_running"], "sweeps": st["sweeps"], "server_ms": timing}


def run_served(args):
    """Served stream through the request pool (each request one Solve_Native
    on the FP64 drop-in): Poisson arrivals at `--rate`/s of hex Poisson (Cg)
    and polyhedral convection-diffusion (Bicg) systems, n log-uniform in
    [1e4, 4e6], 20 GB device budget.  Compared with the same stream served
    one request at a time (one stream), and with the pool at half its
    measured saturation throughput for latency under a sustainable load."""
    from tflows_b200 import systems, workloads
    t0 = time.perf_counter()
    req_sys = workloads.served_pool(seed=5, per_kind=8)
    rhs = {}
    for k, s in enumerate(req_sys):
        a = s.val[s.csr.dia - 1]
        rhs[k] = []
        for v in range(3):
            b = systems.uniform_rhs(s.n, 7000 + 10 * k + v, zero_mean=(s.solver == "cg"))
            rhs[k].append((b, float(np.sqrt(np.sum((b / a) ** 2)))))
    out = {"mode": "served", "gen_s": time.perf_counter() - t0,
           "request_systems": [(s.name, s.n) for s in req_sys],
           "workload": "Poisson arrivals; each request a hex Poisson (Cg) or polyhedral "
                       "convection-diffusion (Bicg) system, n log-uniform [1e4, 4e6] "
                       "(nearest of 16 pre-generated systems), seeded RHS, x0 = 0, "
                       "tol 1e-10 x NRMS(b); FP64 Jacobi drop-in per request; 20 GB budget; "
                       "at most 256 requests outstanding (the rest shed)"}
    budget = 20 << 30
    parts = set(args.parts.split(",")) if args.parts != "all" else {"pool", "mixed"}
    if "pool" in parts:
        _serve_stream(req_sys, rhs, 5.0, 3.0, 8, budget, 1)          # warm-up
        sat = _serve_stream(req_sys, rhs, args.rate, args.seconds, 8, budget, 2)
        out["pool_8_streams"] = sat
        out["one_at_a_time"] = _serve_stream(req_sys, rhs, args.rate, args.seconds / 2, 1,
                                             budget, 2)
        light = max(1.0, 0.5 * sat["solves_per_s"])
        out["pool_8_streams_half_load"] = _serve_stream(req_sys, rhs, light, args.seconds / 2,
                                                        8, budget, 3)
        out["throughput_ratio_pool_vs_one_at_a_time"] = (
            sat["solves_per_s"] / max(out["one_at_a_time"]["solves_per_s"], 1e-9))
    if "mixed" in parts:
        # The mixed-precision continuous-batching server on the same streams
        # (tol: ||b - A x|| / ||b|| <= 1e-10 in FP64).
        _serve_stream_mixed(req_sys, rhs, 5.0, 3.0, budget, 1)     # warm-up
        for k, cap in enumerate(int(c) for c in args.max_running.split(",")):
            tag = "" if k == 0 else f"_max_running_{cap}"
            mixed_k = _serve_stream_mixed(req_sys, rhs, args.rate, args.seconds, budget, 2,
                                          max_running=cap)
            mixed_k["max_running"] = cap
            out["mixed_server" + tag] = mixed_k
            if k == 0:
                mixed = mixed_k
        out["mixed_server_half_load"] = _serve_stream_mixed(
            req_sys, rhs, max(1.0, 0.5 * mixed["solves_per_s"]), args.seconds / 2, budget, 3,
            max_running=int(args.max_running.split(",")[0]))
    if "pool" in parts and "mixed" in parts:
        out["throughput_ratio_mixed_server_vs_one_at_a_time"] = (
            mixed["solves_per_s"] / max(out["one_at_a_time"]["solves_per_s"], 1e-9))
        out["throughput_ratio_mixed_server_vs_pool"] = (
            mixed["solves_per_s"] / max(sat["solves_per_s"], 1e-9))
    print(json.dumps(out), flush=True)


def run_spmv_only(args):
    """Register the pressure matrix and launch the tiled SpMV --steps times."""
    import torch
    from tflows_b200 import native, systems
    from tflows_b200.grids import hex_grid, poly_dual_grid, poly_lattice_grid
    if args.mesh == "hex":
        g = hex_grid(args.size, args.size, args.size, stretch_y=1.02)
    elif args.mesh == "poly-lattice":
        g = poly_lattice_grid(args.cells, 3)
    else:
        g = poly_dual_grid(args.cells, 3)
    s = systems.pressure_system(g, 2, tol=1e-10, miter=1, singular="pin", norm=1.0)
    if args.rcm:
        s = systems.renumber_rcm(s)
    ctx = native.Context(0)
    val = torch.from_numpy(s.val).cuda()
    p = torch.randn(s.n, dtype=torch.float64, device="cuda")
    q = torch.empty_like(p)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream)
    peak, peak_kind = measured_peak()
    # --tile-cfgs: each layout in turn (TF_TILE_CFG at registration); "auto":
    # the layout the tuner picks.
    for cfg in args.tile_cfgs.split(","):
        if cfg == "auto":
            os.environ.pop("TF_TILE_CFG", None)
        else:
            os.environ["TF_TILE_CFG"] = cfg
        m = native.Matrix(ctx, s.csr.row, s.csr.col, s.csr.dia)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        native.spmv(ctx, m, val.data_ptr(), p.data_ptr(), q.data_ptr())
        e0.record(stream)
        for _ in range(args.steps):
            native.spmv(ctx, m, val.data_ptr(), p.data_ptr(), q.data_ptr())
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / max(args.steps, 1)
        by = SPMV_BYTES(s.n, s.nnz, m.row_patterns > 0)
        print(json.dumps({"mode": "spmv", "mesh": args.mesh, "n": s.n, "nnz": s.nnz,
                          "requested": cfg, "tile_cfg": m.tile_config,
                          "row_patterns": m.row_patterns, "tuning": m.tuning(),
                          "launch_ms": t * 1e3, "bytes_per_launch": by,
                          "csr_bytes_per_launch": SPMV_BYTES(s.n, s.nnz),
                          "achieved_gbs": by / t / 1e9, "frac": by / t / 1e9 / peak,
                          "peak_kind": peak_kind}), flush=True)
        m.close()
    os.environ.pop("TF_TILE_CFG", None)
    ctx.close()


def run_fixed_iterations(args):
    """`--steps` Cg + Jacobi solves of exactly `--iters` iterations (tol 0)
    on the bench's pressure matrix: per-iteration time with CUDA events."""
    import torch
    from tflows_b200 import native, systems
    from tflows_b200.grids import poly_dual_grid, poly_lattice_grid
    if args.mesh == "hex":
        p = make_workload(args.size, args.peclet)[0]
    else:
        g = (poly_lattice_grid(args.cells, 3) if args.mesh == "poly-lattice"
             else poly_dual_grid(args.cells, 3))
        p = systems.pressure_system(g, 2, tol=1e-10, miter=1, singular="pin", norm=1.0)
    ctx = native.Context(0)
    m = native.Matrix(ctx, p.csr.row, p.csr.col, p.csr.dia)
    stream = torch.cuda.ExternalStream(ctx.stream)
    val0, b0 = torch.from_numpy(p.val).cuda(), torch.from_numpy(p.b).cuda()
    val, b = val0.clone(), b0.clone()
    x = torch.zeros(p.n, dtype=torch.float64, device="cuda")
    out = []
    for _ in range(args.steps):
        val.copy_(val0)
        b.copy_(b0)
        x.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        it, _ = native.solve_device(ctx, m, "cg", "jacobi", val.data_ptr(), x.data_ptr(),
                                    b.data_ptr(), args.iters, 0.0, 1.0)
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1) / it * 1e3)
    print(json.dumps({"mode": "iters", "mesh": args.mesh, "n": p.n, "nnz": p.nnz,
                      "iters": args.iters, "row_patterns": m.row_patterns,
                      "renumbered": m.renumbered, "us_per_iteration": out,
                      "mcell_iters_per_s": p.n / min(out)}), flush=True)
    m.close()
    ctx.close()


def run_icc(args):
    """The reference's default preconditioner (incomplete Cholesky,
    Prec_Form.f90:68-78, Prec_Solve.f90:64-92) against Jacobi on the bench's
    pressure matrix (--size^3 stretched hex): iterations, time per solve and
    per iteration, and the kernel launches per iteration."""
    import torch
    from tflows_b200 import native
    p = make_workload(args.size, args.peclet)[0]
    ctx = native.Context(0)
    m = native.Matrix(ctx, p.csr.row, p.csr.col, p.csr.dia)
    stream = torch.cuda.ExternalStream(ctx.stream)
    val0, b0 = torch.from_numpy(p.val).cuda(), torch.from_numpy(p.b).cuda()
    out = {"mode": "icc", "n": p.n, "nnz": p.nnz, "tol": p.tol,
           "levels": m.icc_levels()}
    for prec in ("jacobi", "icc"):
        best = None
        for _ in range(max(1, args.steps)):
            val, b = val0.clone(), b0.clone()
            x = torch.zeros(p.n, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            it, res = native.solve_device(ctx, m, "cg", prec, val.data_ptr(), x.data_ptr(),
                                          b.data_ptr(), p.miter, p.tol, p.norm)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            if best is None or ms < best[0]:
                best = (ms, it, res)
        out[prec] = {"ms": best[0], "iters": best[1], "fin_res": best[2],
                     "us_per_iteration": 1e3 * best[0] / max(best[1], 1)}
    lv = out["levels"]
    out["jacobi"]["launches_per_iteration"] = 3
    out["icc"]["launches_per_iteration"] = m.icc_launches_per_iteration()
    out["icc_vs_jacobi_time"] = out["icc"]["ms"] / out["jacobi"]["ms"]
    print(json.dumps(out), flush=True)
    m.close()
    ctx.close()


def run_multi_rhs(args):
    """Three velocity components with one momentum matrix (the bench's
    200^3 Bicg system, three seeded right-hand sides): one tf_solve_multi
    against three tf_solve_device calls, CUDA events, inputs in HBM."""
    import torch
    from tflows_b200 import native, systems
    msys = make_workload(args.size, args.peclet)[1]
    ctx = native.Context(0)
    m = native.Matrix(ctx, msys.csr.row, msys.csr.col, msys.csr.dia)
    stream = torch.cuda.ExternalStream(ctx.stream)
    n = msys.n
    B = np.stack([systems.uniform_rhs(n, 40 + k, zero_mean=False) for k in range(3)])
    val0 = torch.from_numpy(msys.val).cuda()
    B0 = torch.from_numpy(np.ascontiguousarray(B)).cuda()
    val, Bd = val0.clone(), B0.clone()
    X = torch.zeros((3, n), dtype=torch.float64, device="cuda")
    tol, miter, norm = msys.tol, msys.miter, msys.norm

    def timed(fn):
        val.copy_(val0)
        Bd.copy_(B0)
        X.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        its = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), its

    def multi():
        return native.solve_multi_device(ctx, m, "bicg", "jacobi", 3, val.data_ptr(),
                                         X.data_ptr(), Bd.data_ptr(), miter, tol, norm)[0]

    def singles():
        its = []
        for k in range(3):
            it, _ = native.solve_device(ctx, m, "bicg", "jacobi", val.data_ptr(),
                                        X[k].data_ptr(), Bd[k].data_ptr(), miter, tol, norm)
            its.append(it)
        return its

    for _ in range(2):
        timed(multi)
        timed(singles)
    tm, im = min(timed(multi) for _ in range(args.steps))
    ts, is_ = min(timed(singles) for _ in range(args.steps))
    cells = n * sum(im)
    print(json.dumps({"mode": "multi", "n": n, "nnz": msys.nnz, "rhs": 3,
                      "iters_multi": im, "iters_single": is_,
                      "ms_multi": tm, "ms_three_singles": ts, "speedup": ts / tm,
                      "mcell_iters_per_s_multi": cells / tm / 1e3,
                      "mcell_iters_per_s_singles": n * sum(is_) / ts / 1e3}), flush=True)
    m.close()
    ctx.close()


def run_poly_system(args):
    """One large polyhedral Poisson system (the dual of a seeded random
    Delaunay tetrahedralisation, --cells points, numbered by sorted
    centres): the FP64 drop-in against the batch engine with FP64 and with
    FP32 iterates, all to ||b - A x|| / ||b|| <= 1e-10 in FP64."""
    import scipy.sparse as sps
    import torch
    from tflows_b200 import native, systems, workloads
    from tflows_b200.grids import poly_dual_grid, poly_lattice_grid
    t0 = time.perf_counter()
    g = (poly_dual_grid(args.cells, 3) if args.mesh != "poly-lattice"
         else poly_lattice_grid(args.cells, 3))
    s = systems.pressure_system(g, 3, tol=1e-10, miter=100000, singular="pin", norm=1.0,
                                name=f"poly-{args.mesh}-{g.n_cells}")
    gen = time.perf_counter() - t0
    A = sps.csr_matrix((s.val, s.csr.col - 1, s.csr.row - 1), shape=(s.n, s.n))
    rel = lambda x: float(np.linalg.norm(s.b - A @ x) / np.linalg.norm(s.b))  # noqa: E731
    ctx = native.Context(0)
    mesh = "poly-lattice" if args.mesh == "poly-lattice" else "poly-delaunay"
    out = {"mode": "poly", "mesh": mesh, "n": s.n, "nnz": s.nnz, "gen_s": gen}
    # FP64 drop-in.  Its stopping test is the reference's NRMS, which on a
    # mesh with widely varying cell sizes differs from the true relative
    # residual by orders of magnitude: tol is calibrated (tightened until
    # ||b - A x|| / ||b|| <= 1e-10) before the timed runs.
    m = native.Matrix(ctx, s.csr.row, s.csr.col, s.csr.dia)
    out["renumbered"] = m.renumbered
    stream = torch.cuda.ExternalStream(ctx.stream)
    dval, db = torch.from_numpy(s.val).cuda(), torch.from_numpy(s.b).cuda()

    def drop_in(tol):
        v, b = dval.clone(), db.clone()
        x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        it, _ = native.solve_device(ctx, m, "cg", "jacobi", v.data_ptr(), x.data_ptr(),
                                    b.data_ptr(), 100000, tol, 1.0)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), it, rel(x.cpu().numpy())

    tol = 1e-10 * workloads.nrms_b(s)
    for _ in range(6):
        _, _, r = drop_in(tol)
        if r <= 1e-10:
            break
        tol *= 0.5 * 1e-10 / r
    out["fp64_drop_in_tol"] = tol
    best = min((drop_in(tol) for _ in range(max(1, args.steps))), key=lambda t: t[0])
    m.close()
    out["fp64_drop_in"] = {"ms": best[0], "iters": best[1], "true_rel": best[2],
                           "mcell_iters_per_s": s.n * best[1] / best[0] / 1e3}
    for label, opts in (("batch_fp64", dict(vec_fp32=False)), ("batch_mixed", dict(vec_fp32=True)),
                        ("batch_mixed_two_phase", dict(vec_fp32=True, two_phase_rows=1))):
        runs = [_batch_solve(ctx, [s], **opts) for _ in range(1 + args.steps)][1:]
        t_add, t_run, res, info = min(runs, key=lambda r: r[1])
        out[label] = {"ms": t_run * 1e3, "iters": res[0]["iters"], "true_rel": res[0]["rel"],
                      "status": res[0]["status"], "refinements": res[0]["n_updates"],
                      "mcell_iters_per_s": s.n * res[0]["iters"] / t_run / 1e6}
    print(json.dumps(out), flush=True)
    ctx.close()


def run_single_hex(args):
    """One large hex Poisson system (--size^3, stretched 1.02 toward the y
    walls, seed 5) in the batch engine with FP32 iterates and in the FP64
    drop-in, both to ||b - A x|| / ||b|| <= 1e-10: time per iteration (the
    case profiled for the batch SpMV; a small batch warms the engine up)."""
    from tflows_b200 import native, systems
    s = systems.small_hex(args.size, seed=5, kind="pressure", ratio=1.02, tol=1e-10,
                          miter=100000)
    ctx = native.Context(0)
    _batch_solve(ctx, [systems.small_hex(8, seed=1, kind="pressure")], vec_fp32=True)
    t_add, t_run, res, info = _batch_solve(ctx, [s], vec_fp32=True)
    out = {"mode": "single", "mesh": "hex", "n": s.n, "nnz": s.nnz,
           "batch_mixed": {"ms": t_run * 1e3, "iters": res[0]["iters"],
                           "us_per_iteration": t_run * 1e6 / res[0]["iters"],
                           "true_rel": res[0]["rel"], "kernel_ms": info.get("kernel_ms")}}
    if not os.environ.get("TF_BATCH_PROFILE"):
        _drop_in_solve_times(ctx, [systems.small_hex(8, seed=1, kind="pressure")], 1e-10)
        ms, it, rel = _drop_in_solve_times(ctx, [s], 1e-10)[0]
        out["fp64_drop_in"] = {"ms": ms, "iters": it, "us_per_iteration": ms * 1e3 / it,
                               "true_rel": rel}
    print(json.dumps(out), flush=True)
    ctx.close()


def dist_env():
    from tflows_b200.replicas import dist_env as env
    return env()


def make_workload(size, peclet):
    from tflows_b200 import systems
    p, m = systems.stretched_pair(n=size, seed=2, tol=1e-10, miter=20000, ratio=1.02,
                                  peclet=peclet, momentum_miter=2000)
    return [p, m]


def workload_config(sysl, size, peclet):
    p = sysl[0]
    return {
        "workload": f"stretched-hex-{size}^3 (ratio 1.02 toward both y walls): Cg pressure "
                    f"Poisson (one pressure-boundary face pins the level) + Bicg upwind "
                    f"momentum (cell Peclet {peclet:g}, CFL 0.5); FP64, Jacobi, tol 1e-10 "
                    f"(reference NRMS with norm=1)",
        "n_cells": p.n, "nnz": p.nnz, "solves_per_step": len(sysl),
        "l2_policy": f"inputs larger than L2 (val {8 * p.nnz / 1e6:.0f} MB per system)",
        "parallelism": "replicas",
    }


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(size):
    """DRAM bytes per SpMV launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"spmv_fp64_stretched{size}.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def cpu_baseline(sysl, seconds, threads):
    """Oracle Cg on a bounded number of iterations of the pressure system."""
    from oracle import oracle as O
    s = sysl[0]

    def run(k):
        v, x, b = s.val.copy(), s.x0.copy(), s.b.copy()
        t0 = time.perf_counter()
        r = O.solve_native("cg", "jacobi", s.csr.row, s.csr.col, s.csr.dia, v, x, b, k, 0.0,
                           norm=1.0, threads=threads)
        return time.perf_counter() - t0, r["niter"]

    t1, _ = run(2)
    t3, _ = run(6)
    per_it = max((t3 - t1) / 4, 1e-6)
    k = int(max(4, min(2000, seconds / per_it)))
    t, it = run(k)
    return {"value": s.n * it / t / 1e6, "unit": "Mcell-iters/s", "cores": threads,
            "kind": "port",
            "sample": f"oracle Cg+Jacobi, {it} iterations of the {s.n}-cell pressure system "
                      f"(tol 0 -> fixed count), {t:.1f} s wall, OpenMP {threads} threads"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import oracle as O
    sysl = make_workload(args.size, args.peclet)
    threads = O.max_threads()
    sample_iters = int(os.environ.get("TF_REF_ITERS", "40"))

    def step():
        tot = 0
        for s in sysl:
            v, x, b = s.val.copy(), s.x0.copy(), s.b.copy()
            r = O.solve_native(s.solver, s.prec, s.csr.row, s.csr.col, s.csr.dia, v, x, b,
                               sample_iters, s.tol, norm=s.norm, threads=threads)
            tot += s.n * r["niter"]
        return tot

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    cells = sum(step() for _ in range(args.steps))
    dt = time.perf_counter() - t0
    val = cells / dt / 1e6
    line = {
        "impl": "reference", "metric": "Mcell-iters/s", "value": val, "unit": "Mcell-iters/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": workload_config(sysl, args.size, args.peclet),
        "cpu_baseline": {"value": val, "unit": "Mcell-iters/s", "cores": threads,
                         "kind": "port",
                         "sample": f"each step: {sample_iters} iterations (bounded) of "
                                   f"each of the {len(sysl)} solves"},
        "e2e": {"value": val, "unit": "Mcell-iters/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.mode == "spmv":
        run_spmv_only(args)
        return
    if args.mode == "icc":
        run_icc(args)
        return
    if args.mode == "iters":
        run_fixed_iterations(args)
        return
    if args.mode == "multi":
        run_multi_rhs(args)
        return
    if args.mode == "poly":
        run_poly_system(args)
        return
    if args.mode == "single":
        run_single_hex(args)
        return
    if args.mode == "batched":
        run_batched(args)
        return
    if args.mode == "served":
        run_served(args)
        return

    import torch
    from tflows_b200 import native, replicas

    torch.cuda.set_device(local)
    rep = replicas.Replicas("nccl")
    barrier, allmax, allsum = rep.barrier, rep.max, rep.sum

    sysl = make_workload(args.size, args.peclet)
    ctx = native.Context(local)
    mats = [native.Matrix(ctx, s.csr.row, s.csr.col, s.csr.dia) for s in sysl]
    stream = torch.cuda.ExternalStream(ctx.stream)

    # Device-resident inputs (pristine copies) and work buffers.
    dev = []
    for s in sysl:
        d = {k: torch.from_numpy(np.ascontiguousarray(a)).cuda()
             for k, a in (("val0", s.val), ("b0", s.b), ("x0", s.x0))}
        d.update(val=d["val0"].clone(), b=d["b0"].clone(), x=d["x0"].clone())
        dev.append(d)
    torch.cuda.synchronize()

    results = {}

    sys_ev = [[] for _ in sysl]   # per-system (start, end) events of the timed steps

    def device_step(record=False):
        cells, its = 0, []
        with torch.cuda.stream(stream):
            for k, (s, m, d) in enumerate(zip(sysl, mats, dev)):
                d["x"].copy_(d["x0"])
                if record:
                    ea = torch.cuda.Event(enable_timing=True)
                    ea.record(stream)
                it, res = native.solve_device(ctx, m, s.solver, s.prec, d["val"].data_ptr(),
                                              d["x"].data_ptr(), d["b"].data_ptr(), s.miter,
                                              s.tol, s.norm)
                if record:
                    eb = torch.cuda.Event(enable_timing=True)
                    eb.record(stream)
                    sys_ev[k].append((ea, eb))
                cells += s.n * it
                its.append((it, res))
        return cells, its

    for _ in range(args.warmup):
        device_step()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    per_solve = []
    ev0.record(stream)
    cells = 0
    iters = None
    for _ in range(args.steps):
        e_a = torch.cuda.Event(enable_timing=True)
        e_a.record(stream)
        c, its = device_step(record=True)
        e_b = torch.cuda.Event(enable_timing=True)
        e_b.record(stream)
        per_solve.append((e_a, e_b))
        cells += c
        iters = its
    ev1.record(stream)
    barrier()
    clk = clocks.stop()
    t_dev = ev0.elapsed_time(ev1) / 1e3
    t_dev_max = allmax(t_dev)
    cells_all = allsum(cells)
    step_ms = [a.elapsed_time(b) for a, b in per_solve]
    per_system_ms = [sum(a.elapsed_time(b) for a, b in evs) for evs in sys_ev]

    # End-to-end through tf_solve with pinned host buffers.
    host = []
    for s in sysl:
        h = {k: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
             for k, a in (("val", s.val), ("b", s.b), ("x", s.x0))}
        host.append(h)
    h2d = sum(8 * s.nnz + 16 * s.n for s in sysl)
    d2h = h2d

    def e2e_step():
        c = 0
        for s, m, h in zip(sysl, mats, host):
            np.copyto(h["val"], s.val)
            np.copyto(h["b"], s.b)
            np.copyto(h["x"], s.x0)
            it, res = native.solve(ctx, m, s.solver, s.prec, h["val"], h["x"], h["b"],
                                   s.miter, s.tol, s.norm)
            c += s.n * it
        return c

    e2e_step()
    barrier()
    e2e_cells, t_e2e = 0, 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_cells += e2e_step()
        t_e2e += time.perf_counter() - t0
    t_e2e_max = allmax(t_e2e)
    e2e_all = allsum(e2e_cells)

    # Accuracy of the last device solve: true relative residual in FP64.
    import scipy.sparse as sps
    acc = []
    for s, d, (it, res) in zip(sysl, dev, iters):
        A = sps.csr_matrix((s.val, s.csr.col - 1, s.csr.row - 1), shape=(s.n, s.n))
        x = d["x"].cpu().numpy()
        rr = np.linalg.norm(s.b - A @ x) / np.linalg.norm(s.b)
        acc.append({"system": s.name, "solver": s.solver, "niter": it, "fin_res": res,
                    "true_rel_residual": float(rr)})

    # Roofline of the dominant kernel: the tiled SpMV on the pressure matrix.
    s0, m0, d0 = sysl[0], mats[0], dev[0]
    p = torch.randn(s0.n, dtype=torch.float64, device="cuda")
    q = torch.empty_like(p)
    torch.cuda.synchronize()
    nrep = 20
    for _ in range(3):
        native.spmv(ctx, m0, d0["val0"].data_ptr(), p.data_ptr(), q.data_ptr())
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    for _ in range(nrep):
        native.spmv(ctx, m0, d0["val0"].data_ptr(), p.data_ptr(), q.data_ptr())
    r1.record(stream)
    r1.synchronize()
    t_spmv = r0.elapsed_time(r1) / 1e3 / nrep
    peak, peak_kind = measured_peak()
    pat = m0.row_patterns > 0
    bytes_spmv = SPMV_BYTES(s0.n, s0.nnz, pat)
    achieved = bytes_spmv / t_spmv / 1e9
    # Whole Cg iteration (pressure solve): the SpMV, k_update (read r, q,
    # diag; write r) and k_pupdate (read r, diag, p, x; write p, x).
    it_p = iters[0][0] * args.steps
    t_iter = per_system_ms[0] / 1e3 / max(it_p, 1) if per_system_ms else None
    bytes_iter = bytes_spmv + 32 * s0.n + 48 * s0.n

    launches = sum(args.steps * (4 + 3 * it) for it, _ in iters)

    if rank == 0:
        cpu = cpu1 = None
        if not args.no_cpu_baseline and world == 1:
            from oracle import oracle as O
            cpu = cpu_baseline(sysl, args.cpu_seconds, O.max_threads())
            cpu1 = cpu_baseline(sysl, args.cpu_seconds / 2, 1)
        batched = None
        if world == 1 and args.batched_count > 0:
            # The batched workload (512 systems): the mixed-precision batch
            # engine against the FP64 drop-in one request at a time and on 8
            # concurrent streams, same systems, same run.
            b = batched_comparison(ctx, args.batched_count, "mixed,drop_in,streams")
            keep = ("run_s", "upload_s", "solves_per_s", "solves_per_s_incl_upload",
                    "mcell_iters_per_s", "converged_to_1e-10", "max_true_rel",
                    "done_ms_p50", "done_ms_p99", "solve_ms_p50", "solve_ms_p99",
                    "iters_total")
            batched = {"workload": b["workload"], "systems": b["systems"], "cells": b["cells"],
                       "nnz": b["nnz"]}
            for k in ("mixed", "fp64_drop_in", "fp64_drop_in_8streams"):
                if k in b:
                    batched[k] = {kk: v for kk, v in b[k].items() if kk in keep}
            for k, v in b.items():
                if k.startswith("speedup_"):
                    batched[k] = v
        ms = np.array(step_ms)
        solve_count = args.steps * len(sysl) * world
        line = {
            "metric": "Mcell-iters/s", "value": cells_all / t_dev_max / 1e6,
            "unit": "Mcell-iters/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_dev_max / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded stretched hex grid; no reference dataset exists)",
            "config": workload_config(sysl, args.size, args.peclet),
            "solves_per_s": solve_count / t_dev_max,
            "step_ms_p50": float(np.percentile(ms, 50)),
            "step_ms_p99": float(np.percentile(ms, 99)),
            "accuracy": acc,
            "e2e": {"value": e2e_all / t_e2e_max / 1e6, "unit": "Mcell-iters/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm",
                         "kernel": "k_spmv_alpha (tiled SpMV + p.q, "
                                   + ("row-pattern columns)" if pat else "CSR columns)"),
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "bytes_per_launch": bytes_spmv,
                         "csr_bytes_per_launch": SPMV_BYTES(s0.n, s0.nnz),
                         "launch_ms": t_spmv * 1e3,
                         "traffic": ncu_traffic(args.size),
                         "cg_iteration": None if not t_iter else {
                             "bytes": bytes_iter, "us": t_iter * 1e6,
                             "achieved": bytes_iter / t_iter / 1e9,
                             "frac": bytes_iter / t_iter / 1e9 / peak}},
            "cpu_baseline": cpu,
            "cpu_baseline_1core": cpu1,
            "batched": batched,
            "clocks": clk,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)

    for m in mats:
        m.close()
    ctx.close()
    rep.close()


if __name__ == "__main__":
    main()
