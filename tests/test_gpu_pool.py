"""GPU tests of the request pool: concurrent Solve_Native calls on several
streams give exactly the results of tf_solve on the same inputs (the pool
runs the same deterministic drop-in), under a device-memory budget."""
import copy
import threading

import numpy as np
import pytest

from tflows_b200 import native, pool, systems

pytestmark = pytest.mark.gpu


def _systems():
    return [systems.small_hex(12, seed=1, kind="pressure", ratio=1.02),
            systems.small_hex(24, seed=2, kind="pressure", ratio=1.02),
            systems.small_hex(10, seed=3, kind="momentum", peclet=1.0),
            systems.poly_system(2000, seed=4, kind="pressure"),
            systems.small_hex(8, seed=5, kind="pressure", tol=1e-9, miter=300, prec="icc")]


def _reference(ctx, s):
    m = native.Matrix(ctx, s.csr.row, s.csr.col, s.csr.dia)
    try:
        v, x, b = s.val.copy(), s.x0.copy(), s.b.copy()
        it, res = native.solve(ctx, m, s.solver, s.prec, v, x, b, s.miter, s.tol, s.norm)
        return x, it, res
    finally:
        m.close()


def test_pool_matches_single_solves(gpu_ctx):
    sysl = _systems()
    ref = [_reference(gpu_ctx, s) for s in sysl]
    p = pool.Pool(workers=4, mem_budget=1 << 30)
    try:
        rids = {}

        def submitter(offset):
            for k in range(offset, 3 * len(sysl), 2):
                rids[k] = p.submit(sysl[k % len(sysl)])

        th = [threading.Thread(target=submitter, args=(o,)) for o in (0, 1)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for k in sorted(rids):
            r = p.wait(rids[k])
            x, it, res = ref[k % len(sysl)]
            assert r["niter"] == it and r["fin_res"] == res
            assert np.array_equal(r["x"], x)
            assert r["latency_ms"] >= r["queue_ms"] >= 0.0
        st = p.stats()
        assert st["completed"] == 3 * len(sysl) and st["rejected"] == 0
        assert 0 < st["peak_bytes"] <= 1 << 30
    finally:
        p.close()


def test_pool_budget(gpu_ctx):
    small = systems.small_hex(6, seed=1, kind="pressure")
    big = systems.small_hex(40, seed=1, kind="pressure")
    p = pool.Pool(workers=2, mem_budget=4 << 20)
    try:
        r_big = p.submit(big)
        r_small = p.submit(small)
        with pytest.raises(native.TFError) as e:
            p.wait(r_big)
        assert e.value.status == 2          # TF_ERR_OOM: larger than the budget
        assert p.wait(r_small)["niter"] > 0
        assert p.stats()["rejected"] == 1
    finally:
        p.close()


def test_pool_reuses_resident_structures(gpu_ctx):
    """Requests on the same Matrix_Type arrays run on the held registration
    (no re-registration) and give the single-solve results every time, also
    with fresh right-hand sides."""
    s = systems.small_hex(20, seed=7, kind="pressure", ratio=1.03)
    rhs = [systems.uniform_rhs(s.n, 100 + k, zero_mean=True) for k in range(6)]
    refs = []
    for b in rhs:
        t = copy.copy(s)
        t.b = b
        refs.append(_reference(gpu_ctx, t))
    p = pool.Pool(workers=2, mem_budget=1 << 30)
    try:
        for rounds in range(2):
            rids = [p.submit(s, b=b) for b in rhs]
            for rid, (x, it, res) in zip(rids, refs):
                r = p.wait(rid)
                assert r["niter"] == it and r["fin_res"] == res
                assert np.array_equal(r["x"], x)
        res_info = p.resident()
        assert res_info["held"] >= 1 and res_info["reused"] >= 2 * len(rhs) - 2
        assert res_info["held_bytes"] <= 1 << 30
    finally:
        p.close()


def test_pool_releases_held_structures_for_new_requests(gpu_ctx):
    """Held registrations give way (least recently used first) when a new
    request needs the budget."""
    sysl = [systems.small_hex(16 + k, seed=k, kind="pressure") for k in range(4)]
    refs = [_reference(gpu_ctx, s) for s in sysl]
    # room for about two of these systems at a time
    probe = pool.Pool(workers=1, mem_budget=1 << 30)
    try:
        probe.wait(probe.submit(sysl[-1]))
        one = probe.stats()["peak_bytes"]
    finally:
        probe.close()
    budget = int(2.5 * one)
    p = pool.Pool(workers=1, mem_budget=budget)
    try:
        for rounds in range(2):
            for s, (x, it, res) in zip(sysl, refs):
                r = p.wait(p.submit(s))
                assert r["niter"] == it and np.array_equal(r["x"], x)
        info = p.resident()
        assert info["held_bytes"] <= budget and info["held"] <= 2
        assert p.stats()["peak_bytes"] <= budget
    finally:
        p.close()


def test_pool_cancel_queued_request(gpu_ctx):
    """A request still in the queue is dropped (TF_ERR_CANCELLED, x left as
    given); one that ran keeps its result; the pool keeps serving."""
    big = systems.small_hex(48, seed=6, kind="pressure", ratio=1.02)
    small = systems.small_hex(10, seed=7, kind="pressure")
    want = _reference(gpu_ctx, small)
    p = pool.Pool(workers=1, mem_budget=1 << 30)
    try:
        first = [p.submit(big) for _ in range(3)]     # one worker: these run in turn
        last = p.submit(small)
        assert p.cancel(last) == 0                     # still queued behind them
        with pytest.raises(native.TFError) as e:
            p.wait(last)
        assert e.value.status == 8                     # TF_ERR_CANCELLED
        for rid in first:
            p.wait(rid)
        assert p.cancel(first[0]) == 3                 # collected: unknown id
        again = p.submit(small)
        r = p.wait(again)
        assert p.cancel(again) == 3
        assert r["niter"] == want[1] and np.array_equal(r["x"], want[0])
    finally:
        p.close()
