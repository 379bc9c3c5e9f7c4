"""GPU tests of the batched and served mixed-precision solver.

Accuracy bar: every system reaches ||b - A x||_2 / ||b||_2 <= 1e-10 in FP64
(recomputed here with scipy), and x agrees with a direct FP64 solve to
rel-L2 1e-6 (the condition numbers here are <= ~1e4).  Determinism bar: a
system's x and iteration count are bit-identical alone and in any mix.
"""
import threading
import time

import numpy as np
import pytest
import scipy.sparse as sps
import scipy.sparse.linalg as spla

from tflows_b200 import batch, native, systems

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _A(s):
    return sps.csr_matrix((s.val, s.csr.col - 1, s.csr.row - 1), shape=(s.n, s.n))


def _true_rel(s, x):
    return np.linalg.norm(s.b - _A(s) @ x) / np.linalg.norm(s.b)


def _direct(s):
    return spla.spsolve(_A(s).tocsc(), s.b)


def lattice_poly(n, seed, kind="pressure", **kw):
    """Polyhedral system numbered by sorted cell centres (scattered gathers:
    the engine renumbers it)."""
    from tflows_b200.grids import poly_lattice_grid
    g = poly_lattice_grid(n, seed)
    if kind == "pressure":
        return systems.pressure_system(g, seed, tol=TOL, miter=20000, singular="pin", norm=1.0)
    return systems.momentum_system(g, seed, tol=TOL, miter=20000, cfl=0.1, **kw)


def mixed_systems():
    return [
        systems.small_hex(12, seed=1, kind="pressure", ratio=1.02),
        systems.small_hex(20, seed=2, kind="pressure", ratio=1.02),
        systems.small_hex(10, seed=3, kind="momentum", peclet=1.0),
        systems.poly_system(3000, seed=4, kind="pressure"),
        systems.poly_system(2500, seed=5, kind="momentum", peclet=10.0),
        systems.small_hex(3, seed=6, kind="pressure"),
        lattice_poly(20000, 7),
        lattice_poly(15000, 8, kind="momentum", peclet=5.0),
    ]


@pytest.mark.parametrize("mode", [dict(vec_fp32=True), dict(vec_fp32=False),
                                  dict(vec_fp32=True, val_fp32=True)],
                         ids=["fp32vec", "fp64vec", "fp32vec_fp32val"])
def test_batch_converges_to_true_tolerance(gpu_ctx, mode):
    sysl = mixed_systems()
    b = batch.Batch(gpu_ctx, mem_budget=1 << 30, **mode)
    try:
        ids = [b.add(s, tol=TOL, maxit=20000) for s in sysl]
        b.run()
        for s, i in zip(sysl, ids):
            r = b.result(i)
            assert r["status"] == "converged", (s.name, r["status"], r["res"])
            assert r["res"] <= TOL
            assert _true_rel(s, r["x"]) <= 1.01 * TOL
            xd = _direct(s)
            assert np.linalg.norm(r["x"] - xd) / np.linalg.norm(xd) < 1e-6
    finally:
        b.close()


def test_batch_alone_equals_in_mix(gpu_ctx):
    sysl = mixed_systems()
    alone = []
    for s in sysl[:3]:
        b = batch.Batch(gpu_ctx, mem_budget=1 << 28)
        try:
            i = b.add(s)
            b.run()
            alone.append(b.result(i))
        finally:
            b.close()
    b = batch.Batch(gpu_ctx, mem_budget=1 << 30, sweep_iters=5)
    try:
        ids = [b.add(s) for s in reversed(sysl)]
        b.run()
        mix = {len(sysl) - 1 - k: b.result(i) for k, i in enumerate(ids)}
    finally:
        b.close()
    for k in range(3):
        assert mix[k]["iters"] == alone[k]["iters"]
        assert np.array_equal(mix[k]["x"], alone[k]["x"])


@pytest.mark.parametrize("threads", [1, 3, 0])
def test_batch_add_many_equals_adds(gpu_ctx, threads):
    """tf_batch_add_many prepares on worker threads and admits in order:
    the same ids, iterations and bits as one tf_batch_add per system."""
    sysl = mixed_systems()
    out = []
    for many in (False, True):
        b = batch.Batch(gpu_ctx, mem_budget=1 << 30)
        try:
            ids = b.add_many(sysl, threads=threads) if many else [b.add(s) for s in sysl]
            up = b.upload_ms()
            assert set(up) == {"prep", "wait", "admit"}
            assert up["prep"] > 0.0 and up["admit"] > 0.0 and up["wait"] >= 0.0
            b.run()
            out.append((ids, [b.result(i) for i in ids]))
        finally:
            b.close()
    (ids0, r0), (ids1, r1) = out
    assert ids0 == ids1
    for a, c in zip(r0, r1):
        assert a["iters"] == c["iters"] and a["status"] == c["status"] == "converged"
        assert np.array_equal(a["x"], c["x"])


def test_batch_add_many_stops_at_the_budget(gpu_ctx):
    """Systems before the first that does not fit stay added; the rest get -1."""
    from tflows_b200 import native
    small = [systems.small_hex(4, seed=k, kind="pressure") for k in (1, 2)]
    big = systems.small_hex(40, seed=3, kind="pressure")
    b = batch.Batch(gpu_ctx, mem_budget=1 << 20)
    try:
        with pytest.raises(native.TFError) as e:
            b.add_many(small + [big] + small, threads=2)
        assert e.value.status == 7     # TF_ERR_BUSY
        b.run()
        assert len(b.n) == 2
        for i in b.n:
            assert b.result(i)["status"] == "converged"
    finally:
        b.close()


def test_batch_memory_budget(gpu_ctx):
    big = systems.small_hex(40, seed=1, kind="pressure")
    b = batch.Batch(gpu_ctx, mem_budget=1 << 20)
    try:
        from tflows_b200 import native
        with pytest.raises(native.TFError) as e:
            b.add(big)
        assert e.value.status == 7     # TF_ERR_BUSY
        small = systems.small_hex(4, seed=1, kind="pressure")
        i = b.add(small)
        b.run()
        assert b.result(i)["status"] == "converged"
    finally:
        b.close()


def test_batch_maxiter_reported(gpu_ctx):
    s = systems.small_hex(16, seed=1, kind="pressure", ratio=1.02)
    b = batch.Batch(gpu_ctx, mem_budget=1 << 28)
    try:
        i = b.add(s, tol=TOL, maxit=5)
        b.run()
        r = b.result(i)
        assert r["status"] == "maxiter" and r["iters"] == 5 and r["res"] > TOL
    finally:
        b.close()


@pytest.mark.parametrize("profiled", [False, True], ids=["graph", "profiled"])
def test_batch_trace_records(gpu_ctx, profiled, monkeypatch):
    """One record per sweep: the first lists every system with its rows and
    entries; running systems never grow; profiled sweeps (direct launches
    with events) carry the per-kernel times and the same results."""
    if profiled:
        monkeypatch.setenv("TF_BATCH_PROFILE", "1")
    sysl = mixed_systems()[:5]
    b = batch.Batch(gpu_ctx, mem_budget=1 << 30)
    try:
        ids = [b.add(s, tol=TOL, maxit=20000) for s in sysl]
        b.run()
        tr = b.trace()
        assert len(tr) == b.info()["sweeps"]
        assert tr[0]["active"] == len(sysl)
        assert tr[0]["rows"] == sum(s.n for s in sysl)
        assert tr[0]["nnz"] == sum(s.nnz for s in sysl)
        nnz, rows = tr[0]["nnz"], tr[0]["rows"]
        assert 8 * nnz + 56 * rows <= tr[0]["iter_bytes"] <= 12 * nnz + 57 * rows
        assert all(t["ms"] > 0 and t["items"] > 0 for t in tr)
        assert all(a["active"] >= c["active"] and a["rows"] >= c["rows"]
                   for a, c in zip(tr, tr[1:]))
        total = {k: sum(t["kernel_ms"][k] for t in tr) for k in batch.KERNELS}
        if profiled:
            km = b.kernel_ms()
            assert set(km) == set(batch.KERNELS)
            assert km["spmv"] > 0 and km["update"] > 0 and km["alpha"] > 0
            for k in batch.KERNELS:
                assert total[k] == pytest.approx(km[k], rel=1e-9, abs=1e-9)
            assert sum(km.values()) <= 1.05 * sum(t["ms"] for t in tr)
        else:
            assert all(v == 0.0 for v in total.values())
            with pytest.raises(native.TFError):
                b.kernel_ms()
        for s, i in zip(sysl, ids):
            r = b.result(i)
            assert r["status"] == "converged" and _true_rel(s, r["x"]) <= 1.01 * TOL
    finally:
        b.close()


def test_server_continuous_batching(gpu_ctx):
    """Requests arriving while others run join at the next sweep; each result
    equals the same system solved alone."""
    sysl = mixed_systems()
    ref = {}
    b = batch.Batch(gpu_ctx, mem_budget=1 << 30)
    try:
        ids = [b.add(s) for s in sysl]
        b.run()
        ref = {k: b.result(i) for k, i in enumerate(ids)}
    finally:
        b.close()
    srv = batch.Server(gpu_ctx, mem_budget=1 << 30, sweep_iters=4)
    try:
        rids = {}

        def producer():
            for k, s in enumerate(sysl * 2):
                rids[k] = srv.submit(s)
                time.sleep(0.002 * (k % 3))

        t = threading.Thread(target=producer)
        t.start()
        t.join()
        for k in range(len(sysl) * 2):
            r = srv.wait(rids[k])
            want = ref[k % len(sysl)]
            assert r["status"] == "converged"
            assert r["iters"] == want["iters"]
            assert np.array_equal(r["x"], want["x"])
            assert r["latency_ms"] >= r["queue_ms"] >= 0.0
        st = srv.stats()
        assert st["completed"] == len(sysl) * 2 and st["error"] == 0
    finally:
        srv.close()


def test_batch_row_patterns_equal_csr_columns(gpu_ctx, monkeypatch):
    """Structured systems stream row patterns (one byte per row) instead of
    their columns; every row sum, and so every iterate, is the same bit for
    bit (TF_NO_ROW_PATTERNS keeps the columns)."""
    sysl = mixed_systems()
    out = []
    for no_pat in (False, True):
        if no_pat:
            monkeypatch.setenv("TF_NO_ROW_PATTERNS", "1")
        b = batch.Batch(gpu_ctx, mem_budget=1 << 30)
        try:
            free0 = b.info()["free_bytes"]
            ids = [b.add(s) for s in sysl]
            used = free0 - b.info()["free_bytes"]
            b.run()
            out.append((used, [b.result(i) for i in ids]))
        finally:
            b.close()
    (used_pat, r_pat), (used_csr, r_csr) = out
    for a, c in zip(r_pat, r_csr):
        assert a["status"] == c["status"] == "converged"
        assert a["iters"] == c["iters"] and np.array_equal(a["x"], c["x"])
    hex_nnz = sum(s.nnz for s in sysl if "-hex-" in s.name)
    assert used_csr - used_pat >= 3 * hex_nnz   # the hex systems' columns stay home


def _with_values(s, seed):
    """s with the same structure arrays (the same memory) and new values and
    right-hand side: every off-diagonal a_ij scaled by f_i f_j (seeded; a
    symmetric matrix stays symmetric), the diagonal kept dominant."""
    import copy
    rng = np.random.default_rng(seed)
    t = copy.copy(s)
    val = s.val.copy()
    row0 = s.csr.row - 1
    col0 = s.csr.col - 1
    f = rng.uniform(0.7, 1.3, s.n)
    for i in range(s.n):
        js, je = row0[i], row0[i + 1]
        d = s.csr.dia[i] - 1
        off = np.array([j for j in range(js, je) if j != d], dtype=np.int64)
        if off.size:
            val[off] *= f[i] * f[col0[off]]
            val[d] = max(val[d], 1.05 * np.abs(val[off]).sum())
    t.val = val
    t.b = rng.uniform(-1.0, 1.0, s.n)
    return t


def test_shared_structure_equals_separate_structures(gpu_ctx):
    """Systems that share one structure (the same caller arrays) use one
    device copy of it; each result equals the same system in a batch of
    its own, where its structure is uploaded anew."""
    base = [systems.small_hex(14, seed=31, kind="pressure", ratio=1.02),
            lattice_poly(12000, 32)]
    variants = [_with_values(s, 100 + k) for s in base for k in range(3)]
    alone = []
    for v in variants:
        b = batch.Batch(gpu_ctx, mem_budget=1 << 28)
        try:
            i = b.add(v)
            b.run()
            alone.append(b.result(i))
        finally:
            b.close()
    b = batch.Batch(gpu_ctx, mem_budget=1 << 29)
    try:
        free0 = b.info()["free_bytes"]
        ids = [b.add(v) for v in variants]
        used_shared = free0 - b.info()["free_bytes"]
        b.run()
        for v, i, a in zip(variants, ids, alone):
            r = b.result(i)
            assert r["status"] == "converged" and _true_rel(v, r["x"]) <= 1.01 * TOL
            assert r["iters"] == a["iters"] and np.array_equal(r["x"], a["x"])
    finally:
        b.close()
    # One structure copy (4 B per entry and ~8 per row) per base system, not
    # one per variant; each variant adds its values, vectors and tile sums.
    own = sum(8 * v.nnz + 40 * v.n + (8 << 10) for v in variants)
    shared = sum(4 * s.nnz + 12 * s.n + (8 << 10) for s in base)
    assert sum(8 * v.nnz for v in variants) < used_shared <= own + shared


def test_resident_structures_are_evicted_when_space_is_needed(gpu_ctx):
    """A retired system's structure stays on the device for later systems
    with the same structure, and gives its space up when a new structure
    needs it."""
    a = systems.small_hex(30, seed=41, kind="pressure")
    c = systems.small_hex(30, seed=42, kind="pressure", ratio=1.03)
    # Room for one structure (4 B per entry, ~8 per row) and one system's own
    # arrays (8 per entry, ~36 per row), not for a second structure.
    b = batch.Batch(gpu_ctx, mem_budget=12 * a.nnz + 44 * a.n + (64 << 10))
    try:
        i = b.add(a)
        b.run()
        ra = b.result(i)
        b.remove(i)
        i = b.add(_with_values(a, 7))      # same structure: reuses the resident copy
        b.run()
        assert b.result(i)["status"] == "converged"
        b.remove(i)
        i = b.add(c)                       # new structure: evicts the old one
        b.run()
        rc = b.result(i)
        assert rc["status"] == "converged" and _true_rel(c, rc["x"]) <= 1.01 * TOL
        b.remove(i)
        i = b.add(a)                       # the first again, uploaded anew
        b.run()
        r = b.result(i)
        assert r["iters"] == ra["iters"] and np.array_equal(r["x"], ra["x"])
    finally:
        b.close()


def test_server_shared_structures(gpu_ctx):
    """Requests that share a structure but not values (a CFD time loop)
    each equal the same system solved alone."""
    base = systems.small_hex(16, seed=51, kind="pressure", ratio=1.02)
    variants = [_with_values(base, 200 + k) for k in range(6)]
    ref = []
    for v in variants:
        b = batch.Batch(gpu_ctx, mem_budget=1 << 28)
        try:
            i = b.add(v)
            b.run()
            ref.append(b.result(i))
        finally:
            b.close()
    srv = batch.Server(gpu_ctx, mem_budget=1 << 28, sweep_iters=4)
    try:
        rids = [srv.submit(v) for v in variants * 2]
        for k, rid in enumerate(rids):
            r = srv.wait(rid)
            want = ref[k % len(variants)]
            assert r["status"] == "converged"
            assert r["iters"] == want["iters"] and np.array_equal(r["x"], want["x"])
        t = srv.timing()
        assert set(t) == {"prepare", "admit", "rebuild", "sweeps", "retire"}
        assert t["sweeps"] > 0
    finally:
        srv.close()


def test_server_cancel_running_and_queued(gpu_ctx):
    """A running request is retired at the end of its sweep and its slot
    reused; a queued one is dropped; a finished one keeps its result."""
    slow = systems.small_hex(40, seed=21, kind="pressure", ratio=1.05)
    quick = systems.small_hex(8, seed=22, kind="pressure")
    srv = batch.Server(gpu_ctx, mem_budget=1 << 30, sweep_iters=4, max_systems=1)
    try:
        # tol 0: the slow request can only stop at its iteration limit
        running = srv.submit(slow, tol=0.0, maxit=10 ** 7)
        queued = srv.submit(quick)          # one slot: waits behind the slow one
        t0 = time.perf_counter()
        while srv.stats()["admitted"] < 1 and time.perf_counter() - t0 < 5.0:
            time.sleep(0.001)
        assert srv.stats()["admitted"] == 1  # the slow one holds the only slot
        assert srv.cancel(queued) == 0
        assert srv.cancel(running) == 0
        for rid in (queued, running):
            with pytest.raises(native.TFError) as e:
                srv.wait(rid)
            assert e.value.status == 8      # TF_ERR_CANCELLED
        done = srv.submit(quick)
        r = srv.wait(done)
        assert r["status"] == "converged"
        assert srv.cancel(done) == 3        # collected: unknown id
    finally:
        srv.close()
