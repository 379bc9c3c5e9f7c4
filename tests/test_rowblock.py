"""One system split by rows over several ranks (tflows_b200/rowblock.py).

CPU: the partition (every row of every block sums exactly what the global
row sums once the buffer cells hold their owners' values), the solve with
all ranks in one process, and two gloo ranks in two processes running
Cg.f90's sequence of exchanges and sums -- each against the oracle's
single-process solve (iteration counts equal, x to rel-L2 1e-12: only the
association of the sums over ranks differs).
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import oracle as O
from tflows_b200 import rowblock, systems

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _oracle(s, norm):
    v, x, b = s.val.copy(), s.x0.copy(), s.b.copy()
    r = O.solve_native("cg", "jacobi", s.csr.row, s.csr.col, s.csr.dia, v, x, b, s.miter,
                       s.tol, norm=norm, threads=1)
    return x, r["niter"], r["fin_res"]


@pytest.mark.parametrize("nparts", [1, 2, 3, 5])
def test_partition_row_sums_are_global_row_sums(nparts):
    s = systems.poly_system(400, seed=3, kind="pressure")
    blocks = rowblock.partition(s.csr, s.val, nparts)
    assert sum(b.n_own for b in blocks) == s.n
    p = np.random.default_rng(1).standard_normal(s.n)
    want = O.spmv(s.csr.row, s.csr.col, s.csr.dia, s.val, p)
    for b in blocks:
        k = rowblock.HostKernels(b)
        pl = np.concatenate([p[b.start:b.stop], p[b.buf_global]])
        q = np.zeros(b.n_own + b.n_buf)
        k.spmv(b.val, pl, q, b.n_own)
        assert np.array_equal(q[:b.n_own], want[b.start:b.stop])
        # diagonal first in every local row, as Matrix_Type keeps it
        assert np.all(b.col[b.row[:-1] - 1] == np.arange(1, b.n_own + b.n_buf + 1))
        for q2, pos in b.recv.items():
            assert np.array_equal(blocks[q2].start + blocks[q2].send[b.rank], b.buf_global[pos])


@pytest.mark.parametrize("nparts", [2, 3])
@pytest.mark.parametrize("norm", [1.0, None])
def test_local_ranks_equal_single_solve(nparts, norm):
    s = systems.small_hex(7, seed=4, kind="pressure", ratio=1.05, tol=1e-10, miter=500)
    x, it, res = rowblock.solve_local(s.csr, s.val, s.b, s.x0, nparts, s.miter, s.tol, norm)
    ox, oit, ores = _oracle(s, norm)
    assert it == oit
    assert np.linalg.norm(x - ox) <= 1e-12 * np.linalg.norm(ox)
    assert res < s.tol and res == pytest.approx(ores, rel=1e-6)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "t-flows_b200"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist
    from tflows_b200 import rowblock, systems
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        s = systems.poly_system(500, seed=5, kind="pressure", tol=1e-10, miter=500, norm=1.0)
        blocks = rowblock.partition(s.csr, s.val, world)
        b = blocks[rank]
        steps = rowblock.cg_steps(b, rowblock.HostKernels(b), s.b[b.start:b.stop],
                                  s.x0[b.start:b.stop], s.miter, s.tol, 1.0)
        x, it, res = rowblock.run_torch(b, rowblock.HostKernels(b), steps, "cpu")
        q.put((rank, b.start, x.tolist(), it, res))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_single_solve():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    s = systems.poly_system(500, seed=5, kind="pressure", tol=1e-10, miter=500, norm=1.0)
    x = np.concatenate([np.array(g[2]) for g in got])
    ox, oit, ores = _oracle(s, 1.0)
    assert got[0][3] == got[1][3] == oit
    assert got[0][4] == got[1][4] < s.tol
    assert np.linalg.norm(x - ox) <= 1e-12 * np.linalg.norm(ox)
