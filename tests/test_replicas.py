"""Host-side tests of the multi-GPU replica path on CPU: two gloo ranks
(world size 2), and a two-rank torchrun launch of the benchmark's
reference arm.  No GPU needed."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    sys.path.insert(0, os.path.join(ROOT, "t-flows_b200"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from tflows_b200 import replicas
    rep = replicas.Replicas("gloo", timeout_s=60)
    try:
        rep.barrier()
        # rank r "processed" 1000*(r+1) cell-iterations in (r+1)*0.5 s
        thr, units, t = replicas.job_throughput(rep, 1000.0 * (rank + 1), 0.5 * (rank + 1))
        q.put((rank, rep.world, thr, units, t, rep.max(-rank), rep.sum(1)))
    finally:
        rep.close()


def test_replicas_gloo_world2():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, world, thr, units, t, mx, sm in got:
        assert world == 2
        assert units == 3000.0 and t == 1.0 and thr == 3000.0   # sum of work / max time
        assert mx == 0.0 and sm == 2.0


def test_replicas_single_rank_is_identity(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, os.path.join(ROOT, "t-flows_b200"))
    from tflows_b200 import replicas
    rep = replicas.Replicas("gloo")
    assert rep.dist is None and rep.world == 1
    assert replicas.job_throughput(rep, 50.0, 2.0) == (25.0, 50.0, 2.0)
    rep.close()


@pytest.mark.timeout(300)
def test_bench_reference_arm_two_ranks():
    """`bench.py --impl reference` under torchrun with 2 ranks: rank 0 alone
    runs the oracle and prints one JSON line; rank 1 exits 0 without work."""
    port = _free_port()
    env = dict(os.environ, TF_REF_ITERS="3", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--size", "12", "--steps", "2", "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=280)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["steps"] == 2
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port"
