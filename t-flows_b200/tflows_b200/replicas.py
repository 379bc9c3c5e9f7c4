"""Replica plumbing for runs on several GPUs of one node.

T-Flows runs one system per MPI sub-domain and, inside Cg/Bicg, sums the
scalars over processors (Process/Cpu/Native_Mod/Cg.f90:156,197) and
exchanges the buffer cells of p before each SpMV (Cg.f90:176).  The path
built here solves one whole system per GPU, so a multi-GPU run is N
independent replicas, one process per GPU: collectives only bracket the
timed region (a barrier) and reduce the per-rank timings and counts (max
of times, sum of work).  Nothing crosses between ranks inside a solve.

The same class runs over NCCL with CUDA tensors (one rank per GPU) and
over gloo with CPU tensors (the host-side tests, world size 2).
"""
import datetime
import os


def dist_env():
    """(rank, world size, local rank) from the torch.distributed launcher."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """Barrier and reductions across replica ranks.  With a world size of 1
    nothing is initialised and every reduction returns its argument."""

    def __init__(self, backend="nccl", timeout_s=180.0):
        self.rank, self.world, self.local = dist_env()
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _device(self):
        return f"cuda:{self.local}" if self.backend == "nccl" else "cpu"

    def _sync(self):
        if self.backend == "nccl":
            import torch
            torch.cuda.synchronize()

    def barrier(self):
        """All ranks reach this point with their device work finished."""
        self._sync()
        if self.dist:
            self.dist.barrier()
        self._sync()

    def _reduce(self, v, op):
        if not self.dist:
            return float(v)
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, v):
        """Max over ranks (times: the job ends when its slowest rank does)."""
        return self._reduce(v, self.dist.ReduceOp.MAX if self.dist else None)

    def sum(self, v):
        """Sum over ranks (work units processed by the whole job)."""
        return self._reduce(v, self.dist.ReduceOp.SUM if self.dist else None)

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None


def job_throughput(rep, units, seconds):
    """Whole-job throughput: the units every rank processed over the slowest
    rank's time.  Every rank calls it (two collectives, same order)."""
    t = rep.max(seconds)
    u = rep.sum(units)
    return u / t if t > 0 else 0.0, u, t
