"""One system split by rows over several ranks (one GPU each).

T-Flows runs a large case as METIS sub-domains, one MPI process each.  Every
process holds its own cells plus buffer cells -- copies of the neighbouring
sub-domains' cells its rows reach -- and Cg/Bicg exchange the buffer values
of p before every SpMV (Native_Mod/Cg.f90:176, Grid % Exchange_Cells_Real)
and of x at the end (:240), and sum every dot product and the normalisation
over processes (Global % Sum_Real / Sum_Int, Cg.f90:72-73,156,197;
Normalized_Root_Mean_Square.f90:38,53-54 with Min_Real / Max_Real).

Here the sub-domains are contiguous row blocks of the matrix as given
(`partition`), each rank's block is a Matrix_Type of n_own = its rows and
n_cells = rows + buffer cells (the layout the library's solvers already
take: rows past n_own are never iterated), and `cg_steps` runs Cg.f90's
sequence as a coroutine that yields the same exchanges and sums, driven by
`run_torch` (torch.distributed: NCCL with device tensors or gloo with host
tensors, one rank per process) or by `run_local` (all ranks in one process,
in lockstep).  The arithmetic goes through a kernel set: `DeviceKernels`, the
library's sm_100a kernels through its C ABI (SpMV over the own rows, the
vector updates, the partial sums), or `HostKernels`, numpy on the host (the
CPU tests with gloo ranks).  Two all-reduces per iteration, as the
drop-in's kernels fuse them: p.q after the SpMV, and {sum r^2/a^2, next rho}
after the update (z = r / diag is formed in the same pass); with `norm`
absent also the min and max of x.

The result equals a single-process solve to the rounding of the sums
(their association changes with the number of ranks).
"""
import numpy as np


# ---------------------------------------------------------------------------
# Partition
# ---------------------------------------------------------------------------
class Block:
    """Rank r's rows [start, stop) of the global matrix with its buffer cells.

    row/col/dia: 1-based local Matrix_Type arrays of n_cells = n_own + n_buf
    rows (buffer rows hold only their diagonal, value 1, and are never
    solved); val: the own rows' values in the global storage order;
    buf_global: global 0-based index of each buffer cell; recv[q]: buffer
    positions (0-based, from n_own) that rank q fills; send[q]: own rows
    (0-based local) whose values rank q needs, in the order q expects."""

    def __init__(self, **kw):
        self.__dict__.update(kw)


def block_starts(row, nparts):
    """Contiguous row blocks with about equal entries."""
    row0 = np.asarray(row, dtype=np.int64) - 1
    n = len(row0) - 1
    nnz = int(row0[-1])
    cuts = [0]
    for r in range(1, nparts):
        target = nnz * r // nparts
        cuts.append(int(np.searchsorted(row0, target, side="left")))
    cuts.append(n)
    return np.maximum.accumulate(np.array(cuts, dtype=np.int64))


def partition(csr, val, nparts):
    """Blocks of `csr` (systems.Csr, 1-based) for `nparts` ranks."""
    row0 = np.asarray(csr.row, dtype=np.int64) - 1
    col0 = np.asarray(csr.col, dtype=np.int64) - 1
    starts = block_starts(csr.row, nparts)
    owner_of = np.searchsorted(starts[1:], np.arange(len(row0) - 1), side="right")
    blocks = []
    for r in range(nparts):
        s, e = int(starts[r]), int(starts[r + 1])
        ni = e - s
        js, je = int(row0[s]), int(row0[e])
        cols = col0[js:je]
        outside = (cols < s) | (cols >= e)
        buf = np.unique(cols[outside])
        local = np.where(outside, ni + np.searchsorted(buf, cols), cols - s)
        nb = len(buf)
        nt = ni + nb
        lrow = np.empty(nt + 1, dtype=np.int64)
        lrow[:ni + 1] = row0[s:e + 1] - js
        lrow[ni + 1:] = lrow[ni] + np.arange(1, nb + 1)
        lcol = np.concatenate([local, ni + np.arange(nb)])
        ldia = np.empty(nt, dtype=np.int64)
        ldia[:ni] = np.asarray(csr.dia[s:e], dtype=np.int64) - 1 - js
        ldia[ni:] = lrow[ni:nt]
        lval = np.concatenate([np.asarray(val[js:je], dtype=np.float64), np.ones(nb)])
        own_buf = owner_of[buf] if nb else np.zeros(0, dtype=np.int64)
        recv = {int(q): np.nonzero(own_buf == q)[0] for q in np.unique(own_buf)}
        blocks.append(Block(rank=r, start=s, stop=e, n_own=ni, n_buf=nb,
                            row=(lrow + 1).astype(np.int32), col=(lcol + 1).astype(np.int32),
                            dia=(ldia + 1).astype(np.int32), val=lval, buf_global=buf,
                            recv=recv, send={}))
    for b in blocks:                      # send lists mirror the receivers' lists
        for q, pos in b.recv.items():
            blocks[q].send[b.rank] = (b.buf_global[pos] - blocks[q].start).astype(np.int64)
    return blocks


# ---------------------------------------------------------------------------
# Communication: the solve is a coroutine that yields its collectives
# ---------------------------------------------------------------------------
# ("sum" | "min" | "max", [floats]) -> the element-wise reduction over ranks
# ("exchange", vector)              -> None, the buffer cells filled
def run_torch(block, kern, steps, device):
    """Drive one rank's solve coroutine with torch.distributed collectives
    (NCCL with CUDA tensors, gloo with CPU tensors).  Every rank issues the
    same collectives in the same order."""
    import torch
    import torch.distributed as dist
    ops = {"sum": dist.ReduceOp.SUM, "min": dist.ReduceOp.MIN, "max": dist.ReduceOp.MAX}
    reply = None
    while True:
        try:
            req = steps.send(reply)
        except StopIteration as fin:
            return fin.value
        if req[0] == "exchange":
            vec = req[1]
            p2p, incoming = [], []
            for q in sorted(set(block.send) | set(block.recv)):
                if q in block.send:
                    p2p.append(dist.P2POp(dist.isend, kern.to_comm(kern.gather(vec, block.send[q]),
                                                                   device), q))
                if q in block.recv:
                    buf = torch.empty(len(block.recv[q]), dtype=torch.float64, device=device)
                    p2p.append(dist.P2POp(dist.irecv, buf, q))
                    incoming.append((q, buf))
            if p2p:
                for w in dist.batch_isend_irecv(p2p):
                    w.wait()
            for q, buf in incoming:
                kern.scatter(vec, block.n_own + block.recv[q], kern.from_comm(buf))
            reply = None
        else:
            t = torch.tensor(req[1], dtype=torch.float64, device=device)
            dist.all_reduce(t, op=ops[req[0]])
            reply = t.tolist()


def run_local(blocks, kerns, steps):
    """Drive every rank's coroutine in one process, in lockstep: the
    reductions combine the ranks' values (in rank order), the exchange
    copies between their vectors.  Used where fewer devices than ranks are
    at hand (the ranks then share one device, one after another)."""
    replies = [None] * len(steps)
    done = [None] * len(steps)
    while True:
        reqs = []
        for k, g in enumerate(steps):
            try:
                reqs.append(g.send(replies[k]))
            except StopIteration as fin:
                done[k] = fin.value
                reqs.append(None)
        if all(d is not None for d in done):
            return done
        kind = reqs[0][0]
        if kind == "exchange":
            vecs = [r[1] for r in reqs]
            for b, kern, vec in zip(blocks, kerns, vecs):
                for q, pos in b.recv.items():
                    vals = kerns[q].gather(vecs[q], blocks[q].send[b.rank])
                    kern.scatter(vec, b.n_own + pos, kern.from_comm(kerns[q].to_comm(vals, None)))
            replies = [None] * len(steps)
        else:
            fn = {"sum": lambda a, b: a + b, "min": min, "max": max}[kind]
            acc = list(reqs[0][1])
            for r in reqs[1:]:
                acc = [fn(u, v) for u, v in zip(acc, r[1])]
            replies = [list(acc) for _ in steps]


# ---------------------------------------------------------------------------
# Kernel sets
# ---------------------------------------------------------------------------
class HostKernels:
    """numpy on the host (the CPU tests).  Row sums in storage order."""

    def __init__(self, block):
        self.b = block
        self.row0 = block.row.astype(np.int64) - 1
        self.col0 = block.col.astype(np.int64) - 1
        self.dia0 = block.dia.astype(np.int64) - 1

    def vec(self, a):
        return np.array(a, dtype=np.float64)

    def host(self, v):
        return v.copy()

    def gather(self, v, idx):
        return v[idx].copy()

    def scatter(self, v, idx, vals):
        v[np.asarray(idx, dtype=np.int64)] = vals

    def to_comm(self, v, device):
        import torch
        t = torch.from_numpy(np.ascontiguousarray(v))
        return t if device is None else t.to(device)

    def from_comm(self, t):
        return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)

    def spmv(self, val, p, q, ni):
        """q = A p over the own rows; returns the partial p.q."""
        for i in range(ni):
            acc = 0.0
            for j in range(self.row0[i], self.row0[i + 1]):
                acc = acc + val[j] * p[self.col0[j]]
            q[i] = acc
        return float(np.dot(p[:ni], q[:ni]))

    def residual(self, val, b, x, r, ni):
        for i in range(ni):
            acc = b[i]
            for j in range(self.row0[i], self.row0[i + 1]):
                acc = acc - val[j] * x[self.col0[j]]
            r[i] = acc

    def scale(self, v, f, n):
        v[:n] *= f

    def diag(self, val, n):
        return val[self.dia0[:n]].copy()

    def diag_sum(self, val, n):
        return float(np.sum(val[self.dia0[:n]]))

    def recip(self, d, n):
        return 1.0 / d[:n]

    def nrms_sum(self, r, diag, ni):
        return float(np.sum((r[:ni] * r[:ni]) / (diag[:ni] * diag[:ni])))

    def minmax(self, x, ni):
        return float(x[:ni].min()), float(x[:ni].max())

    def precond(self, r, dinv, z, ni):
        """z = d_inv r (Jacobi); returns the partial z.r."""
        z[:ni] = r[:ni] * dinv[:ni]
        return float(np.dot(z[:ni], r[:ni]))

    def pupdate(self, z, beta, p, ni, first):
        p[:ni] = z[:ni] if first else z[:ni] + beta * p[:ni]

    def update(self, alpha, p, q, x, r, ni):
        x[:ni] += alpha * p[:ni]
        r[:ni] -= alpha * q[:ni]


class DeviceKernels:
    """The library's sm_100a kernels through its C ABI, vectors on the GPU:
    the SpMV and residual of the registered block (own rows only), and the
    vector kernels tf_vec_* (updates, Jacobi, partial sums)."""

    def __init__(self, block, ctx):
        import torch
        from . import native
        self.torch, self.native, self.ctx = torch, native, ctx
        self.b = block
        self.m = native.Matrix(ctx, block.row, block.col, block.dia, n_own=block.n_own)
        self.dia0 = torch.from_numpy(block.dia.astype(np.int64) - 1).cuda()
        self.scal = torch.zeros(4, dtype=torch.float64, device="cuda")
        self.idx = {}

    def _idx(self, idx):
        """Device copy of an index list, kept per content (the exchange
        passes the same few lists every iteration)."""
        a = np.ascontiguousarray(idx, dtype=np.int64)
        key = a.tobytes()
        t = self.idx.get(key)
        if t is None:
            t = self.torch.from_numpy(a).cuda()
            self.idx[key] = t
        return t

    def vec(self, a):
        t = self.torch.from_numpy(np.array(a, dtype=np.float64)).cuda()
        self.torch.cuda.synchronize()
        return t

    def host(self, v):
        self.ctx.sync()
        return v.cpu().numpy()

    def _scalars(self, k):
        self.ctx.sync()
        return [float(v) for v in self.scal[:k].tolist()]

    def gather(self, v, idx):
        ix = self._idx(idx)
        out = self.torch.empty(len(ix), dtype=self.torch.float64, device="cuda")
        self.native.vec_gather(self.ctx, len(ix), v, ix, out)
        return out

    def scatter(self, v, idx, vals):
        ix = self._idx(idx)
        self.native.vec_scatter(self.ctx, len(ix), v, ix, vals)

    def to_comm(self, v, device):
        self.ctx.sync()
        return v if device is None or str(device).startswith("cuda") else v.cpu()

    def from_comm(self, t):
        return t.cuda()

    def spmv(self, val, p, q, ni):
        self.native.spmv(self.ctx, self.m, val.data_ptr(), p.data_ptr(), q.data_ptr(),
                         self.scal.data_ptr())
        return self._scalars(1)[0]

    def residual(self, val, b, x, r, ni):
        self.native.residual(self.ctx, self.m, val.data_ptr(), b.data_ptr(), x.data_ptr(),
                             r.data_ptr())

    def scale(self, v, f, n):
        self.native.vec_axpby(self.ctx, n, 0.0, v, f, v)

    def diag(self, val, n):
        out = self.torch.empty(n, dtype=self.torch.float64, device="cuda")
        self.native.vec_gather(self.ctx, n, val, self.dia0[:n], out)
        return out

    def diag_sum(self, val, n):
        d = self.diag(val, n)
        self.native.vec_dot(self.ctx, n, d, None, self.scal)
        return self._scalars(1)[0]

    def recip(self, d, n):
        out = self.torch.empty(n, dtype=self.torch.float64, device="cuda")
        self.native.vec_recip(self.ctx, n, d, out)
        return out

    def nrms_sum(self, r, diag, ni):
        self.native.vec_nrms_sum(self.ctx, ni, r, diag, self.scal)
        return self._scalars(1)[0]

    def minmax(self, x, ni):
        self.native.vec_minmax(self.ctx, ni, x, self.scal)
        return tuple(self._scalars(2))

    def precond(self, r, dinv, z, ni):
        self.native.vec_jacobi(self.ctx, ni, r, dinv, z, self.scal)
        return self._scalars(1)[0]

    def pupdate(self, z, beta, p, ni, first):
        if first:
            self.native.vec_axpby(self.ctx, ni, 1.0, z, 0.0, p, first=True)
        else:
            self.native.vec_axpby(self.ctx, ni, 1.0, z, beta, p)

    def update(self, alpha, p, q, x, r, ni):
        self.native.vec_axpby(self.ctx, ni, alpha, p, 1.0, x)
        self.native.vec_axpby(self.ctx, ni, -alpha, q, 1.0, r)

    def close(self):
        self.m.close()


# ---------------------------------------------------------------------------
# The solve
# ---------------------------------------------------------------------------
TINY, HUGE = 1.0e-15, 1.0e15   # Sources/Shared/Const_Mod.f90


def cg_steps(block, kern, b, x0, miter, tol, norm=None):
    """Cg.f90 (Jacobi) on this rank's block, as a coroutine yielding its
    collectives (see run_torch / run_local).  b, x0: this rank's own
    entries.  Returns (x own, niter, fin_res); every rank ends with the same
    niter and fin_res."""
    ni, nt = block.n_own, block.n_own + block.n_buf
    val = kern.vec(block.val)
    bb = kern.vec(np.concatenate([b, np.zeros(block.n_buf)]))
    x = kern.vec(np.concatenate([x0, np.zeros(block.n_buf)]))
    r, p, q, z = (kern.vec(np.zeros(nt)) for _ in range(4))

    # Normalise the system (Cg.f90:62-84): the diagonal's mean over all ranks.
    sum_a, sum_n = yield ("sum", [kern.diag_sum(val, ni), float(ni)])
    fn = 1.0 / (sum_a / sum_n)
    kern.scale(val, fn, len(block.val))
    kern.scale(bb, fn, ni)
    diag = kern.diag(val, ni)
    dinv = kern.recip(diag, ni)

    def x_range():
        if norm is not None:
            return 0.0, norm
        lo, hi = kern.minmax(x, ni) if ni else (HUGE, -HUGE)
        lo, = yield ("min", [lo])
        hi, = yield ("max", [hi])
        return lo, hi

    def nrms_of(sumsq, lohi):
        return float(np.sqrt(sumsq)) / max(lohi[1] - lohi[0], TINY)

    res, it = 0.0, 0
    s, = yield ("sum", [kern.nrms_sum(bb, diag, ni)])
    bnrm2 = nrms_of(s, (yield from x_range()))
    if bnrm2 >= tol:
        yield ("exchange", x)
        kern.residual(val, bb, x, r, ni)
        s, = yield ("sum", [kern.nrms_sum(r, diag, ni)])
        res = nrms_of(s, (yield from x_range()))
        if res >= tol:
            rho_old = 0.0
            rho, = yield ("sum", [kern.precond(r, dinv, z, ni)])
            for it in range(1, miter + 1):
                kern.pupdate(z, rho / rho_old if it > 1 else 0.0, p, ni, it == 1)
                yield ("exchange", p)                               # Cg.f90:176
                pq, = yield ("sum", [kern.spmv(val, p, q, ni)])     # :177-197
                alpha = rho / pq
                kern.update(alpha, p, q, x, r, ni)                  # :204-209
                s, rho_next = yield ("sum", [kern.nrms_sum(r, diag, ni),
                                             kern.precond(r, dinv, z, ni)])
                res = nrms_of(s, (yield from x_range()))            # :213-222
                if res < tol:
                    break
                rho_old, rho = rho, rho_next
    yield ("exchange", x)                                           # Cg.f90:240
    return kern.host(x)[:ni], it, res


def solve_local(csr, val, b, x0, nparts, miter, tol, norm=None, make_kernels=None):
    """All nparts ranks in one process (run_local); returns the assembled x,
    niter and fin_res."""
    blocks = partition(csr, val, nparts)
    make = make_kernels or HostKernels
    kerns = [make(bl) for bl in blocks]
    steps = [cg_steps(bl, k, b[bl.start:bl.stop], x0[bl.start:bl.stop], miter, tol, norm)
             for bl, k in zip(blocks, kerns)]
    out = run_local(blocks, kerns, steps)
    for k in kerns:
        if hasattr(k, "close"):
            k.close()
    x = np.concatenate([o[0] for o in out])
    return x, out[0][1], out[0][2]
