"""ctypes binding of the batched / served solver API (tf_batch_*, tf_server_*)."""
import ctypes

import numpy as np

from . import native

_vp = ctypes.c_void_p
STATUS = {0: "free", 1: "init", 2: "active", 3: "converged", 4: "maxiter", 5: "breakdown"}


class BatchOpts(ctypes.Structure):
    _fields_ = [("vec_fp32", ctypes.c_int), ("val_fp32", ctypes.c_int),
                ("sweep_iters", ctypes.c_int), ("max_systems", ctypes.c_int),
                ("ru_delta", ctypes.c_double), ("mem_budget", ctypes.c_size_t),
                ("two_phase_rows", ctypes.c_int)]


class SweepRec(ctypes.Structure):
    """tf_batch_sweep: one sweep of a tf_batch_run."""
    _fields_ = [("active", ctypes.c_int), ("items", ctypes.c_int),
                ("rows", ctypes.c_int64), ("nnz", ctypes.c_int64),
                ("iter_bytes", ctypes.c_double), ("ms", ctypes.c_double),
                ("kernel_ms", ctypes.c_double * 8)]


KERNELS = ("pupdate", "spmv", "alpha", "update", "beta", "ru_fold", "ru_res", "ru_finish")


def _lib():
    L = native.load()
    if getattr(L, "_tf_batch_bound", False):
        return L
    ip, dp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    L.tf_batch_create.argtypes = [_vp, ctypes.POINTER(BatchOpts), ctypes.POINTER(_vp)]
    L.tf_batch_destroy.argtypes = [_vp]
    L.tf_batch_add.argtypes = [_vp, ctypes.c_int, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp,
                               _vp, ctypes.c_double, ctypes.c_int, ip]
    L.tf_batch_add_many.argtypes = [_vp, ctypes.c_int, ip, ctypes.POINTER(ctypes.c_int64),
                                    _vp, _vp, _vp, _vp, _vp, _vp, dp, ip, ctypes.c_int, ip]
    L.tf_batch_run.argtypes = [_vp]
    L.tf_batch_result.argtypes = [_vp, ctypes.c_int, _vp, ip, dp, ip, ip, dp]
    L.tf_batch_remove.argtypes = [_vp, ctypes.c_int]
    L.tf_batch_trace.argtypes = [_vp, ctypes.POINTER(SweepRec), ctypes.c_int, ip]
    L.tf_batch_kernel_ms.argtypes = [_vp, dp]
    L.tf_batch_info.argtypes = [_vp, ip, ip, ctypes.POINTER(ctypes.c_size_t)]
    L.tf_batch_upload_ms.argtypes = [_vp, dp, dp, dp]
    L.tf_server_create.argtypes = [_vp, ctypes.POINTER(BatchOpts), ctypes.POINTER(_vp)]
    L.tf_server_submit.argtypes = [_vp, ctypes.c_int, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp,
                                   _vp, ctypes.c_double, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_int64)]
    L.tf_server_wait.argtypes = [_vp, ctypes.c_int64, _vp, ip, dp, ip, dp, dp]
    L.tf_server_stats.argtypes = [_vp, ctypes.POINTER(ctypes.c_longlong),
                                  ctypes.POINTER(ctypes.c_longlong), ip, ip]
    L.tf_server_destroy.argtypes = [_vp]
    L.tf_server_cancel.argtypes = [_vp, ctypes.c_int64]
    L.tf_server_timing.argtypes = [_vp, dp]
    L._tf_batch_bound = True
    return L


def _opts(vec_fp32=True, val_fp32=False, sweep_iters=8, max_systems=1024, ru_delta=0.1,
          mem_budget=4 << 30, two_phase_rows=0):
    return BatchOpts(int(vec_fp32), int(val_fp32), int(sweep_iters), int(max_systems),
                     float(ru_delta), int(mem_budget), int(two_phase_rows))


def _sys_args(s):
    row = np.ascontiguousarray(s.csr.row, np.int32)
    col = np.ascontiguousarray(s.csr.col, np.int32)
    dia = np.ascontiguousarray(s.csr.dia, np.int32)
    val = np.ascontiguousarray(s.val, np.float64)
    b = np.ascontiguousarray(s.b, np.float64)
    x0 = np.ascontiguousarray(s.x0, np.float64)
    keep = (row, col, dia, val, b, x0)
    p = lambda a: a.ctypes.data_as(_vp)  # noqa: E731
    return keep, (s.n, s.nnz, p(row), p(col), p(dia), p(val), p(b), p(x0))


class Batch:
    def __init__(self, ctx, **opts):
        self.L = _lib()
        self.opts = _opts(**opts)
        h = _vp()
        native._check(self.L.tf_batch_create(ctx.h, ctypes.byref(self.opts), ctypes.byref(h)),
                      "tf_batch_create")
        self.h = h
        self.n = {}

    def add(self, s, tol=1e-10, maxit=20000):
        keep, args = _sys_args(s)
        sid = ctypes.c_int(-1)
        native._check(self.L.tf_batch_add(self.h, *args, float(tol), int(maxit),
                                          ctypes.byref(sid)), "tf_batch_add")
        self.n[sid.value] = s.n
        return sid.value

    def add_many(self, systems, tol=1e-10, maxit=20000, threads=0):
        """tf_batch_add_many: the host preparation of the systems runs on
        `threads` threads (0: all hardware threads); ids and results equal
        add() called for each system in order."""
        cnt = len(systems)
        if cnt == 0:
            return []
        packed = [_sys_args(s) for s in systems]
        keep = [k for k, _ in packed]
        cols = list(zip(*[a for _, a in packed]))   # n, nnz, row, col, dia, val, b, x0
        ptrs = [(_vp * cnt)(*c) for c in cols[2:]]
        n = (ctypes.c_int * cnt)(*cols[0])
        nnz = (ctypes.c_int64 * cnt)(*cols[1])
        tols = (ctypes.c_double * cnt)(*([float(tol)] * cnt))
        its = (ctypes.c_int * cnt)(*([int(maxit)] * cnt))
        sid = (ctypes.c_int * cnt)()
        st = self.L.tf_batch_add_many(self.h, cnt, n, nnz, *ptrs, tols, its, int(threads), sid)
        del keep
        for s, i in zip(systems, sid):
            if i >= 0:
                self.n[i] = s.n
        native._check(st, "tf_batch_add_many")
        return list(sid)

    def run(self):
        native._check(self.L.tf_batch_run(self.h), "tf_batch_run")

    def result(self, sid, want_x=True):
        x = np.empty(self.n[sid]) if want_x else None
        it, st, nru = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        res, dms = ctypes.c_double(), ctypes.c_double()
        native._check(self.L.tf_batch_result(self.h, sid, x.ctypes.data_as(_vp) if want_x else None,
                                             ctypes.byref(it), ctypes.byref(res),
                                             ctypes.byref(st), ctypes.byref(nru),
                                             ctypes.byref(dms)),
                      "tf_batch_result")
        return dict(x=x, iters=it.value, res=res.value, status=STATUS[st.value],
                    n_updates=nru.value, done_ms=dms.value)

    def trace(self):
        """One dict per sweep of the last run: systems running, work items,
        rows and entries of the running systems, wall ms, and (profiling
        only) the sweep's ms per kernel."""
        cnt = ctypes.c_int(0)
        native._check(self.L.tf_batch_trace(self.h, None, 0, ctypes.byref(cnt)),
                      "tf_batch_trace")
        n = cnt.value
        recs = (SweepRec * max(n, 1))()
        native._check(self.L.tf_batch_trace(self.h, recs, n, ctypes.byref(cnt)),
                      "tf_batch_trace")
        return [dict(active=r.active, items=r.items, rows=r.rows, nnz=r.nnz,
                     iter_bytes=r.iter_bytes, ms=r.ms,
                     kernel_ms=dict(zip(KERNELS, list(r.kernel_ms))))
                for r in recs[:n]]

    def kernel_ms(self):
        """{kernel: ms} over the runs so far (batch created with TF_BATCH_PROFILE)."""
        out = (ctypes.c_double * len(KERNELS))()
        native._check(self.L.tf_batch_kernel_ms(self.h, out), "tf_batch_kernel_ms")
        return dict(zip(KERNELS, list(out)))

    def remove(self, sid):
        native._check(self.L.tf_batch_remove(self.h, sid), "tf_batch_remove")
        self.n.pop(sid, None)

    def info(self):
        sw, wi = ctypes.c_int(), ctypes.c_int()
        fb = ctypes.c_size_t()
        native._check(self.L.tf_batch_info(self.h, ctypes.byref(sw), ctypes.byref(wi),
                                           ctypes.byref(fb)), "tf_batch_info")
        return dict(sweeps=sw.value, work_items=wi.value, free_bytes=fb.value)

    def upload_ms(self):
        """{prep, wait, admit}: milliseconds over all adds so far (host
        preparation summed over systems, the admitting thread's wait for it,
        admission with the copies to the device)."""
        v = [ctypes.c_double() for _ in range(3)]
        native._check(self.L.tf_batch_upload_ms(self.h, *[ctypes.byref(x) for x in v]),
                      "tf_batch_upload_ms")
        return dict(zip(("prep", "wait", "admit"), (x.value for x in v)))

    def close(self):
        if getattr(self, "h", None):
            self.L.tf_batch_destroy(self.h)
            self.h = None


class Server:
    def __init__(self, ctx, **opts):
        self.L = _lib()
        self.opts = _opts(**opts)
        h = _vp()
        native._check(self.L.tf_server_create(ctx.h, ctypes.byref(self.opts), ctypes.byref(h)),
                      "tf_server_create")
        self.h = h
        self.n = {}

    def submit(self, s, tol=1e-10, maxit=20000):
        keep, args = _sys_args(s)
        rid = ctypes.c_int64()
        native._check(self.L.tf_server_submit(self.h, *args, float(tol), int(maxit),
                                              ctypes.byref(rid)), "tf_server_submit")
        self.n[rid.value] = s.n
        return rid.value

    def wait(self, rid):
        x = np.empty(self.n.pop(rid))
        it, st = ctypes.c_int(), ctypes.c_int()
        res, lat, qms = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        rc = self.L.tf_server_wait(self.h, rid, x.ctypes.data_as(_vp), ctypes.byref(it),
                                   ctypes.byref(res), ctypes.byref(st), ctypes.byref(lat),
                                   ctypes.byref(qms))
        native._check(rc, "tf_server_wait")
        return dict(x=x, iters=it.value, res=res.value, status=STATUS.get(st.value, st.value),
                    latency_ms=lat.value, queue_ms=qms.value)

    def cancel(self, rid):
        """tf_server_cancel: 0 (will end cancelled), 7 (already finished)."""
        return self.L.tf_server_cancel(self.h, rid)

    def stats(self):
        a, c = ctypes.c_longlong(), ctypes.c_longlong()
        pk, sw = ctypes.c_int(), ctypes.c_int()
        err = self.L.tf_server_stats(self.h, ctypes.byref(a), ctypes.byref(c), ctypes.byref(pk),
                                     ctypes.byref(sw))
        return dict(admitted=a.value, completed=c.value, peak_running=pk.value,
                    sweeps=sw.value, error=err)

    def timing(self):
        """Milliseconds by activity since creation (tf_server_timing)."""
        out = (ctypes.c_double * 5)()
        native._check(self.L.tf_server_timing(self.h, out), "tf_server_timing")
        return dict(zip(("prepare", "admit", "rebuild", "sweeps", "retire"),
                        (round(v, 1) for v in out)))

    def close(self):
        if getattr(self, "h", None):
            self.L.tf_server_destroy(self.h)
            self.h = None
