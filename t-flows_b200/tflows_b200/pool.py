"""ctypes binding of the request pool (tf_pool_*): concurrent Solve_Native
calls on a pool of CUDA streams."""
import ctypes

import numpy as np

from . import native

_vp = ctypes.c_void_p


def _lib():
    L = native.load()
    if getattr(L, "_tf_pool_bound", False):
        return L
    ip, dp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    L.tf_pool_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_size_t,
                                 ctypes.POINTER(_vp)]
    L.tf_pool_submit.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                 _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_double,
                                 dp, ctypes.POINTER(ctypes.c_int64)]
    L.tf_pool_wait.argtypes = [_vp, ctypes.c_int64, ip, dp, dp, dp]
    L.tf_pool_stats.argtypes = [_vp] + [ctypes.POINTER(ctypes.c_longlong)] * 3 + [
        ctypes.POINTER(ctypes.c_size_t)]
    L.tf_pool_resident.argtypes = [_vp, ctypes.POINTER(ctypes.c_longlong),
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_size_t)]
    L.tf_pool_destroy.argtypes = [_vp]
    L.tf_pool_cancel.argtypes = [_vp, ctypes.c_int64]
    L._tf_pool_bound = True
    return L


class Pool:
    """Worker streams that run Solve_Native requests concurrently."""

    def __init__(self, workers=8, mem_budget=0, device=0):
        self.L = _lib()
        h = _vp()
        native._check(self.L.tf_pool_create(device, workers, mem_budget, ctypes.byref(h)),
                      "tf_pool_create")
        self.h = h
        self.keep = {}   # arrays the library reads/writes until wait() returns

    def submit(self, s, miter=None, tol=None, norm="system", b=None, x0=None, solver=None,
               prec=None):
        """Queue system `s` (a systems.System).  tol/miter/norm default to the
        system's own; b/x0 override its right-hand side / initial guess."""
        row = np.ascontiguousarray(s.csr.row, np.int32)
        col = np.ascontiguousarray(s.csr.col, np.int32)
        dia = np.ascontiguousarray(s.csr.dia, np.int32)
        val = np.ascontiguousarray(s.val, np.float64)
        bb = np.ascontiguousarray(s.b if b is None else b, np.float64)
        xx = np.array(s.x0 if x0 is None else x0, dtype=np.float64, copy=True)
        nv = s.norm if norm == "system" else norm
        normp = None if nv is None else ctypes.byref(ctypes.c_double(nv))
        sv = native.SOLVERS[solver or s.solver]
        pv = native.PRECS[prec or s.prec]
        p = lambda a: a.ctypes.data_as(_vp)  # noqa: E731
        rid = ctypes.c_int64()
        native._check(self.L.tf_pool_submit(self.h, sv, pv, s.n, s.nnz, p(row), p(col), p(dia),
                                            p(val), p(bb), p(xx),
                                            int(s.miter if miter is None else miter),
                                            float(s.tol if tol is None else tol), normp,
                                            ctypes.byref(rid)), "tf_pool_submit")
        self.keep[rid.value] = (row, col, dia, val, bb, xx)
        return rid.value

    def wait(self, rid):
        it = ctypes.c_int()
        res, lat, qms = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        try:
            native._check(self.L.tf_pool_wait(self.h, rid, ctypes.byref(it), ctypes.byref(res),
                                              ctypes.byref(lat), ctypes.byref(qms)),
                          "tf_pool_wait")
        finally:
            arrs = self.keep.pop(rid)
        return dict(x=arrs[5], niter=it.value, fin_res=res.value, latency_ms=lat.value,
                    queue_ms=qms.value)

    def cancel(self, rid):
        """tf_pool_cancel: 0 (dropped from the queue), 7 (running or finished)."""
        return self.L.tf_pool_cancel(self.h, rid)

    def stats(self):
        a, c, r = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        pk = ctypes.c_size_t()
        native._check(self.L.tf_pool_stats(self.h, ctypes.byref(a), ctypes.byref(c),
                                           ctypes.byref(r), ctypes.byref(pk)), "tf_pool_stats")
        return dict(submitted=a.value, completed=c.value, rejected=r.value, peak_bytes=pk.value)

    def resident(self):
        """Requests that reused a held registration, registrations held and
        their bytes."""
        r, h, b = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_size_t()
        native._check(self.L.tf_pool_resident(self.h, ctypes.byref(r), ctypes.byref(h),
                                              ctypes.byref(b)), "tf_pool_resident")
        return dict(reused=r.value, held=h.value, held_bytes=b.value)

    def close(self):
        if getattr(self, "h", None):
            self.L.tf_pool_destroy(self.h)
            self.h = None
            self.keep.clear()
