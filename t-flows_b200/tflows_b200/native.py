"""ctypes binding of libtfkrylov.so (the C ABI declared in include/tf_krylov.h).

This is the Python counterpart of the Fortran ``bind(C)`` shim: it exposes
the same entry points with the same argument meaning as
``Native_Type % Solve_Native`` (Sources/Process/Cpu/Native_Mod/Solve_Native.f90).
There is no fallback: if the shared library or a CUDA device is missing, every
call raises.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "lib", "libtfkrylov.so")

TF_OK = 0
STATUS = {
    0: "TF_OK", 1: "TF_ERR_CUDA", 2: "TF_ERR_OOM", 3: "TF_ERR_ARG",
    4: "TF_ERR_TIMEOUT", 5: "TF_ERR_LAYOUT", 6: "TF_ERR_NO_DEVICE",
    7: "TF_ERR_BUSY", 8: "TF_ERR_CANCELLED", 9: "TF_ERR_HOST", 64: "TF_ERR_UNKNOWN_SOLVER",
    72: "TF_ERR_UNKNOWN_PREC",
}
SOLVERS = {"cg": 0, "bicg": 1}
PRECS = {"none": 0, "jacobi": 1, "diagonal": 1, "icc": 2, "incomplete_cholesky": 2}

# Every symbol include/tf_krylov.h declares; tests check the library exports them.
EXPORTS = [
    "tf_status_string", "tf_version", "tf_ctx_create", "tf_ctx_destroy",
    "tf_matrix_register", "tf_matrix_release", "tf_matrix_info", "tf_solve",
    "tf_solve_native", "tf_solve_device", "tf_ctx_set_history", "tf_last_history",
    "tf_ctx_set_wait_limit",
    "tf_host_pin", "tf_host_unpin", "tf_spmv", "tf_residual", "tf_nrms",
    "tf_ctx_sync", "tf_ctx_stream", "tf_last_error_message", "tf_matrix_tile_config",
    "tf_matrix_row_patterns", "tf_matrix_renumbered", "tf_matrix_tuning",
    "tf_tuning_cache_clear", "tf_pool_cancel", "tf_server_cancel", "tf_matrix_icc_levels",
    "tf_vec_axpby", "tf_vec_gather", "tf_vec_scatter", "tf_vec_recip", "tf_vec_dot",
    "tf_vec_nrms_sum", "tf_vec_jacobi", "tf_vec_minmax",
    "tf_faces_register", "tf_assemble_pressure", "tf_assemble_momentum",
    "tf_solve_multi", "tf_solve_multi_device", "tf_batch_add_many",
]


class TFError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        msg = f"{where}: {STATUS.get(status, status)}"
        try:
            detail = _lib.tf_last_error_message().decode()
            if detail and status in (1, 2):
                msg += f" ({detail})"
        except Exception:
            pass
        super().__init__(msg)


_lib = None

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


def load(path=LIB_PATH):
    """Load libtfkrylov.so (once).  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} not built; run `python t-flows_b200/build.py --lib`")
    L = ctypes.CDLL(path)
    L.tf_status_string.restype = ctypes.c_char_p
    L.tf_status_string.argtypes = [ctypes.c_int]
    L.tf_version.restype = ctypes.c_char_p
    L.tf_last_error_message.restype = ctypes.c_char_p
    L.tf_ctx_create.argtypes = [ctypes.c_int, ctypes.POINTER(_vp)]
    L.tf_ctx_destroy.argtypes = [_vp]
    L.tf_ctx_sync.argtypes = [_vp]
    L.tf_ctx_stream.argtypes = [_vp]
    L.tf_ctx_stream.restype = _vp
    L.tf_ctx_set_history.argtypes = [_vp, ctypes.c_int]
    L.tf_ctx_set_wait_limit.argtypes = [_vp, ctypes.c_double]
    L.tf_last_history.argtypes = [_vp, _c_dbl_p, ctypes.c_int, _c_int_p]
    L.tf_matrix_register.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                     _c_int_p, _c_int_p, _c_int_p, ctypes.POINTER(_vp)]
    L.tf_matrix_release.argtypes = [_vp]
    L.tf_matrix_info.argtypes = [_vp, _c_int_p, _c_int_p,
                                 ctypes.POINTER(ctypes.c_int64), _c_int_p]
    L.tf_matrix_tile_config.argtypes = [_vp]
    L.tf_matrix_tuning.argtypes = [_vp, _c_int_p, _c_dbl_p, ctypes.c_int, _c_int_p]
    L.tf_matrix_icc_levels.argtypes = [_vp, _c_int_p, _c_int_p]
    ci, cd = ctypes.c_int, ctypes.c_double
    L.tf_vec_axpby.argtypes = [_vp, ci, cd, _vp, cd, _vp, ci]
    L.tf_vec_gather.argtypes = [_vp, ci, _vp, _vp, _vp]
    L.tf_vec_scatter.argtypes = [_vp, ci, _vp, _vp, _vp]
    L.tf_vec_recip.argtypes = [_vp, ci, _vp, _vp]
    for f in (L.tf_vec_dot, L.tf_vec_nrms_sum):
        f.argtypes = [_vp, ci, _vp, _vp, _vp]
    L.tf_vec_jacobi.argtypes = [_vp, ci, _vp, _vp, _vp, _vp]
    L.tf_vec_minmax.argtypes = [_vp, ci, _vp, _vp]
    L.tf_matrix_row_patterns.argtypes = [_vp]
    L.tf_matrix_renumbered.argtypes = [_vp]
    solve_args = [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int,
                  _c_int_p, ctypes.c_double, _c_dbl_p, _c_dbl_p]
    L.tf_solve.argtypes = solve_args
    L.tf_solve_device.argtypes = solve_args
    L.tf_solve_native.argtypes = [_vp, _vp, ctypes.c_char_p, ctypes.c_char_p, _vp, _vp,
                                  _vp, ctypes.c_int, _c_int_p, ctypes.c_double,
                                  _c_dbl_p, _c_dbl_p]
    L.tf_host_pin.argtypes = [_vp, ctypes.c_size_t]
    L.tf_host_unpin.argtypes = [_vp]
    L.tf_spmv.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp]
    L.tf_faces_register.argtypes = [_vp, _vp, ctypes.c_int, _vp, _vp]
    L.tf_solve_multi.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp,
                                 _vp, ctypes.c_int, _vp, ctypes.c_double, _vp, _vp]
    L.tf_solve_multi_device.argtypes = L.tf_solve_multi.argtypes
    L.tf_assemble_pressure.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.tf_assemble_momentum.argtypes = [_vp, _vp, _vp, _vp, _vp, ctypes.c_double,
                                       ctypes.c_double, _vp, ctypes.c_double, _vp]
    L.tf_residual.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp]
    L.tf_nrms.argtypes = [_vp, _vp, _vp, _vp, _vp, _c_dbl_p, _vp]
    _lib = L
    return L


def _check(st, where):
    if st != TF_OK:
        raise TFError(st, where)


def _ptr(a):
    return a.ctypes.data_as(_vp)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Context:
    """One device + CUDA stream + Krylov workspace (tf_ctx)."""

    def __init__(self, device=-1, history=False):
        L = load()
        h = _vp()
        _check(L.tf_ctx_create(device, ctypes.byref(h)), "tf_ctx_create")
        self.h = h
        self.set_history(history)

    def set_wait_limit(self, seconds):
        """Limit of the device-side bounded waits (0: the 2 s default)."""
        _check(load().tf_ctx_set_wait_limit(self.h, float(seconds)), "tf_ctx_set_wait_limit")

    def set_history(self, on):
        _check(load().tf_ctx_set_history(self.h, 1 if on else 0), "tf_ctx_set_history")

    def history(self):
        cnt = ctypes.c_int(0)
        _check(load().tf_last_history(self.h, None, 0, ctypes.byref(cnt)), "tf_last_history")
        out = np.zeros(max(cnt.value, 1))
        _check(load().tf_last_history(self.h, out.ctypes.data_as(_c_dbl_p), cnt.value,
                                      ctypes.byref(cnt)), "tf_last_history")
        return out[:cnt.value]

    def sync(self):
        _check(load().tf_ctx_sync(self.h), "tf_ctx_sync")

    @property
    def stream(self):
        return load().tf_ctx_stream(self.h)

    def close(self):
        if getattr(self, "h", None):
            load().tf_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _dptr(t):
    """Device pointer of a torch tensor (or None / int)."""
    if t is None or isinstance(t, int):
        return t
    return t.data_ptr()


def vec_axpby(ctx, n, a, x, b, y, first=False):
    _check(load().tf_vec_axpby(ctx.h, int(n), float(a), _dptr(x), float(b), _dptr(y),
                               1 if first else 0), "tf_vec_axpby")


def vec_gather(ctx, n, src, idx, out):
    _check(load().tf_vec_gather(ctx.h, int(n), _dptr(src), _dptr(idx), _dptr(out)),
           "tf_vec_gather")


def vec_scatter(ctx, n, dst, idx, vals):
    _check(load().tf_vec_scatter(ctx.h, int(n), _dptr(dst), _dptr(idx), _dptr(vals)),
           "tf_vec_scatter")


def vec_recip(ctx, n, x, out):
    _check(load().tf_vec_recip(ctx.h, int(n), _dptr(x), _dptr(out)), "tf_vec_recip")


def vec_dot(ctx, n, a, b, out):
    _check(load().tf_vec_dot(ctx.h, int(n), _dptr(a), _dptr(b), _dptr(out)), "tf_vec_dot")


def vec_nrms_sum(ctx, n, r, diag, out):
    _check(load().tf_vec_nrms_sum(ctx.h, int(n), _dptr(r), _dptr(diag), _dptr(out)),
           "tf_vec_nrms_sum")


def vec_jacobi(ctx, n, r, dinv, z, out):
    _check(load().tf_vec_jacobi(ctx.h, int(n), _dptr(r), _dptr(dinv), _dptr(z), _dptr(out)),
           "tf_vec_jacobi")


def vec_minmax(ctx, n, x, out):
    _check(load().tf_vec_minmax(ctx.h, int(n), _dptr(x), _dptr(out)), "tf_vec_minmax")


def tuning_cache_clear():
    """tf_tuning_cache_clear: the next matrix of every class is timed again."""
    _check(load().tf_tuning_cache_clear(), "tf_tuning_cache_clear")


class Matrix:
    """Device-resident structure of one Matrix_Type (tf_matrix)."""

    def __init__(self, ctx, row, col, dia, n_own=None):
        L = load()
        self.row, self.col, self.dia = _i32(row), _i32(col), _i32(dia)
        self.n = len(self.row) - 1
        self.nnz = int(self.row[-1] - 1) if self.n > 0 else 0
        self.n_own = self.n if n_own is None else int(n_own)
        h = _vp()
        _check(L.tf_matrix_register(ctx.h, self.n, self.n_own, self.nnz,
                                    self.row.ctypes.data_as(_c_int_p),
                                    self.col.ctypes.data_as(_c_int_p),
                                    self.dia.ctypes.data_as(_c_int_p), ctypes.byref(h)),
               "tf_matrix_register")
        self.h = h
        self.ctx = ctx

    @property
    def tile_config(self):
        return load().tf_matrix_tile_config(self.h)

    def tuning(self):
        """[(tile configuration, median us per SpMV)] timed at registration
        (empty when the layout came from the cache, TF_TILE_CFG or the rule)."""
        L = load()
        cnt = ctypes.c_int(0)
        _check(L.tf_matrix_tuning(self.h, None, None, 0, ctypes.byref(cnt)), "tf_matrix_tuning")
        cfg = (ctypes.c_int * max(cnt.value, 1))()
        us = (ctypes.c_double * max(cnt.value, 1))()
        _check(L.tf_matrix_tuning(self.h, cfg, us, cnt.value, ctypes.byref(cnt)),
               "tf_matrix_tuning")
        return [(cfg[i], us[i]) for i in range(cnt.value)]

    def icc_levels(self):
        """(forward, backward) level counts of the incomplete-Cholesky sweeps."""
        f, b = ctypes.c_int(0), ctypes.c_int(0)
        _check(load().tf_matrix_icc_levels(self.h, ctypes.byref(f), ctypes.byref(b)),
               "tf_matrix_icc_levels")
        return f.value, b.value

    def icc_launches_per_iteration(self):
        """Kernel launches of one ICC-preconditioned Cg iteration: the three
        iteration kernels, one per sweep level, and the rho reduction."""
        f, b = self.icc_levels()
        return 3 + f + b + 1

    @property
    def renumbered(self):
        """True when Jacobi / none solves run on a renumbered copy."""
        return bool(load().tf_matrix_renumbered(self.h))

    @property
    def row_patterns(self):
        """Row patterns of the compressed column layout (0: CSR columns)."""
        return load().tf_matrix_row_patterns(self.h)

    def close(self):
        if getattr(self, "h", None):
            load().tf_matrix_release(self.h)
            self.h = None


def _norm_arg(norm):
    return None if norm is None else ctypes.byref(ctypes.c_double(norm))


def solve(ctx, mat, solver, prec, val, x, b, miter, tol, norm=None):
    """tf_solve: updates val, x, b in place like the reference; returns (niter, fin_res)."""
    for a in (val, x, b):
        assert a.dtype == np.float64 and a.flags.c_contiguous
    s = SOLVERS[solver] if isinstance(solver, str) else solver
    p = PRECS[prec] if isinstance(prec, str) else prec
    niter, res = ctypes.c_int(0), ctypes.c_double(0.0)
    _check(load().tf_solve(ctx.h, mat.h, s, p, _ptr(val), _ptr(x), _ptr(b), int(miter),
                           ctypes.byref(niter), float(tol), ctypes.byref(res),
                           _norm_arg(norm)), "tf_solve")
    return niter.value, res.value


def solve_native(ctx, mat, solver, prec, val, x, b, miter, tol, norm=None):
    """tf_solve_native: solver/prec by name, as Solve_Native dispatches them."""
    niter, res = ctypes.c_int(0), ctypes.c_double(0.0)
    st = load().tf_solve_native(ctx.h, mat.h, solver.encode(), prec.encode(), _ptr(val),
                                _ptr(x), _ptr(b), int(miter), ctypes.byref(niter),
                                float(tol), ctypes.byref(res), _norm_arg(norm))
    _check(st, "tf_solve_native")
    return niter.value, res.value


def solve_device(ctx, mat, solver, prec, d_val, d_x, d_b, miter, tol, norm=None):
    """tf_solve_device with raw device pointers (ints)."""
    s = SOLVERS[solver] if isinstance(solver, str) else solver
    p = PRECS[prec] if isinstance(prec, str) else prec
    niter, res = ctypes.c_int(0), ctypes.c_double(0.0)
    _check(load().tf_solve_device(ctx.h, mat.h, s, p, _vp(d_val), _vp(d_x), _vp(d_b),
                                  int(miter), ctypes.byref(niter), float(tol),
                                  ctypes.byref(res), _norm_arg(norm)), "tf_solve_device")
    return niter.value, res.value


def solve_multi(ctx, mat, solver, prec, val, X, B, miter, tol, norm=None):
    """nrhs solves with one matrix: X, B are (nrhs, n_cells) float64 arrays
    (updated in place like tf_solve's x and b); val is updated once.
    Returns (niter list, fin_res list)."""
    L = load()
    nr = X.shape[0]
    assert X.flags.c_contiguous and B.flags.c_contiguous and X.shape == B.shape
    it = np.zeros(nr, np.int32)
    res = np.zeros(nr)
    nv = None if norm is None else ctypes.byref(ctypes.c_double(norm))
    _check(L.tf_solve_multi(ctx.h, mat.h, SOLVERS[solver], PRECS[prec], nr,
                            val.ctypes.data_as(_vp), X.ctypes.data_as(_vp),
                            B.ctypes.data_as(_vp), int(miter), it.ctypes.data_as(_vp),
                            float(tol), res.ctypes.data_as(_vp), nv), "tf_solve_multi")
    return [int(v) for v in it], [float(v) for v in res]


def solve_multi_device(ctx, mat, solver, prec, nrhs, d_val, d_x, d_b, miter, tol, norm=None):
    """solve_multi on device pointers (d_x, d_b: nrhs * n_cells doubles)."""
    L = load()
    it = np.zeros(nrhs, np.int32)
    res = np.zeros(nrhs)
    nv = None if norm is None else ctypes.byref(ctypes.c_double(norm))
    _check(L.tf_solve_multi_device(ctx.h, mat.h, SOLVERS[solver], PRECS[prec], nrhs, d_val,
                                   d_x, d_b, int(miter), it.ctypes.data_as(_vp), float(tol),
                                   res.ctypes.data_as(_vp), nv), "tf_solve_multi_device")
    return [int(v) for v in it], [float(v) for v in res]


def faces_register(ctx, mat, faces_c, pos):
    """Face topology for device-side assembly: faces_c and pos are
    (n_faces, 2) 1-based arrays as Grid % faces_c and Matrix_Type % pos."""
    fcs = np.ascontiguousarray(faces_c, dtype=np.int32)
    ps = np.ascontiguousarray(pos, dtype=np.int32)
    _check(load().tf_faces_register(ctx.h, mat.h, len(fcs), fcs.ctypes.data_as(_vp),
                                    ps.ctypes.data_as(_vp)), "tf_faces_register")


def assemble_pressure(ctx, mat, d_fc, d_fw, d_vm, d_bnd_open, d_val):
    """Device pointers (ints); d_vm / d_bnd_open may be 0 (all ones / none)."""
    _check(load().tf_assemble_pressure(ctx.h, mat.h, d_fc, d_fw, d_vm or None,
                                       d_bnd_open or None, d_val), "tf_assemble_pressure")


def assemble_momentum(ctx, mat, d_fc, d_flux, d_bnd_wall, vis, rho, d_vol, dt, d_val):
    _check(load().tf_assemble_momentum(ctx.h, mat.h, d_fc, d_flux, d_bnd_wall or None,
                                       float(vis), float(rho), d_vol, float(dt), d_val),
           "tf_assemble_momentum")


def spmv(ctx, mat, d_val, d_p, d_q, d_pq=None):
    _check(load().tf_spmv(ctx.h, mat.h, _vp(d_val), _vp(d_p), _vp(d_q),
                          _vp(d_pq) if d_pq else None), "tf_spmv")


def residual(ctx, mat, d_val, d_b, d_x, d_r):
    _check(load().tf_residual(ctx.h, mat.h, _vp(d_val), _vp(d_b), _vp(d_x), _vp(d_r)),
           "tf_residual")


def nrms(ctx, mat, d_val, d_r, d_x, d_out, norm=None):
    _check(load().tf_nrms(ctx.h, mat.h, _vp(d_val), _vp(d_r), _vp(d_x), _norm_arg(norm),
                          _vp(d_out)), "tf_nrms")


def pin(arr):
    _check(load().tf_host_pin(_ptr(arr), arr.nbytes), "tf_host_pin")


def unpin(arr):
    _check(load().tf_host_unpin(_ptr(arr)), "tf_host_unpin")
