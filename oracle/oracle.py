"""ctypes loader of the CPU oracle (oracle/libtforacle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product.  Pinned to the reference:
the reference's own Fortran source, executed by oracle/f90exec.py, produced
the golden fixtures this oracle reproduces bit for bit (see tf_oracle.cpp).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtforacle.so")

_L = None
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


def load(build=True):
    global _L
    if _L is not None:
        return _L
    if build and not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    L = ctypes.CDLL(LIB_PATH)
    L.tfo_set_threads.argtypes = [ctypes.c_int]
    L.tfo_max_threads.restype = ctypes.c_int
    L.tfo_solve_native.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   _ip, _ip, _ip, _dp, _dp, _dp, ctypes.c_int, _ip,
                                   ctypes.c_double, _dp, ctypes.c_int, ctypes.c_double, _dp]
    L.tfo_nrms.restype = ctypes.c_double
    L.tfo_nrms.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _ip, _dp, _dp, _dp,
                           ctypes.c_int, ctypes.c_double]
    L.tfo_rms.restype = ctypes.c_double
    L.tfo_rms.argtypes = [ctypes.c_int, _dp]
    L.tfo_residual_vector.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _ip, _dp, _dp,
                                      _dp, _dp]
    L.tfo_spmv.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _ip, _dp, _dp, _dp]
    L.tfo_prec_form.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _ip, _dp, _dp, _dp,
                                ctypes.c_int]
    L.tfo_prec_solve.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _ip, _dp, _dp, _dp,
                                 _dp, _dp, ctypes.c_int]
    L.tfo_set_singular.argtypes = [ctypes.c_int, _ip, _dp]
    L.tfo_create_matrix.restype = ctypes.c_long
    L.tfo_create_matrix.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _ip, ctypes.c_long,
                                    _ip, _ip]
    L.tfo_face_coef.argtypes = [ctypes.c_int] + [_dp] * 7
    L.tfo_assemble_pressure.argtypes = [ctypes.c_int, _ip, _ip, _ip, _dp, _dp, _dp, _ip, _dp]
    L.tfo_assemble_momentum.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _ip, _dp, _dp,
                                        _ip, ctypes.c_double, ctypes.c_double, _dp,
                                        ctypes.c_double, _dp]
    _L = L
    return L


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def ip(a):
    return a.ctypes.data_as(_ip)


def dp(a):
    return a.ctypes.data_as(_dp)


SOLVER = {"cg": 0, "bicg": 1}
PREC = {"none": 0, "jacobi": 1, "icc": 2}


def solve_native(solver, prec, row, col, dia, val, x, b, miter, tol, norm=None,
                 n_own=None, threads=1, history=False):
    """Run the restated Cg/Bicg.  val, x, b are modified in place (float64,
    C-contiguous).  Returns dict(niter, fin_res, hist)."""
    L = load()
    L.tfo_set_threads(threads)
    row, col, dia = _i(row), _i(col), _i(dia)
    nt = len(row) - 1
    ni = nt if n_own is None else n_own
    for a in (val, x, b):
        assert a.dtype == np.float64 and a.flags.c_contiguous
    niter = ctypes.c_int(0)
    res = ctypes.c_double(0.0)
    hist = np.full(miter + 1, np.nan) if history else None
    st = L.tfo_solve_native(SOLVER[solver], PREC[prec], nt, ni, ip(row), ip(col), ip(dia),
                            dp(val), dp(x), dp(b), int(miter), ctypes.byref(niter),
                            float(tol), ctypes.byref(res), 0 if norm is None else 1,
                            0.0 if norm is None else float(norm),
                            dp(hist) if history else None)
    if st != 0:
        raise RuntimeError(f"oracle solve_native status {st}")
    out = dict(niter=niter.value, fin_res=res.value)
    if history:
        out["hist"] = hist[: niter.value + 1]
    return out


def spmv(row, col, dia, val, p):
    L = load()
    L.tfo_set_threads(1)
    row, col, dia, val, p = _i(row), _i(col), _i(dia), _d(val), _d(p)
    nt = len(row) - 1
    q = np.zeros(nt)
    L.tfo_spmv(nt, nt, ip(row), ip(col), ip(dia), dp(val), dp(p), dp(q))
    return q


def residual(row, col, dia, val, b, x):
    L = load()
    L.tfo_set_threads(1)
    row, col, dia, val, b, x = _i(row), _i(col), _i(dia), _d(val), _d(b), _d(x)
    nt = len(row) - 1
    r = np.zeros(nt)
    L.tfo_residual_vector(nt, nt, ip(row), ip(col), ip(dia), dp(val), dp(r), dp(b), dp(x))
    return r


def nrms(row, col, dia, val, r, x, norm=None):
    L = load()
    row, col, dia, val, r, x = _i(row), _i(col), _i(dia), _d(val), _d(r), _d(x)
    nt = len(row) - 1
    return L.tfo_nrms(nt, nt, ip(row), ip(col), ip(dia), dp(val), dp(r), dp(x),
                      0 if norm is None else 1, 0.0 if norm is None else float(norm))


def create_matrix(n_cells, faces_c):
    """Create_Matrix.f90 restated in C: returns (row, col, dia, pos)."""
    L = load()
    fc = np.ascontiguousarray(faces_c, dtype=np.int32)
    nf = len(fc)
    cap = n_cells + 2 * nf
    row = np.zeros(n_cells + 1, np.int32)
    col = np.zeros(max(cap, 1), np.int32)
    dia = np.zeros(n_cells, np.int32)
    pos = np.zeros((nf, 2), np.int32)
    nnz = L.tfo_create_matrix(n_cells, nf, ip(fc), ip(row), ip(col), cap, ip(dia), ip(pos))
    if nnz < 0:
        raise RuntimeError(f"tfo_create_matrix failed: {nnz}")
    return row, col[:nnz].copy(), dia, pos


def face_coef(grid):
    L = load()
    out = np.zeros(grid.n_faces)
    arrs = [_d(getattr(grid, k)) for k in ("sx", "sy", "sz", "dx", "dy", "dz")]
    L.tfo_face_coef(grid.n_faces, *[dp(a) for a in arrs], dp(out))
    return out


def assemble_pressure(grid, pos, dia, nnz, fc, bnd_open=None, v_m=None):
    L = load()
    val = np.zeros(nnz)
    fcs = np.ascontiguousarray(grid.faces_c, dtype=np.int32)
    bo = None if bnd_open is None else _i(bnd_open.astype(np.int32))
    vm = np.ones(grid.n_cells) if v_m is None else _d(v_m)
    L.tfo_assemble_pressure(grid.n_faces, ip(fcs), ip(_i(dia)), ip(_i(pos)), dp(_d(fc)),
                            dp(_d(grid.fw)), dp(vm), ip(bo) if bo is not None else None,
                            dp(val))
    return val


def assemble_momentum(grid, pos, dia, nnz, fc, flux, vis, rho, dt, bnd_wall):
    L = load()
    val = np.zeros(nnz)
    fcs = np.ascontiguousarray(grid.faces_c, dtype=np.int32)
    bw = _i(bnd_wall.astype(np.int32))
    L.tfo_assemble_momentum(grid.n_cells, grid.n_faces, ip(fcs), ip(_i(dia)), ip(_i(pos)),
                            dp(_d(fc)), dp(_d(flux)), ip(bw), float(vis), float(rho),
                            dp(_d(grid.vol)), float(dt), dp(val))
    return val


def max_threads():
    return load().tfo_max_threads()
