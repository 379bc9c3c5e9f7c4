"""Multi-RHS solves (one matrix, up to four right-hand sides): each
right-hand side gives exactly its own tf_solve result on row-pattern
matrices, and the oracle's within the usual bars everywhere."""
import numpy as np
import pytest

from oracle import oracle as O
from tflows_b200 import grids, native, systems

pytestmark = pytest.mark.gpu


def _single(ctx, m, s, prec, b, x0, miter, tol, norm):
    v, x, bb = s.val.copy(), x0.copy(), b.copy()
    it, res = native.solve(ctx, m, "bicg", prec, v, x, bb, miter, tol, norm)
    return x, v, bb, it, res


@pytest.mark.parametrize("prec", ["jacobi", "none"])
@pytest.mark.parametrize("norm", [1.0, None])
@pytest.mark.parametrize("nrhs", [1, 3, 4])
def test_multi_rhs_equals_single_solves_bitwise(gpu_ctx, prec, norm, nrhs):
    s = systems.small_hex(21, seed=4, kind="momentum", peclet=1.0, ratio=1.02)
    rng = np.random.default_rng(7)
    B = np.ascontiguousarray(rng.uniform(-1, 1, (nrhs, s.n)))
    X0 = np.ascontiguousarray(rng.uniform(-0.1, 0.1, (nrhs, s.n)))
    if nrhs > 1:
        B[1] *= 1e-3                   # converges at another iteration
    m = native.Matrix(gpu_ctx, s.csr.row, s.csr.col, s.csr.dia)
    try:
        assert m.row_patterns > 0
        ref = [_single(gpu_ctx, m, s, prec, B[i], X0[i], 2000, 1e-10, norm) for i in range(nrhs)]
        val, X, Bm = s.val.copy(), X0.copy(), B.copy()
        its, res = native.solve_multi(gpu_ctx, m, "bicg", prec, val, X, Bm, 2000, 1e-10, norm)
    finally:
        m.close()
    for i in range(nrhs):
        x, v, bb, it, r = ref[i]
        assert (its[i], res[i]) == (it, r)
        assert np.array_equal(X[i], x) and np.array_equal(Bm[i], bb)
        assert np.array_equal(val, v)


def test_multi_rhs_early_exits_and_miter(gpu_ctx):
    """A zero right-hand side stops at iteration 0 with fin_res 0 (Cg.f90:101-104)
    while the others run; miter caps each one."""
    s = systems.small_hex(15, seed=2, kind="pressure", ratio=1.03)
    rng = np.random.default_rng(3)
    B = np.ascontiguousarray(np.stack([s.b, np.zeros(s.n), rng.uniform(-1, 1, s.n)]))
    X = np.zeros_like(B)
    m = native.Matrix(gpu_ctx, s.csr.row, s.csr.col, s.csr.dia)
    try:
        its, res = native.solve_multi(gpu_ctx, m, "cg", "jacobi", s.val.copy(), X, B.copy(),
                                      7, 1e-12, 1.0)
    finally:
        m.close()
    assert its == [7, 0, 7] and res[1] == 0.0 and np.all(X[1] == 0.0)


def test_multi_rhs_on_csr_matrices_matches_oracle(gpu_ctx):
    """Without row patterns (polyhedral mesh) the matrix is read by a
    thread-per-row SpMV: same row sums, dot products in another order."""
    g = grids.poly_lattice_grid(4000, 9)
    s = systems.momentum_system(g, 9, tol=1e-10, miter=3000, peclet=5.0, cfl=0.1)
    rng = np.random.default_rng(1)
    B = np.ascontiguousarray(rng.uniform(-1, 1, (3, s.n)))
    X = np.zeros_like(B)
    m = native.Matrix(gpu_ctx, s.csr.row, s.csr.col, s.csr.dia)
    try:
        assert m.row_patterns == 0
        its, res = native.solve_multi(gpu_ctx, m, "bicg", "jacobi", s.val.copy(), X, B.copy(),
                                      3000, 1e-10, 1.0)
    finally:
        m.close()
    for i in range(3):
        v, x, b = s.val.copy(), np.zeros(s.n), B[i].copy()
        o = O.solve_native("bicg", "jacobi", s.csr.row, s.csr.col, s.csr.dia, v, x, b, 3000,
                           1e-10, norm=1.0)
        assert abs(its[i] - o["niter"]) <= max(1, 0.02 * o["niter"])
        assert np.linalg.norm(X[i] - x) <= 1e-8 * np.linalg.norm(x)
        assert res[i] < 1e-10


def test_multi_rhs_rejects_icc_and_too_many(gpu_ctx):
    s = systems.small_hex(5, seed=1, kind="pressure")
    m = native.Matrix(gpu_ctx, s.csr.row, s.csr.col, s.csr.dia)
    try:
        for prec, nr in (("icc", 2), ("jacobi", 5)):
            X = np.zeros((nr, s.n))
            with pytest.raises(native.TFError):
                native.solve_multi(gpu_ctx, m, "cg", prec, s.val.copy(), X, np.ones((nr, s.n)),
                                   10, 1e-8, 1.0)
    finally:
        m.close()
