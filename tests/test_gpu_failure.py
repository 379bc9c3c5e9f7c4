"""Failure paths of the drop-in, made without faulting the GPU.

* The watchdog: the context's limit is set to a nanosecond, so the SpMV
  streamers' first waits for a tile's copies come after their deadline and
  give up; the solve must end with TF_ERR_TIMEOUT (the CTAs still wait for
  the copies they started, with the default limit, before exiting), and
  the same context must then solve normally again.  Run on the row-pattern
  streamer (hex) and on the CSR streamer (polyhedral).
* Degenerate input the reference does not reject (Message_Mod/Error.f90 is
  never reached for it): NaN in b and a zero diagonal.  The numbers
  propagate; the drop-in must run the same iterations as the oracle (which
  is pinned to the reference's own source) and produce NaN/inf where it
  does.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tflows_b200 import native, systems

pytestmark = pytest.mark.gpu


def oracle(s, val, b, miter, tol, norm, prec="jacobi"):
    v, x, bb = val.copy(), s.x0.copy(), b.copy()
    r = O.solve_native("cg", prec, s.csr.row, s.csr.col, s.csr.dia, v, x, bb, miter, tol,
                       norm=norm, threads=8)
    return x, r["niter"], r["fin_res"]


def gpu(ctx, m, s, val, b, miter, tol, norm, prec="jacobi"):
    v, x, bb = val.copy(), s.x0.copy(), b.copy()
    it, res = native.solve(ctx, m, "cg", prec, v, x, bb, miter, tol, norm)
    return x, it, res


@pytest.mark.parametrize("kind", ["hex-row-patterns", "poly-csr-tiles"])
def test_wait_limit_runs_out_then_context_recovers(kind, monkeypatch):
    if kind == "hex-row-patterns":
        s = systems.small_hex(64, seed=4, kind="pressure", ratio=1.02)
    else:
        monkeypatch.setenv("TF_TILE_CFG", "6")   # variable CSR tiles, 4 lanes per row
        s = systems.poly_system(60000, seed=5, kind="pressure", tol=1e-10, miter=5000,
                                norm=1.0)
    ctx = native.Context(0)
    try:
        m = native.Matrix(ctx, s.csr.row, s.csr.col, s.csr.dia)
        try:
            ctx.set_wait_limit(1e-9)
            with pytest.raises(native.TFError) as e:
                gpu(ctx, m, s, s.val, s.b, 200, 1e-10, 1.0)
            assert e.value.status == 4                     # TF_ERR_TIMEOUT
            ctx.set_wait_limit(0.0)                        # back to the default
            x, it, res = gpu(ctx, m, s, s.val, s.b, 5000, 1e-10, 1.0)
            ox, oit, ores = oracle(s, s.val, s.b, 5000, 1e-10, 1.0)
            assert abs(it - oit) <= max(1, 0.02 * oit) and res < 1e-10
            assert np.linalg.norm(x - ox) <= 1e-8 * np.linalg.norm(ox)
        finally:
            m.close()
    finally:
        ctx.close()


def test_wait_limit_argument_checks(gpu_ctx):
    with pytest.raises(native.TFError):
        gpu_ctx.set_wait_limit(-1.0)
    gpu_ctx.set_wait_limit(0.0)


def same_propagation(g, o):
    x, it, res = g
    ox, oit, ores = o
    assert it == oit
    assert np.array_equal(np.isnan(x), np.isnan(ox))
    assert np.array_equal(np.isinf(x), np.isinf(ox))
    fin = np.isfinite(ox)
    if fin.any():
        assert np.allclose(x[fin], ox[fin], rtol=1e-8, atol=1e-12)
    assert (np.isnan(res) and np.isnan(ores)) or res == pytest.approx(ores, rel=1e-8)


@pytest.mark.parametrize("n", [6, 40])
def test_nan_in_rhs_propagates_like_the_reference(gpu_ctx, n):
    s = systems.small_hex(n, seed=6, kind="pressure")
    b = s.b.copy()
    b[s.n // 3] = np.nan
    m = native.Matrix(gpu_ctx, s.csr.row, s.csr.col, s.csr.dia)
    try:
        g = gpu(gpu_ctx, m, s, s.val, b, 25, 1e-10, 1.0)
    finally:
        m.close()
    o = oracle(s, s.val, b, 25, 1e-10, 1.0)
    assert o[1] == 25          # NaN never compares below tol: the loop runs out
    same_propagation(g, o)


@pytest.mark.parametrize("prec", ["jacobi", "none"])
def test_zero_diagonal_propagates_like_the_reference(gpu_ctx, prec):
    s = systems.small_hex(6, seed=7, kind="pressure")
    val = s.val.copy()
    val[s.csr.dia[11] - 1] = 0.0
    m = native.Matrix(gpu_ctx, s.csr.row, s.csr.col, s.csr.dia)
    try:
        g = gpu(gpu_ctx, m, s, val, s.b, 25, 1e-10, 1.0, prec)
    finally:
        m.close()
    same_propagation(g, oracle(s, val, s.b, 25, 1e-10, 1.0, prec))
