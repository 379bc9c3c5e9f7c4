"""Parity of the FP64 drop-in with the oracle at the workloads' full sizes.

* stretched 200^3 hex (8.0M cells, 55.76M entries): the Cg pressure-
  correction Poisson system and the Bicg momentum system (cell Peclet 1,
  CFL 0.5), tol 1e-10 in the reference's NRMS with norm = 1;
* the 2.0M-cell polyhedral dual of a seeded Delaunay tetrahedralisation:
  the Cg Poisson system, tol 1e-10 x NRMS(b).

Two checks per system, against oracle/tf_oracle.cpp on all host threads:
  - a fixed 50-iteration prefix (tol 0, so both run exactly 50 iterations of
    Cg.f90:139-224): the iterates still agree to rounding, x to rel-L2
    1e-12 and fin_res to 1e-11 relative;
  - the whole solve: x to rel-L2 1e-8, niter within 2 %, fin_res below tol.
The oracle's whole solve of the 200^3 pressure system (~3,400 iterations)
takes about three minutes on 16 host threads.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tflows_b200 import grids, native, systems, workloads

pytestmark = pytest.mark.gpu

PREFIX = 50
PREFIX_X = 1e-12       # rel-L2 of x after the prefix
PREFIX_RES = 1e-11     # relative difference of fin_res after the prefix
REL_L2 = 1e-8          # whole solve
ITER_TOL = 0.02

THREADS = os.cpu_count() or 1


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def stretched200():
    p, m = systems.stretched_pair(200, seed=2, tol=1e-10, miter=20000, ratio=1.02,
                                  peclet=1.0)
    return {"pressure": p, "momentum": m}


@pytest.fixture(scope="module")
def delaunay2m():
    g = grids.poly_dual_grid(2_000_000, 3)
    s = systems.pressure_system(g, 3, tol=1e-10, miter=20000, singular="pin", norm=1.0,
                                name=f"poly-delaunay-{g.n_cells}")
    s.tol = 1e-10 * workloads.nrms_b(s)
    return s


def run_both(ctx, s, miter, tol):
    m = native.Matrix(ctx, s.csr.row, s.csr.col, s.csr.dia)
    try:
        v, x, b = s.val.copy(), s.x0.copy(), s.b.copy()
        it, res = native.solve(ctx, m, s.solver, s.prec, v, x, b, miter, tol, s.norm)
    finally:
        m.close()
    ov, ox, ob = s.val.copy(), s.x0.copy(), s.b.copy()
    r = O.solve_native(s.solver, s.prec, s.csr.row, s.csr.col, s.csr.dia, ov, ox, ob, miter,
                       tol, norm=s.norm, threads=THREADS)
    return (x, it, res), (ox, r["niter"], r["fin_res"])


def report(what, g, o):
    (x, it, res), (ox, oit, ores) = g, o
    print(f"\n{what}: niter {it} (oracle {oit}), rel-L2(x) {rel_l2(x, ox):.2e}, "
          f"fin_res {res:.6e} (oracle {ores:.6e})")


def check_prefix(g, o):
    (x, it, res), (ox, oit, ores) = g, o
    assert it == oit == PREFIX
    assert rel_l2(x, ox) <= PREFIX_X, rel_l2(x, ox)
    assert abs(res - ores) <= PREFIX_RES * ores, (res, ores)


def check_whole(g, o, tol):
    (x, it, res), (ox, oit, ores) = g, o
    assert abs(it - oit) <= max(1, ITER_TOL * oit), (it, oit)
    assert rel_l2(x, ox) <= REL_L2, rel_l2(x, ox)
    assert ores < tol and res < tol, (res, ores, tol)


@pytest.mark.parametrize("kind", ["pressure", "momentum"])
def test_stretched200_prefix(gpu_ctx, stretched200, kind):
    s = stretched200[kind]
    r = run_both(gpu_ctx, s, PREFIX, 0.0)
    report(f"stretched 200^3 {kind}, {PREFIX}-iteration prefix", *r)
    check_prefix(*r)


@pytest.mark.parametrize("kind", ["momentum", "pressure"])
def test_stretched200_whole_solve(gpu_ctx, stretched200, kind):
    s = stretched200[kind]
    r = run_both(gpu_ctx, s, s.miter, s.tol)
    report(f"stretched 200^3 {kind}, whole solve", *r)
    check_whole(*r, s.tol)


def test_delaunay2m_prefix(gpu_ctx, delaunay2m):
    r = run_both(gpu_ctx, delaunay2m, PREFIX, 0.0)
    report(f"Delaunay dual {delaunay2m.n} cells, {PREFIX}-iteration prefix", *r)
    check_prefix(*r)


def test_delaunay2m_whole_solve(gpu_ctx, delaunay2m):
    s = delaunay2m
    r = run_both(gpu_ctx, s, s.miter, s.tol)
    report(f"Delaunay dual {s.n} cells, whole solve", *r)
    check_whole(*r, s.tol)
