"""The reference's own Fortran source against the oracle (CPU, no GPU).

oracle/f90exec.py executes T-Flows' Native_Mod sources (Solve_Native, Cg,
Bicg, Prec_Form, Prec_Solve, Residual_Vector, Normalized_Root_Mean_Square,
Root_Mean_Square) and Solver_Mod/Set_Singular.f90.  These tests pin the C++
oracle (oracle/tf_oracle.cpp, one thread) to it bit for bit on every
preconditioner, with and without `norm`, on the early exits of Cg.f90:95-123,
and on degenerate input (NaN in b, a zero diagonal).  They need the T-Flows
tree and are skipped where it is absent; the committed fixtures carry the
same evidence (tests/golden/make_golden.py writes none unless the reference
source produced it).
"""
import numpy as np
import pytest

from conftest import golden_cases
from oracle import f90exec as F
from oracle import oracle as O
from tflows_b200 import systems

pytestmark = pytest.mark.skipif(not F.available(), reason="T-Flows sources not present")


def both(solver, prec, row, col, dia, val, b, x0, miter, tol, norm):
    v, x, bb = val.copy(), x0.copy(), b.copy()
    o = O.solve_native(solver, prec, row, col, dia, v, x, bb, miter, tol, norm=norm,
                       threads=1)
    r = F.solve_native(solver, prec, row, col, dia, val, x0, b, miter, tol, norm)
    return (x, v, bb, o["niter"], o["fin_res"]), (np.array(r["x"]), np.array(r["val"]),
                                                  np.array(r["b"]), r["niter"], r["fin_res"])


def assert_same(o, r, nan_ok=False):
    for a, b in zip(o[:3], r[:3]):
        assert np.array_equal(a, b, equal_nan=nan_ok)
    assert o[3] == r[3]
    assert o[4] == r[4] or (nan_ok and np.isnan(o[4]) and np.isnan(r[4]))


def test_every_unit_translates():
    P = F.program()
    assert set(P.units) == {"solve_native", "cg", "bicg", "prec_form", "prec_solve",
                            "residual_vector", "normalized_root_mean_square",
                            "root_mean_square", "set_singular"}
    # constants read from Const_Mod.f90
    assert P.consts["micro"] == 1.0e-6 and P.consts["tiny"] == 1.0e-15
    assert P.consts["huge"] == 1.0e15


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c["name"])
def test_reference_source_reproduces_fixture(case):
    r = F.solve_native(case["solver"], case["prec"], case["row"], case["col"], case["dia"],
                       case["val"], case["x0"], case["b"], case["miter"], case["tol"],
                       case["norm"])
    assert r["niter"] == case["niter"] and r["fin_res"] == case["fin_res"]
    assert np.array_equal(r["x"], case["x_out"])
    assert np.array_equal(r["val"], case["val_out"])
    assert np.array_equal(r["b"], case["b_out"])


@pytest.mark.parametrize("solver", ["cg", "bicg"])
@pytest.mark.parametrize("prec", ["jacobi", "icc", "none"])
@pytest.mark.parametrize("norm", [None, 1.0])
def test_reference_source_equals_oracle(solver, prec, norm):
    kind = "momentum" if solver == "bicg" else "pressure"
    kw = {"peclet": 1.0} if kind == "momentum" else {}
    s = systems.small_hex(4, seed=31, kind=kind, ratio=1.07, **kw)
    x0 = np.random.default_rng(4).uniform(-1, 1, s.n)
    o, r = both(solver, prec, s.csr.row, s.csr.col, s.csr.dia, s.val, s.b, x0, 120, 1e-10,
                norm)
    assert_same(o, r)


@pytest.mark.parametrize("prec", ["jacobi", "icc"])
def test_reference_source_equals_oracle_poly(prec):
    p = systems.poly_system(120, seed=9, kind="pressure", tol=1e-10, miter=300, norm=1.0)
    o, r = both("cg", prec, p.csr.row, p.csr.col, p.csr.dia, p.val, p.b, p.x0, 300, 1e-10,
                1.0)
    assert_same(o, r)


def test_early_exits_and_iteration_limits():
    s = systems.small_hex(3, seed=5, kind="pressure")
    row, col, dia = s.csr.row, s.csr.col, s.csr.dia
    cases = [
        (np.zeros(s.n), s.x0, 50),               # bnrm2 < tol: niter 0, fin_res 0
        (s.b, s.x0, 0),                          # miter = 0: the loop never runs
        (s.b, s.x0, 1),                          # one iteration
    ]
    for b, x0, miter in cases:
        o, r = both("cg", "jacobi", row, col, dia, s.val, b, x0, miter, 1e-10, 1.0)
        assert_same(o, r)
    # x0 already the solution: res < tol before the loop (Cg.f90:114-123)
    v, x, bb = s.val.copy(), s.x0.copy(), s.b.copy()
    O.solve_native("cg", "jacobi", row, col, dia, v, x, bb, 500, 1e-14, norm=1.0, threads=1)
    o, r = both("cg", "jacobi", row, col, dia, s.val, s.b, x, 50, 1e-6, 1.0)
    assert_same(o, r)
    assert r[3] == 0


def test_degenerate_input_propagates_like_the_reference():
    """NaN in b and a zero diagonal: no error in the reference, the numbers
    just propagate (Jacobi's 1/0 is inf, then NaN); the oracle must do the
    same, iteration for iteration."""
    s = systems.small_hex(3, seed=6, kind="pressure")
    row, col, dia = s.csr.row, s.csr.col, s.csr.dia
    b = s.b.copy()
    b[4] = np.nan
    o, r = both("cg", "jacobi", row, col, dia, s.val, b, s.x0, 20, 1e-10, 1.0)
    assert_same(o, r, nan_ok=True)
    val = s.val.copy()
    val[dia[7] - 1] = 0.0
    for prec in ("jacobi", "none"):
        o, r = both("cg", prec, row, col, dia, val, s.b, s.x0, 20, 1e-10, 1.0)
        assert_same(o, r, nan_ok=True)


def test_set_singular_and_nrms():
    g = systems.small_hex(4, seed=8, kind="pressure", singular="none")
    ref = np.array(F.set_singular(g.csr.row, g.csr.dia, g.val))
    mine = g.val.copy()
    systems.set_singular(g.csr, mine)
    assert np.array_equal(ref, mine)
    rng = np.random.default_rng(2)
    r, x = rng.uniform(-1, 1, g.n), rng.uniform(-3, 2, g.n)
    for norm in (None, 2.5):
        want = F.nrms(g.csr.row, g.csr.dia, g.val, r, x, norm)
        got = O.nrms(g.csr.row, g.csr.col, g.csr.dia, g.val, r, x, norm=norm)
        assert want == got


def test_unknown_solver_is_error_64():
    s = systems.small_hex(2, seed=1, kind="pressure")
    with pytest.raises(F.FortranRuntimeError) as e:
        F.solve_native("gmres", "jacobi", s.csr.row, s.csr.col, s.csr.dia, s.val, s.x0,
                       s.b, 10, 1e-8, 1.0)
    assert e.value.code == 64


def test_unknown_preconditioner_name_runs_unpreconditioned():
    """Prec_Form / Prec_Solve's else branches: any other name is 'none'
    (tf_solve_native maps names the same way)."""
    s = systems.small_hex(3, seed=3, kind="pressure")
    a = (s.csr.row, s.csr.col, s.csr.dia, s.val, s.x0, s.b, 60, 1e-10, 1.0)
    r1 = F.solve_native("cg", "ilu", *a)
    r2 = F.solve_native("cg", "none", *a)
    assert (r1["niter"], r1["fin_res"], r1["x"]) == (r2["niter"], r2["fin_res"], r2["x"])
