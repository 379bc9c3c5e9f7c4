"""CPU tests of the oracle (the C++ restatement of Native_Mod) and of the
synthetic-system generators.  No GPU needed."""
import numpy as np
import pytest
import scipy.sparse as sps
import scipy.sparse.linalg as spla

from conftest import build_generated, generated_cases, golden_cases
from oracle import oracle as O
from oracle import pyref
from tflows_b200 import grids, systems


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c["name"])
def test_oracle_reproduces_golden(case):
    val, x, b = case["val"].copy(), case["x0"].copy(), case["b"].copy()
    r = O.solve_native(case["solver"], case["prec"], case["row"], case["col"], case["dia"],
                       val, x, b, case["miter"], case["tol"], norm=case["norm"], threads=1,
                       history=True)
    assert r["niter"] == case["niter"]
    assert r["fin_res"] == case["fin_res"]
    assert np.array_equal(x, case["x_out"])
    assert np.array_equal(val, case["val_out"])
    assert np.array_equal(b, case["b_out"])
    assert np.array_equal(r["hist"], case["hist"])


@pytest.mark.parametrize("solver", ["cg", "bicg"])
@pytest.mark.parametrize("prec", ["jacobi", "none", "icc"])
@pytest.mark.parametrize("norm", [None, 1.0])
def test_oracle_matches_python_transliteration(solver, prec, norm):
    s = systems.small_hex(4, seed=21, kind="momentum" if solver == "bicg" else "pressure",
                          tol=1e-9, miter=200, ratio=1.05, **({"peclet": 1.0} if solver == "bicg" else {}))
    x0 = np.random.default_rng(3).uniform(-1, 1, s.n)
    val, x, b = s.val.copy(), x0.copy(), s.b.copy()
    r = O.solve_native(solver, prec, s.csr.row, s.csr.col, s.csr.dia, val, x, b, 200, 1e-9,
                       norm=norm)
    px, pval, pb, pit, pres = pyref.solve(solver, prec, s.csr.row, s.csr.col, s.csr.dia,
                                          s.val, x0, s.b, 200, 1e-9, norm)
    assert (r["niter"], r["fin_res"]) == (pit, pres)
    assert np.array_equal(x, px) and np.array_equal(val, pval) and np.array_equal(b, pb)


def test_example_4x4_layout():
    """Matrix_Mod.f90:44-55: the CSR of the hand example holds the dense matrix.
    (The comment's dia(3) = 9 is a typo for 8; the fixture uses 8.)"""
    from golden.make_golden import example_4x4
    row, col, dia, val = example_4x4()
    dense = np.array([[10, 0, 4, 5], [2, 12, -1, 0], [0, 1, 99, 7], [-3, 11, 0, 53]], float)
    A = sps.csr_matrix((val, col - 1, row - 1), shape=(4, 4)).toarray()
    assert np.array_equal(A, dense)
    assert all(col[dia[i] - 1] == i + 1 for i in range(4))
    p = np.array([1.0, -2.0, 0.5, 3.0])
    assert np.array_equal(O.spmv(row, col, dia, val, p), dense @ p)


@pytest.mark.parametrize("ratio", [1.0, 1.1])
def test_create_matrix_numpy_equals_restatement(ratio):
    g = grids.hex_grid(5, 4, 6, stretch_y=ratio)
    c = systems.create_matrix(g)
    row, col, dia, pos = O.create_matrix(g.n_cells, g.faces_c)
    assert np.array_equal(c.row, row) and np.array_equal(c.col, col)
    assert np.array_equal(c.dia, dia) and np.array_equal(c.pos, pos)
    # diagonal first, the rest ascending (Create_Matrix.f90:112-119)
    for i in range(g.n_cells):
        seg = c.col[c.row[i] - 1:c.row[i + 1] - 1]
        assert seg[0] == i + 1 and np.all(np.diff(seg[1:]) > 0)


def test_create_matrix_poly():
    g = grids.poly_dual_grid(300, seed=5)
    c = systems.create_matrix(g)
    row, col, dia, pos = O.create_matrix(g.n_cells, g.faces_c)
    assert np.array_equal(c.col, col) and np.array_equal(c.pos, pos)
    assert 10 <= g.meta["faces_per_cell_mean"] <= 18


def test_assembly_equals_restatement():
    g = grids.hex_grid(5, 6, 4, stretch_y=1.1)
    c = systems.create_matrix(g)
    fc = systems.face_coef(g)
    assert np.array_equal(fc, O.face_coef(g))
    bo = np.zeros(g.n_faces, bool)
    bo[np.nonzero((~g.interior) & (g.faces_c[:, 0] == 1))[0][0]] = True
    assert np.array_equal(systems.assemble_pressure(g, c, fc, bnd_open=bo),
                          O.assemble_pressure(g, c.pos, c.dia, c.nnz, fc, bo))
    flux = np.where(g.interior, np.linspace(-1, 1, g.n_faces) * 1e-3, 0.0)
    assert np.array_equal(systems.assemble_momentum(g, c, fc, flux, 2e-3, 1.0, 0.01),
                          O.assemble_momentum(g, c.pos, c.dia, c.nnz, fc, flux, 2e-3, 1.0,
                                              0.01, ~g.interior))


def test_bicg_equals_cg_bitwise():
    """Bicg.f90:129-133 sets r2 = r1 and never forms A^T, so its iterates are Cg's."""
    s = systems.small_hex(6, seed=4, kind="momentum", tol=1e-10, miter=300, peclet=2.0)
    outs = []
    for solver in ("cg", "bicg"):
        v, x, b = s.val.copy(), s.x0.copy(), s.b.copy()
        r = O.solve_native(solver, "jacobi", s.csr.row, s.csr.col, s.csr.dia, v, x, b, 300,
                           1e-10, norm=1.0, history=True)
        outs.append((x, v, b, r))
    (x1, v1, b1, r1), (x2, v2, b2, r2) = outs
    assert r1["niter"] == r2["niter"] and r1["fin_res"] == r2["fin_res"]
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2) and np.array_equal(b1, b2)


def test_pcg_iterates_match_scipy():
    """The oracle's x after k iterations equals scipy's Jacobi-PCG iterate x_k."""
    s = systems.small_hex(7, seed=8, kind="pressure", ratio=1.05)
    A = sps.csr_matrix((s.val, s.csr.col - 1, s.csr.row - 1), shape=(s.n, s.n))
    M = sps.diags(1.0 / s.val[s.csr.dia - 1])
    xs = []
    spla.cg(A, s.b, x0=np.zeros(s.n), M=M, rtol=1e-300, atol=0.0, maxiter=25,
            callback=lambda xk: xs.append(xk.copy()))
    for k in (1, 2, 5, 10, 25):
        v, x, b = s.val.copy(), np.zeros(s.n), s.b.copy()
        r = O.solve_native("cg", "jacobi", s.csr.row, s.csr.col, s.csr.dia, v, x, b, k,
                           0.0, norm=1.0)
        assert r["niter"] == k
        err = np.linalg.norm(x - xs[k - 1]) / np.linalg.norm(xs[k - 1])
        assert err < 1e-10, (k, err)


def test_converged_solution_solves_system():
    s = systems.small_hex(8, seed=9, kind="pressure", ratio=1.02, tol=1e-12, miter=1000)
    v, x, b = s.val.copy(), s.x0.copy(), s.b.copy()
    r = O.solve_native("cg", "jacobi", s.csr.row, s.csr.col, s.csr.dia, v, x, b, 1000, 1e-12,
                       norm=1.0)
    A = sps.csr_matrix((s.val, s.csr.col - 1, s.csr.row - 1), shape=(s.n, s.n))
    xs = spla.spsolve(A.tocsc(), s.b)
    assert r["fin_res"] < 1e-12
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-9


def test_early_exits_and_zero_trip():
    s = systems.small_hex(4, seed=1, kind="pressure")
    row, col, dia = s.csr.row, s.csr.col, s.csr.dia
    # b = 0: bnrm2 < tol -> niter 0, fin_res 0.0, x untouched (Cg.f90:101-104)
    v, x, b = s.val.copy(), np.full(s.n, 0.25), np.zeros(s.n)
    r = O.solve_native("cg", "jacobi", row, col, dia, v, x, b, 100, 1e-6, norm=1.0)
    assert r == dict(niter=0, fin_res=0.0) and np.all(x == 0.25)
    # miter = 0: loop does not run, fin_res is the initial residual
    v, x, b = s.val.copy(), np.zeros(s.n), s.b.copy()
    r = O.solve_native("cg", "jacobi", row, col, dia, v, x, b, 0, 1e-6, norm=1.0)
    assert r["niter"] == 0 and r["fin_res"] > 1e-6 and np.all(x == 0.0)
    # x already the solution: res < tol before the loop (Cg.f90:120-123)
    v, x, b = s.val.copy(), np.zeros(s.n), s.b.copy()
    O.solve_native("cg", "jacobi", row, col, dia, v, x, b, 500, 1e-13, norm=1.0)
    v2, b2 = s.val.copy(), s.b.copy()
    r = O.solve_native("cg", "jacobi", row, col, dia, v2, x, b2, 500, 1e-11, norm=1.0)
    assert r["niter"] == 0 and r["fin_res"] < 1e-11


def test_unknown_solver_code():
    s = systems.small_hex(3, seed=1, kind="pressure")
    L = O.load()
    import ctypes
    v, x, b = s.val.copy(), s.x0.copy(), s.b.copy()
    st = L.tfo_solve_native(7, 1, s.n, s.n, O.ip(s.csr.row), O.ip(s.csr.col),
                            O.ip(s.csr.dia), O.dp(v), O.dp(x), O.dp(b), 10,
                            ctypes.byref(ctypes.c_int()), 1e-6,
                            ctypes.byref(ctypes.c_double()), 0, 0.0, None)
    assert st == 64   # Solve_Native.f90:38, Message % Error(64, ...)


def test_nrms_definition():
    s = systems.small_hex(5, seed=2, kind="pressure")
    r = np.random.default_rng(0).standard_normal(s.n)
    x = np.random.default_rng(1).standard_normal(s.n)
    a = s.val[s.csr.dia - 1]
    want = np.sqrt(np.sum(r * r / (a * a))) / (x.max() - x.min())
    got = O.nrms(s.csr.row, s.csr.col, s.csr.dia, s.val, r, x)
    assert abs(got - want) <= 1e-13 * want
    assert O.nrms(s.csr.row, s.csr.col, s.csr.dia, s.val, r, x, norm=2.0) == pytest.approx(
        np.sqrt(np.sum(r * r / (a * a))) / 2.0, rel=1e-13)


@pytest.mark.parametrize("case", generated_cases(), ids=lambda c: c["name"])
def test_generated_fixture_inputs_are_reproducible(case):
    """The 30^3 fixtures hold the reference source's outputs; their inputs
    are rebuilt from the generator (SHA-256 checked) -- here without the
    reference: the oracle must reproduce them bit for bit."""
    s = build_generated(case)
    v, x, bb = s.val.copy(), s.x0.copy(), s.b.copy()
    o = O.solve_native(case["solver"], case["prec"], s.csr.row, s.csr.col, s.csr.dia, v, x,
                       bb, case["miter"], case["tol"], norm=case["norm"], threads=1)
    assert o["niter"] == case["niter"] and o["fin_res"] == case["fin_res"]
    assert np.array_equal(x, case["x_out"])
