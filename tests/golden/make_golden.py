"""Generate the golden fixtures under tests/golden/ (committed).

Each fixture is a small seeded system in Matrix_Type layout plus the
expected outputs of Native_Mod's Cg/Bicg.  The expected outputs come from
the C++ restatement (oracle/tf_oracle.cpp, one thread) and are cross-checked
here, bit for bit, against the independent pure-Python transliteration
(oracle/pyref.py); the script refuses to write a fixture on any mismatch.
The reference itself cannot be run here (it is Fortran and no Fortran
compiler exists), so these fixtures pin the restatements against each other
and against the hand example of Matrix_Mod.f90:44-55, not against reference
output.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "t-flows_b200"))

from oracle import oracle as O  # noqa: E402
from oracle import pyref  # noqa: E402
from tflows_b200 import grids, systems  # noqa: E402


def example_4x4():
    """Matrix_Mod.f90:44-55, with row completed by row(5) = 13 and dia(3)
    corrected to 8: the comment lists dia = [1 5 9 12], but entry 9 is
    (row 3, col 4); the diagonal 99 of row 3 is entry 8."""
    val = np.array([10, 4, 5, 2, 12, -1, 1, 99, 7, -3, 11, 53], dtype=np.float64)
    col = np.array([1, 3, 4, 1, 2, 3, 2, 3, 4, 1, 2, 4], dtype=np.int32)
    row = np.array([1, 4, 7, 10, 13], dtype=np.int32)
    dia = np.array([1, 5, 8, 12], dtype=np.int32)
    return row, col, dia, val


def cases():
    out = []
    row, col, dia, val = example_4x4()
    b = np.array([1.0, 2.0, 3.0, 4.0])
    for solver in ("cg", "bicg"):
        out.append(dict(name=f"example4x4_{solver}_jacobi", row=row, col=col, dia=dia,
                        val=val, b=b, x0=np.zeros(4), solver=solver, prec="jacobi",
                        miter=50, tol=1e-12, norm=None))
    s = systems.small_hex(5, seed=11, kind="pressure", tol=1e-10, miter=500)
    out.append(dict(name="hex5_pressure_cg_jacobi", row=s.csr.row, col=s.csr.col,
                    dia=s.csr.dia, val=s.val, b=s.b, x0=s.x0, solver="cg", prec="jacobi",
                    miter=500, tol=1e-10, norm=1.0))
    out.append(dict(name="hex5_pressure_cg_none_nonorm", row=s.csr.row, col=s.csr.col,
                    dia=s.csr.dia, val=s.val, b=s.b, x0=s.x0, solver="cg", prec="none",
                    miter=500, tol=1e-9, norm=None))
    out.append(dict(name="hex5_pressure_cg_icc", row=s.csr.row, col=s.csr.col,
                    dia=s.csr.dia, val=s.val, b=s.b, x0=s.x0, solver="cg", prec="icc",
                    miter=500, tol=1e-10, norm=1.0))
    m = systems.small_hex(4, seed=12, kind="momentum", tol=1e-10, miter=400, peclet=1.0,
                          ratio=1.1)
    out.append(dict(name="hex4_momentum_bicg_jacobi", row=m.csr.row, col=m.csr.col,
                    dia=m.csr.dia, val=m.val, b=m.b, x0=m.x0, solver="bicg", prec="jacobi",
                    miter=400, tol=1e-10, norm=1.0))
    m10 = systems.small_hex(4, seed=13, kind="momentum", tol=1e-10, miter=60, peclet=10.0,
                            ratio=1.1)
    out.append(dict(name="hex4_momentum_pe10_bicg_diverging", row=m10.csr.row,
                    col=m10.csr.col, dia=m10.csr.dia, val=m10.val, b=m10.b, x0=m10.x0,
                    solver="bicg", prec="jacobi", miter=60, tol=1e-10, norm=1.0))
    out.append(dict(name="hex4_momentum_bicg_icc", row=m.csr.row, col=m.csr.col,
                    dia=m.csr.dia, val=m.val, b=m.b, x0=m.x0, solver="bicg", prec="icc",
                    miter=400, tol=1e-10, norm=None))
    p = systems.poly_system(150, seed=14, kind="pressure", tol=1e-10, miter=500, norm=1.0)
    x0 = np.random.default_rng(15).uniform(-0.1, 0.1, p.n)
    out.append(dict(name="poly150_pressure_cg_jacobi_x0", row=p.csr.row, col=p.csr.col,
                    dia=p.csr.dia, val=p.val, b=p.b, x0=x0, solver="cg", prec="jacobi",
                    miter=500, tol=1e-10, norm=1.0))
    return out


def run_oracle(c):
    val, x, b = c["val"].copy(), c["x0"].copy(), c["b"].copy()
    r = O.solve_native(c["solver"], c["prec"], c["row"], c["col"], c["dia"], val, x, b,
                       c["miter"], c["tol"], norm=c["norm"], threads=1, history=True)
    return x, val, b, r


def main():
    for c in cases():
        x, val, b, r = run_oracle(c)
        px, pval, pb, pit, pres = pyref.solve(c["solver"], c["prec"], c["row"], c["col"],
                                              c["dia"], c["val"], c["x0"], c["b"],
                                              c["miter"], c["tol"], c["norm"])
        same = (np.array_equal(x, np.array(px)) and np.array_equal(val, np.array(pval))
                and np.array_equal(b, np.array(pb)) and r["niter"] == pit
                and r["fin_res"] == pres)
        if not same:
            raise SystemExit(f"{c['name']}: C++ oracle and Python transliteration differ")
        path = os.path.join(HERE, c["name"] + ".npz")
        np.savez_compressed(
            path, row=c["row"], col=c["col"], dia=c["dia"], val=c["val"], b=c["b"],
            x0=c["x0"], solver=c["solver"], prec=c["prec"], miter=c["miter"], tol=c["tol"],
            norm=np.nan if c["norm"] is None else c["norm"], x_out=x, val_out=val,
            b_out=b, niter=r["niter"], fin_res=r["fin_res"], hist=r["hist"])
        print(f"{c['name']}: n={len(c['row']) - 1} niter={r['niter']} "
              f"fin_res={r['fin_res']:.3e}")


if __name__ == "__main__":
    main()
