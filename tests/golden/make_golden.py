"""Generate the golden fixtures under tests/golden/ (committed).

Each fixture is a seeded system in Matrix_Type layout plus the expected
outputs of Native_Mod's Solve_Native (Cg/Bicg).  The expected outputs are
those of the reference's own Fortran source
(Sources/Process/Cpu/Native_Mod/*.f90, executed by oracle/f90exec.py,
which needs the T-Flows tree), and the script refuses to write a fixture
unless three other evaluations agree with it bit for bit (x, val, b, niter,
fin_res): the C++ restatement (oracle/tf_oracle.cpp, one thread) and the
pure-Python transliteration (oracle/pyref.py).

Two kinds of fixture:
  * small systems stored whole (row, col, dia, val, b, x0 and outputs);
  * `gen_*` fixtures of the 30^3 lid-driven-cavity pressure system (27,000
    cells), stored as the generator call that rebuilds the inputs, a SHA-256
    of those inputs, and the reference source's outputs.  The singular
    system is made solvable both ways the workload allows: one cell pinned
    by an open pressure-boundary face, and the reference's own Set_Singular
    (Solver_Mod/Set_Singular.f90, executed too).

    python tests/golden/make_golden.py            # everything (~2 minutes)
    python tests/golden/make_golden.py --small    # the small fixtures only
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "t-flows_b200"))

import hashlib  # noqa: E402

from oracle import f90exec  # noqa: E402
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


def run_reference(c):
    """The reference's Solve_Native on the case, from its Fortran source."""
    r = f90exec.solve_native(c["solver"], c["prec"], c["row"], c["col"], c["dia"], c["val"],
                             c["x0"], c["b"], c["miter"], c["tol"], c["norm"])
    return np.array(r["x"]), np.array(r["val"]), np.array(r["b"]), r["niter"], r["fin_res"]


def same(a, b):
    return (np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
            and np.array_equal(a[2], b[2]) and a[3] == b[3] and a[4] == b[4])


def input_sha(row, col, dia, val, b, x0):
    h = hashlib.sha256()
    for a in (row, col, dia):
        h.update(np.ascontiguousarray(a, dtype=np.int32).tobytes())
    for a in (val, b, x0):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def ldc30(singular):
    """The 30^3 lid-driven-cavity pressure system; `set_singular` applies the
    reference's own Set_Singular to the unshifted matrix and checks that the
    generator's numpy version gives the same values."""
    if singular == "pin":
        return systems.ldc_pressure_30(seed=1, singular="pin")
    s = systems.ldc_pressure_30(seed=1, singular="none")
    ref_val = np.array(f90exec.set_singular(s.csr.row, s.csr.dia, s.val))
    systems.set_singular(s.csr, s.val)
    if not np.array_equal(ref_val, s.val):
        raise SystemExit("Set_Singular: reference source and generator differ")
    return s


def generated_cases():
    out = []
    for singular in ("pin", "set_singular"):
        out.append(dict(name=f"gen_ldc30_{singular}_cg_jacobi",
                        generator=f"ldc_pressure_30(seed=1, singular={singular!r})",
                        build=lambda singular=singular: ldc30(singular)))
    return out


def main(small_only=False):
    if not f90exec.available():
        raise SystemExit("the T-Flows sources are needed to generate the fixtures")
    for c in cases():
        x, val, b, r = run_oracle(c)
        ref = run_reference(c)
        py = pyref.solve(c["solver"], c["prec"], c["row"], c["col"], c["dia"], c["val"],
                         c["x0"], c["b"], c["miter"], c["tol"], c["norm"])
        py = (np.array(py[0]), np.array(py[1]), np.array(py[2]), py[3], py[4])
        if not same(ref, (x, val, b, r["niter"], r["fin_res"])):
            raise SystemExit(f"{c['name']}: reference source and C++ oracle differ")
        if not same(ref, py):
            raise SystemExit(f"{c['name']}: reference source and Python transliteration differ")
        path = os.path.join(HERE, c["name"] + ".npz")
        np.savez_compressed(
            path, row=c["row"], col=c["col"], dia=c["dia"], val=c["val"], b=c["b"],
            x0=c["x0"], solver=c["solver"], prec=c["prec"], miter=c["miter"], tol=c["tol"],
            norm=np.nan if c["norm"] is None else c["norm"], x_out=ref[0], val_out=ref[1],
            b_out=ref[2], niter=ref[3], fin_res=ref[4], hist=r["hist"],
            source="reference Fortran source via oracle/f90exec.py")
        print(f"{c['name']}: n={len(c['row']) - 1} niter={r['niter']} "
              f"fin_res={r['fin_res']:.3e} (reference source = C++ oracle = pyref)")
    if small_only:
        return
    for g in generated_cases():
        s = g["build"]()
        c = dict(row=s.csr.row, col=s.csr.col, dia=s.csr.dia, val=s.val, b=s.b, x0=s.x0,
                 solver=s.solver, prec=s.prec, miter=s.miter, tol=s.tol, norm=s.norm)
        x, val, b, r = run_oracle(c)
        ref = run_reference(c)
        if not same(ref, (x, val, b, r["niter"], r["fin_res"])):
            raise SystemExit(f"{g['name']}: reference source and C++ oracle differ")
        path = os.path.join(HERE, g["name"] + ".npz")
        np.savez_compressed(
            path, generator=g["generator"],
            input_sha256=input_sha(c["row"], c["col"], c["dia"], c["val"], c["b"], c["x0"]),
            solver=c["solver"], prec=c["prec"], miter=c["miter"], tol=c["tol"],
            norm=np.nan if c["norm"] is None else c["norm"], x_out=ref[0], niter=ref[3],
            fin_res=ref[4], hist=r["hist"],
            source="reference Fortran source via oracle/f90exec.py")
        print(f"{g['name']}: n={s.n} niter={ref[3]} fin_res={ref[4]:.3e} "
              f"(reference source = C++ oracle)")


if __name__ == "__main__":
    main(small_only="--small" in sys.argv)
