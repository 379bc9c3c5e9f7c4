"""MatrixMarket (.mtx) import and export of Matrix_Type systems.

T-Flows analyses its matrices with scipy from a MatrixMarket file
(Sources/Utilities/analyze_matrix.py reads "t-flows.mtx" with
scipy.io.mmread).  `write_matrix` writes a Matrix_Type (1-based CSR, the
diagonal first in each row) in that format, entries row by row in storage
order, values with 17 significant digits so that a round trip is exact.
`read_matrix` reads any coordinate MatrixMarket matrix back into the
Matrix_Type layout: per row the diagonal first, then the other entries by
ascending column (Create_Matrix.f90:112-119), duplicates summed in file
order; a row without a stored diagonal gets an explicit 0.0 diagonal.

Command line (runs the system on the GPU through the drop-in):

    python -m tflows_b200.mtx solve A.mtx [--rhs b.mtx] [--x0 x0.mtx]
        [--solver cg|bicg] [--prec jacobi|icc|none] [--tol 1e-10]
        [--miter 10000] [--norm 1.0] [--out x.mtx]
"""
import argparse
import sys

import numpy as np

from .systems import Csr


def write_matrix(path, csr, val, comment=""):
    """Matrix_Type (row/col 1-based, val) -> MatrixMarket coordinate real general."""
    n, nnz = csr.n, csr.nnz
    rows = np.repeat(np.arange(1, n + 1), np.diff(csr.row))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        for line in comment.splitlines():
            f.write(f"% {line}\n")
        f.write(f"{n} {n} {nnz}\n")
        for i, j, v in zip(rows, csr.col[:nnz], val[:nnz]):
            f.write(f"{i} {j} {float(v):.17g}\n")


def write_vector(path, v, comment=""):
    """A dense vector as a MatrixMarket array (n x 1)."""
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix array real general\n")
        for line in comment.splitlines():
            f.write(f"% {line}\n")
        f.write(f"{len(v)} 1\n")
        for x in v:
            f.write(f"{float(x):.17g}\n")


def _header(f):
    line = f.readline()
    if not line.startswith("%%MatrixMarket"):
        raise ValueError("not a MatrixMarket file")
    words = line.lower().split()
    if words[1] != "matrix" or words[3] != "real" and words[3] != "integer":
        raise ValueError(f"unsupported MatrixMarket object: {line.strip()}")
    fmt, sym = words[2], words[4]
    line = f.readline()
    while line.startswith("%"):
        line = f.readline()
    return fmt, sym, [int(t) for t in line.split()]


def read_vector(path):
    with open(path) as f:
        fmt, _, dims = _header(f)
        if fmt == "array":
            data = np.array(f.read().split(), dtype=np.float64)
            return data[: dims[0] * dims[1]]
        # coordinate n x 1
        n, _, nnz = dims
        v = np.zeros(n)
        for _ in range(nnz):
            i, _, x = f.readline().split()
            v[int(i) - 1] += float(x)
        return v


def read_matrix(path):
    """MatrixMarket coordinate matrix -> (Csr, val) in the Matrix_Type layout."""
    with open(path) as f:
        fmt, sym, dims = _header(f)
        if fmt != "coordinate":
            raise ValueError("matrix must be in coordinate format")
        n, m, nnz = dims
        if n != m:
            raise ValueError(f"matrix is {n} x {m}, not square")
        data = np.loadtxt(f, ndmin=2, max_rows=nnz) if nnz else np.zeros((0, 3))
    i = data[:, 0].astype(np.int64) - 1
    j = data[:, 1].astype(np.int64) - 1
    v = data[:, 2].astype(np.float64)
    if sym in ("symmetric", "skew-symmetric"):
        off = i != j
        sgn = -1.0 if sym == "skew-symmetric" else 1.0
        i, j, v = (np.concatenate([i, j[off]]), np.concatenate([j, i[off]]),
                   np.concatenate([v, sgn * v[off]]))
    # rows without a stored diagonal get an explicit zero
    has_diag = np.zeros(n, bool)
    has_diag[i[i == j]] = True
    miss = np.nonzero(~has_diag)[0]
    i = np.concatenate([i, miss])
    j = np.concatenate([j, miss])
    v = np.concatenate([v, np.zeros(len(miss))])
    # duplicates summed in file order, then per row: diagonal, ascending columns
    key = i * n + j
    order = np.argsort(key, kind="stable")
    key, v = key[order], v[order]
    uniq, start = np.unique(key, return_index=True)
    sums = np.array([sum(v[a:b]) for a, b in zip(start, list(start[1:]) + [len(v)])]) \
        if len(uniq) != len(key) else v
    ii, jj = uniq // n, uniq % n
    first = np.where(ii == jj, 0, 1)
    order = np.lexsort((jj, first, ii))
    ii, jj, vals = ii[order], jj[order], sums[order]
    counts = np.bincount(ii, minlength=n)
    row = np.concatenate([[1], 1 + np.cumsum(counts)]).astype(np.int32)
    col = (jj + 1).astype(np.int32)
    dia = row[:-1].copy()
    return Csr(n=n, row=row, col=col, dia=dia, pos=np.zeros((0, 2), np.int32)), vals


def _main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m tflows_b200.mtx")
    sub = ap.add_subparsers(dest="cmd", required=True)
    sp = sub.add_parser("solve", help="solve A x = b on the GPU through the drop-in")
    sp.add_argument("matrix")
    sp.add_argument("--rhs")
    sp.add_argument("--x0")
    sp.add_argument("--solver", default="cg", choices=["cg", "bicg"])
    sp.add_argument("--prec", default="jacobi", choices=["jacobi", "icc", "none"])
    sp.add_argument("--tol", type=float, default=1e-10)
    sp.add_argument("--miter", type=int, default=10000)
    sp.add_argument("--norm", type=float, default=None)
    sp.add_argument("--out")
    a = ap.parse_args(argv)
    from . import native
    csr, val = read_matrix(a.matrix)
    b = read_vector(a.rhs) if a.rhs else np.ones(csr.n)
    x = read_vector(a.x0) if a.x0 else np.zeros(csr.n)
    ctx = native.Context(0)
    m = native.Matrix(ctx, csr.row, csr.col, csr.dia)
    try:
        it, res = native.solve(ctx, m, a.solver, a.prec, val.copy(), x, b.copy(), a.miter,
                               a.tol, a.norm)
    finally:
        m.close()
        ctx.close()
    print(f"n {csr.n} nnz {csr.nnz} niter {it} fin_res {res:.6e}")
    if a.out:
        write_vector(a.out, x, comment=f"solution: {a.solver}/{a.prec}, niter {it}")
    return 0


if __name__ == "__main__":
    sys.exit(_main())
