"""MatrixMarket import/export of Matrix_Type systems (CPU)."""
import io

import numpy as np
import pytest
import scipy.io
import scipy.sparse as sps

from oracle import oracle as O
from tflows_b200 import mtx, systems


def _csr_scipy(csr, val):
    return sps.csr_matrix((val, csr.col - 1, csr.row - 1), shape=(csr.n, csr.n))


@pytest.mark.parametrize("kind", ["hex", "poly"])
def test_round_trip_is_exact(tmp_path, kind):
    s = (systems.small_hex(7, seed=2, kind="momentum", peclet=2.0, ratio=1.05) if kind == "hex"
         else systems.poly_system(400, seed=3, kind="pressure"))
    p = tmp_path / "a.mtx"
    mtx.write_matrix(p, s.csr, s.val, comment="test matrix\nsecond line")
    csr, val = mtx.read_matrix(p)
    assert np.array_equal(csr.row, s.csr.row) and np.array_equal(csr.col, s.csr.col)
    assert np.array_equal(csr.dia, s.csr.dia)
    assert np.array_equal(val, s.val)            # 17 significant digits: bit-exact


def test_scipy_reads_what_we_write(tmp_path):
    """The reference's analysis script reads the file with scipy.io.mmread."""
    s = systems.small_hex(6, seed=1, kind="pressure")
    p = tmp_path / "t-flows.mtx"
    mtx.write_matrix(p, s.csr, s.val)
    A = scipy.io.mmread(str(p)).tocsr()
    assert (A != _csr_scipy(s.csr, s.val)).nnz == 0


def test_reads_foreign_files_into_matrix_type_layout(tmp_path):
    """A symmetric file with entries in arbitrary order comes back with the
    diagonal first in each row and ascending columns after it."""
    s = systems.small_hex(5, seed=4, kind="pressure", ratio=1.1)
    A = _csr_scipy(s.csr, s.val).tocoo()
    lower = sps.tril(A).tocoo()
    perm = np.random.default_rng(0).permutation(lower.nnz)
    lower = sps.coo_matrix((lower.data[perm], (lower.row[perm], lower.col[perm])), shape=A.shape)
    p = tmp_path / "sym.mtx"
    scipy.io.mmwrite(str(p), lower, symmetry="symmetric", precision=17)
    csr, val = mtx.read_matrix(p)
    assert np.array_equal(csr.row, s.csr.row) and np.array_equal(csr.col, s.csr.col)
    assert np.array_equal(val, s.val)
    for i in range(csr.n):
        seg = csr.col[csr.row[i] - 1:csr.row[i + 1] - 1]
        assert seg[0] == i + 1 and np.all(np.diff(seg[1:]) > 0)
    # and the oracle solves it like the original
    b = s.b
    v1, x1, b1 = val.copy(), np.zeros(s.n), b.copy()
    r1 = O.solve_native("cg", "jacobi", csr.row, csr.col, csr.dia, v1, x1, b1, 500, 1e-10,
                        norm=1.0)
    v2, x2, b2 = s.val.copy(), np.zeros(s.n), b.copy()
    r2 = O.solve_native("cg", "jacobi", s.csr.row, s.csr.col, s.csr.dia, v2, x2, b2, 500,
                        1e-10, norm=1.0)
    assert r1 == r2 and np.array_equal(x1, x2)


def test_missing_diagonal_and_duplicates(tmp_path):
    text = """%%MatrixMarket matrix coordinate real general
3 3 6
1 1 4.0
1 2 -1.0
2 1 -1.0
2 3 -1.0
1 2 -0.5
3 2 2.0
"""
    p = tmp_path / "d.mtx"
    p.write_text(text)
    csr, val = mtx.read_matrix(p)
    dense = _csr_scipy(csr, val).toarray()
    want = np.array([[4.0, -1.5, 0.0], [-1.0, 0.0, -1.0], [0.0, 2.0, 0.0]])
    assert np.array_equal(dense, want)
    assert all(csr.col[csr.dia[i] - 1] == i + 1 for i in range(3))


def test_vector_round_trip(tmp_path):
    v = np.random.default_rng(1).standard_normal(17)
    p = tmp_path / "v.mtx"
    mtx.write_vector(p, v)
    assert np.array_equal(mtx.read_vector(p), v)
