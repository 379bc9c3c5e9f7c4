"""The MatrixMarket command line solves a .mtx system on the GPU."""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O
from tflows_b200 import mtx, systems

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_mtx_solve_command(tmp_path):
    s = systems.small_hex(9, seed=11, kind="pressure", ratio=1.04)
    mtx.write_matrix(tmp_path / "A.mtx", s.csr, s.val)
    mtx.write_vector(tmp_path / "b.mtx", s.b)
    env = dict(os.environ, PYTHONPATH=os.path.join(ROOT, "t-flows_b200"))
    r = subprocess.run([sys.executable, "-m", "tflows_b200.mtx", "solve", str(tmp_path / "A.mtx"),
                        "--rhs", str(tmp_path / "b.mtx"), "--tol", "1e-10", "--miter", "2000",
                        "--norm", "1.0", "--out", str(tmp_path / "x.mtx")],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    x = mtx.read_vector(tmp_path / "x.mtx")
    v, xo, b = s.val.copy(), np.zeros(s.n), s.b.copy()
    o = O.solve_native("cg", "jacobi", s.csr.row, s.csr.col, s.csr.dia, v, xo, b, 2000, 1e-10,
                       norm=1.0)
    assert f"niter {o['niter']}" in r.stdout
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
