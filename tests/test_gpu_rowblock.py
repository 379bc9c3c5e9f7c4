"""The row-block solve on the GPU: the library's kernels (tf_spmv and
tf_residual over a block's own rows, the tf_vec_* updates and sums) with the
ranks driven in lockstep in one process (run_local), on one device -- no
kernel waits on another, the driver sequences the ranks' collectives.
Against the oracle's single-process solve."""
import numpy as np
import pytest

from oracle import oracle as O
from tflows_b200 import rowblock, systems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mesh,nparts,norm", [("hex", 1, 1.0), ("hex", 2, 1.0),
                                              ("hex", 3, None), ("poly", 2, 1.0)])
def test_row_blocks_on_the_device(gpu_ctx, mesh, nparts, norm):
    if mesh == "hex":
        s = systems.small_hex(20, seed=6, kind="pressure", ratio=1.03, tol=1e-10, miter=2000)
    else:
        s = systems.poly_system(8000, seed=7, kind="pressure", tol=1e-10, miter=2000, norm=1.0)
    x, it, res = rowblock.solve_local(
        s.csr, s.val, s.b, s.x0, nparts, s.miter, s.tol, norm,
        make_kernels=lambda b: rowblock.DeviceKernels(b, gpu_ctx))
    v, ox, bb = s.val.copy(), s.x0.copy(), s.b.copy()
    r = O.solve_native("cg", "jacobi", s.csr.row, s.csr.col, s.csr.dia, v, ox, bb, s.miter,
                       s.tol, norm=norm, threads=8)
    assert abs(it - r["niter"]) <= max(1, 0.02 * r["niter"])
    assert np.linalg.norm(x - ox) <= 1e-8 * np.linalg.norm(ox)
    assert res < s.tol
