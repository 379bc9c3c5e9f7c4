"""tf_spmv_noalloc: the SpMV + p.q entry point that allocates nothing.

It exists for callers whose device memory is owned elsewhere (an OpenACC data
region, a pooled allocator, a fixed device-memory budget) or who cannot
afford cudaFree's device synchronisation, so they hand every buffer in and
the kernel's scratch comes from a fixed array inside the library.  These
tests call it through the C ABI and check it against the regular entry point
(tf_spmv on a registered matrix) with the tolerances the other SpMV tests
use: q bit for bit, p.q to 1e-13 relative -- on two calls in a row, so the
second call shows the shared scratch is cleared between calls.  The file is
named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from tflows_b200 import native, systems

pytestmark = pytest.mark.gpu

MAX_ROWS = 16777216          # TF_SPMV_NOALLOC_MAX_ROWS in include/tf_krylov.h


def _lib():
    L = native.load()
    vp = ctypes.c_void_p
    L.tf_spmv_noalloc.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, vp, vp]
    L.tf_spmv_noalloc.restype = ctypes.c_int
    return L


def _cuda(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _reference_spmv(torch, ctx, s, p):
    """q and p.q from the regular entry point (registered matrix)."""
    m = native.Matrix(ctx, s.csr.row, s.csr.col, s.csr.dia)
    try:
        dval, dp = _cuda(torch, s.val), _cuda(torch, p)
        dq = torch.zeros(s.n, dtype=torch.float64, device="cuda")
        dpq = torch.zeros(1, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        native.spmv(ctx, m, dval.data_ptr(), dp.data_ptr(), dq.data_ptr(), dpq.data_ptr())
        ctx.sync()
        return dq.cpu().numpy(), dpq.item()
    finally:
        m.close()


def _noalloc_spmv(torch, L, s, p):
    drow = _cuda(torch, s.csr.row.astype(np.int32))
    dcol = _cuda(torch, s.csr.col.astype(np.int32))
    dval, dp = _cuda(torch, s.val), _cuda(torch, p)
    dq = torch.full((s.n,), np.nan, dtype=torch.float64, device="cuda")
    dpq = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = L.tf_spmv_noalloc(s.n, drow.data_ptr(), dcol.data_ptr(), dval.data_ptr(),
                           dp.data_ptr(), dq.data_ptr(), dpq.data_ptr(), None)
    assert st == 0, L.tf_last_error_message()
    torch.cuda.synchronize()
    return dq.cpu().numpy(), dpq.item()


def _one_by_one():
    """The 1 x 1 system: one row, one tile that is first and last at once."""
    csr = systems.Csr(n=1, row=np.array([1, 2], np.int32), col=np.array([1], np.int32),
                      dia=np.array([1], np.int32), pos=np.zeros((0, 2), np.int32))
    return systems.System(name="1x1", solver="cg", prec="jacobi", csr=csr,
                          val=np.array([2.5]), b=np.array([1.0]), x0=np.zeros(1),
                          tol=1e-8, miter=10, norm=1.0, meta={})


def test_noalloc_matches_regular_spmv_twice(gpu_ctx):
    import torch
    assert torch.cuda.is_available()
    L = _lib()
    cases = [_one_by_one(),                                                 # n = 1
             systems.small_hex(5, seed=2, kind="pressure"),                 # n = 125 < 256
             systems.small_hex(7, seed=2, kind="momentum", peclet=1.0),     # 343: a partial tile
             systems.small_hex(40, seed=3, kind="momentum", ratio=1.02),    # 250 whole tiles
             systems.poly_system(5000, seed=4, kind="pressure")]
    rng = np.random.default_rng(11)
    for s in cases:
        p = rng.standard_normal(s.n)
        q_ref, pq_ref = _reference_spmv(torch, gpu_ctx, s, p)
        # The same input twice in a row: the second call starts from the
        # scratch the first one left, and must give the same bits.
        q1, pq1 = _noalloc_spmv(torch, L, s, p)
        q2, pq2 = _noalloc_spmv(torch, L, s, p)
        assert np.array_equal(q1, q_ref) and np.array_equal(q2, q_ref), s.name
        assert pq1 == pytest.approx(pq_ref, rel=1e-13), s.name
        assert pq2 == pq1, s.name


def test_noalloc_rejects_oversize():
    import torch
    L = _lib()
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    ptr = dummy.data_ptr()
    st = L.tf_spmv_noalloc(MAX_ROWS + 1, ptr, ptr, ptr, ptr, ptr, ptr, None)
    assert st == 3          # TF_ERR_ARG, before anything is launched
    assert b"scratch limit" in L.tf_last_error_message()
