"""Device-side assembly through pos: the pressure and momentum matrices are
bit-identical to the reference's face loops (the oracle's restatement), and
a solve on the device-assembled values equals one on host-assembled ones."""
import numpy as np
import pytest

from oracle import oracle as O
from tflows_b200 import grids, native, systems

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _grid(kind):
    return (grids.hex_grid(11, 9, 13, stretch_y=1.05) if kind == "hex"
            else grids.poly_lattice_grid(3000, 4))


def _bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.int64)


@pytest.mark.parametrize("kind", ["hex", "poly"])
@pytest.mark.parametrize("with_vm", [False, True])
def test_device_pressure_assembly_is_bitwise(gpu_ctx, kind, with_vm):
    torch = _torch()
    g = _grid(kind)
    c = systems.create_matrix(g)
    fc = systems.face_coef(g)
    rng = np.random.default_rng(5)
    bo = np.zeros(g.n_faces, bool)
    bnd = np.nonzero(~g.interior)[0]      # the polyhedral generator has none
    if len(bnd):
        bo[bnd[rng.choice(len(bnd), min(7, len(bnd)), replace=False)]] = True
    vm = rng.uniform(0.5, 2.0, g.n_cells) if with_vm else None
    want = O.assemble_pressure(g, c.pos, c.dia, c.nnz, fc, bo, v_m=vm)
    m = native.Matrix(gpu_ctx, c.row, c.col, c.dia)
    try:
        native.faces_register(gpu_ctx, m, g.faces_c, c.pos)
        d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda()
             for k, v in (("fc", fc), ("fw", g.fw), ("bo", bo.astype(np.int32)))}
        dvm = torch.from_numpy(vm).cuda() if with_vm else None
        dval = torch.full((c.nnz,), 7.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        native.assemble_pressure(gpu_ctx, m, d["fc"].data_ptr(), d["fw"].data_ptr(),
                                 dvm.data_ptr() if with_vm else 0, d["bo"].data_ptr(),
                                 dval.data_ptr())
        gpu_ctx.sync()
        assert np.array_equal(_bits(dval.cpu().numpy()), _bits(want))
    finally:
        m.close()


@pytest.mark.parametrize("kind", ["hex", "poly"])
def test_device_momentum_assembly_is_bitwise_and_solves_alike(gpu_ctx, kind):
    torch = _torch()
    g = _grid(kind)
    c = systems.create_matrix(g)
    fc = systems.face_coef(g)
    rng = np.random.default_rng(6)
    area = np.sqrt(g.sx ** 2 + g.sy ** 2 + g.sz ** 2)
    flux = np.where(g.interior, rng.uniform(-1, 1, g.n_faces) * area, 0.0)
    vis, rho, dt = 0.01 * g.h_mean, 1.0, 0.1 * g.h_min
    wall = ~g.interior
    want = O.assemble_momentum(g, c.pos, c.dia, c.nnz, fc, flux, vis, rho, dt, wall)
    m = native.Matrix(gpu_ctx, c.row, c.col, c.dia)
    try:
        native.faces_register(gpu_ctx, m, g.faces_c, c.pos)
        d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda()
             for k, v in (("fc", fc), ("flux", flux), ("wall", wall.astype(np.int32)),
                          ("vol", g.vol))}
        dval = torch.zeros(c.nnz, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        native.assemble_momentum(gpu_ctx, m, d["fc"].data_ptr(), d["flux"].data_ptr(),
                                 d["wall"].data_ptr(), vis, rho, d["vol"].data_ptr(), dt,
                                 dval.data_ptr())
        gpu_ctx.sync()
        assert np.array_equal(_bits(dval.cpu().numpy()), _bits(want))
        # the device-assembled matrix solves exactly like the host one
        b = systems.uniform_rhs(g.n_cells, 3, zero_mean=False)
        db = torch.from_numpy(b).cuda()
        dx = torch.zeros(g.n_cells, dtype=torch.float64, device="cuda")
        it1, r1 = native.solve_device(gpu_ctx, m, "bicg", "jacobi", dval.data_ptr(),
                                      dx.data_ptr(), db.data_ptr(), 2000, 1e-10, 1.0)
        x1 = dx.cpu().numpy()
        v2, x2, b2 = want.copy(), np.zeros(g.n_cells), b.copy()
        it2, r2 = native.solve(gpu_ctx, m, "bicg", "jacobi", v2, x2, b2, 2000, 1e-10, 1.0)
        assert (it1, r1) == (it2, r2) and np.array_equal(x1, x2)
    finally:
        m.close()
