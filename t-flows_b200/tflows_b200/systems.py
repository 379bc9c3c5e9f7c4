"""Matrix_Type construction and synthetic system assembly (numpy).

* :func:`create_matrix` restates Matrix_Mod/Create_Matrix.f90:45-155: CSR
  with the diagonal first in each row and the other columns ascending, ``dia``,
  ``pos(2, n_faces)`` and the bare face coefficient ``fc = |S|^2 / (S.d)``.
* :func:`assemble_pressure` restates the pressure-correction matrix of
  Process_Mod/Rhie_And_Chow.f90:199-204 (interior faces) and
  Compute_Pressure.f90:154-158 (pressure/ambient boundary faces).
* :func:`assemble_momentum` restates Compute_Momentum.f90:270-297 with the
  upwind-blended convection (``blend_matrix``), wall faces adding to the
  diagonal, and Numerics_Mod/Inertial_Term.f90 (LINEAR) adding rho V / dt.

Every diagonal is accumulated in the reference's face-loop order
(``np.bincount`` adds its weights sequentially in input order), so the
values equal those of the loop restatements in the oracle bit for bit.
All indices returned are 1-based, as T-Flows stores them.
"""
from dataclasses import dataclass, field

import numpy as np

from .grids import Grid, hex_grid, poly_dual_grid

MICRO = 1.0e-6   # Sources/Shared/Const_Mod.f90


@dataclass
class Csr:
    n: int
    row: np.ndarray      # int32 (n+1), 1-based
    col: np.ndarray      # int32 (nnz), 1-based
    dia: np.ndarray      # int32 (n), 1-based
    pos: np.ndarray      # int32 (n_faces, 2), 1-based, 0 for boundary faces

    @property
    def nnz(self):
        return int(self.row[-1] - 1)


@dataclass
class System:
    """One linear system as Solve_Native receives it."""
    name: str
    solver: str              # 'cg' or 'bicg'
    prec: str
    csr: Csr
    val: np.ndarray
    b: np.ndarray
    x0: np.ndarray
    tol: float
    miter: int
    norm: float = None       # None: the optional argument is absent
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.csr.n

    @property
    def nnz(self):
        return self.csr.nnz


def create_matrix(grid: Grid) -> Csr:
    n = grid.n_cells
    fc_ = grid.faces_c
    interior = fc_[:, 1] > 0
    c1 = fc_[interior, 0].astype(np.int64)
    c2 = fc_[interior, 1].astype(np.int64)
    m = len(c1)
    diag = np.arange(1, n + 1, dtype=np.int64)
    rows = np.concatenate([diag, c1, c2])
    cols = np.concatenate([diag, c2, c1])
    keycol = np.where(rows == cols, 0, cols)            # diagonal first
    key = rows * (n + 1) + keycol
    order = np.argsort(key, kind="stable")
    counts = np.bincount(rows, minlength=n + 1)[1:]
    row = np.empty(n + 1, dtype=np.int64)
    row[0] = 1
    np.cumsum(counts, out=row[1:])
    row[1:] += 1
    col = cols[order].astype(np.int32)
    dia = row[:-1].astype(np.int32)
    inv = np.empty(len(order), dtype=np.int64)
    inv[order] = np.arange(len(order))
    pos = np.zeros((len(fc_), 2), dtype=np.int32)
    idx = np.nonzero(interior)[0]
    pos[idx, 0] = inv[n + np.arange(m)] + 1
    pos[idx, 1] = inv[n + m + np.arange(m)] + 1
    return Csr(n=n, row=row.astype(np.int32), col=col, dia=dia, pos=pos)


def face_coef(grid: Grid) -> np.ndarray:
    """fc = (S.S)/(d.S), Create_Matrix.f90:148-155."""
    return ((grid.sx * grid.sx + grid.sy * grid.sy + grid.sz * grid.sz)
            / (grid.dx * grid.sx + grid.dy * grid.sy + grid.dz * grid.sz))


def _accumulate_diag(n, idx0, vals):
    """Sequential += into a zero diagonal, in input order (like the face loops)."""
    return np.bincount(idx0, weights=vals, minlength=n)


def assemble_pressure(grid: Grid, csr: Csr, fc, v_m=None, bnd_open=None):
    """Pressure-correction matrix values (val has nnz entries)."""
    n = grid.n_cells
    if v_m is None:
        v_m = np.ones(n)
    val = np.zeros(csr.nnz)
    interior = grid.interior
    s_int = np.nonzero(interior)[0]
    c1 = grid.faces_c[s_int, 0] - 1
    c2 = grid.faces_c[s_int, 1] - 1
    fs = grid.fw[s_int]
    a12 = fc[s_int] * (fs * v_m[c1] + (1.0 - fs) * v_m[c2])
    val[csr.pos[s_int, 0] - 1] = -a12
    val[csr.pos[s_int, 1] - 1] = -a12
    didx = np.stack([c1, c2], axis=1).ravel()
    dval = np.stack([a12, a12], axis=1).ravel()
    d = _accumulate_diag(n, didx, dval)
    if bnd_open is not None and np.any(bnd_open):
        s_b = np.nonzero((~interior) & bnd_open)[0]
        cb = grid.faces_c[s_b, 0] - 1
        # second face loop (Compute_Pressure.f90:140-160) adds after the first
        for c, a in zip(cb, fc[s_b] * v_m[cb]):
            d[c] = d[c] + a
    val[csr.dia - 1] = d
    return val


def assemble_momentum(grid: Grid, csr: Csr, fc, flux, vis, rho, dt, bnd_wall=None):
    """Momentum matrix values with upwind blending and the inertial term."""
    n = grid.n_cells
    nf = grid.n_faces
    val = np.zeros(csr.nnz)
    m0 = vis * fc
    m12 = m0 - np.minimum(flux, 0.0) * rho
    m21 = m0 + np.maximum(flux, 0.0) * rho
    interior = grid.interior
    s_int = np.nonzero(interior)[0]
    val[csr.pos[s_int, 0] - 1] = -m12[s_int]
    val[csr.pos[s_int, 1] - 1] = -m21[s_int]
    if bnd_wall is None:
        bnd_wall = ~interior
    # diagonal contributions in face order: interior (c1 += m12, c2 += m21),
    # wall (c1 += m12)
    c1 = grid.faces_c[:, 0].astype(np.int64) - 1
    c2 = grid.faces_c[:, 1].astype(np.int64) - 1
    wall = (~interior) & bnd_wall
    ent_idx = np.stack([c1, np.where(interior, c2, -1)], axis=1)
    ent_val = np.stack([m12, m21], axis=1)
    keep = np.stack([interior | wall, interior], axis=1)
    d = _accumulate_diag(n, ent_idx[keep], ent_val[keep])
    a0 = rho * grid.vol / dt
    d = d + a0
    val[csr.dia - 1] = d
    return val


def set_singular(csr: Csr, val):
    """Set_Singular.f90:29-31: every diagonal times (1 + MICRO)."""
    val[csr.dia - 1] = val[csr.dia - 1] * (1.0 + MICRO)


def uniform_rhs(n, seed, zero_mean):
    b = np.random.default_rng(seed).uniform(-1.0, 1.0, n)
    if zero_mean:
        b = b - b.mean()
    return b


def pressure_system(grid, seed, tol, miter, singular="pin", norm=1.0, name=None,
                    prec="jacobi", solver="cg", csr=None):
    """Pressure Poisson system with all walls.  singular='pin' opens the first
    boundary face of cell 1 as a pressure boundary (Compute_Pressure.f90:154-158);
    'set_singular' scales every diagonal by 1+MICRO (Set_Singular.f90)."""
    csr = create_matrix(grid) if csr is None else csr
    fc = face_coef(grid)
    bnd_open = None
    if singular == "pin":
        bnd_open = np.zeros(grid.n_faces, dtype=bool)
        cand = np.nonzero((~grid.interior) & (grid.faces_c[:, 0] == 1))[0]
        if len(cand):
            bnd_open[cand[0]] = True
        else:   # no boundary face (poly grids): pin with the mean interior coefficient
            bnd_open = None
    val = assemble_pressure(grid, csr, fc, bnd_open=bnd_open)
    if singular == "pin" and bnd_open is None:
        val[csr.dia[0] - 1] += float(np.mean(fc[grid.interior]))
    elif singular == "set_singular":
        set_singular(csr, val)
    b = uniform_rhs(grid.n_cells, seed, zero_mean=True)
    return System(name=name or f"pressure-{grid.kind}-{grid.n_cells}", solver=solver,
                  prec=prec, csr=csr, val=val, b=b, x0=np.zeros(grid.n_cells), tol=tol,
                  miter=miter, norm=norm,
                  meta=dict(grid.meta, singular=singular, seed=seed, grid=grid.kind))


def momentum_system(grid, seed, tol, miter, peclet=10.0, cfl=0.5, u0=1.0, norm=None,
                    name=None, prec="jacobi", solver="bicg", csr=None):
    """Momentum (convection-diffusion) system: face velocity U[-1,1]*u0,
    viscosity from the cell Peclet number, dt from the CFL number."""
    rng = np.random.default_rng(seed + 1000003)
    csr = create_matrix(grid) if csr is None else csr
    fc = face_coef(grid)
    area = np.sqrt(grid.sx ** 2 + grid.sy ** 2 + grid.sz ** 2)
    u = rng.uniform(-1.0, 1.0, grid.n_faces) * u0
    flux = np.where(grid.interior, u * area, 0.0)
    rho = 1.0
    vis = u0 * grid.h_mean / peclet
    dt = cfl * grid.h_min / u0
    val = assemble_momentum(grid, csr, fc, flux, vis, rho, dt)
    b = uniform_rhs(grid.n_cells, seed, zero_mean=False)
    return System(name=name or f"momentum-{grid.kind}-{grid.n_cells}", solver=solver,
                  prec=prec, csr=csr, val=val, b=b, x0=np.zeros(grid.n_cells), tol=tol,
                  miter=miter, norm=u0 if norm is None else norm,
                  meta=dict(grid.meta, peclet=peclet, cfl=cfl, vis=vis, dt=dt, seed=seed,
                            grid=grid.kind))


# ---------------------------------------------------------------------------
# The named workloads
# ---------------------------------------------------------------------------
def ldc_pressure_30(seed=1, singular="pin"):
    """Lid-driven-cavity pressure matrix: uniform 30^3 hex, walls, Cg +
    Jacobi, tol 1e-8, miter 500, norm = 1 (p_nor's default)."""
    g = hex_grid(30, 30, 30)
    return pressure_system(g, seed, tol=1e-8, miter=500, singular=singular, norm=1.0,
                           name="ldc-pressure-30^3")


def stretched_pair(n=200, seed=2, tol=1e-10, miter=20000, ratio=1.02, peclet=10.0,
                   momentum_miter=None):
    """n^3 hex stretched by `ratio` toward both y walls: Cg Poisson + Bicg
    momentum sharing one Matrix_Type topology (Create_Native.f90:19-20)."""
    g = hex_grid(n, n, n, stretch_y=ratio)
    csr = create_matrix(g)
    p = pressure_system(g, seed, tol=tol, miter=miter, singular="pin", norm=1.0,
                        name=f"stretched-pressure-{n}^3", csr=csr)
    m = momentum_system(g, seed, tol=tol, miter=momentum_miter or miter, peclet=peclet,
                        cfl=0.5, name=f"stretched-momentum-{n}^3", csr=csr)
    return p, m


def small_hex(n=8, seed=0, kind="pressure", **kw):
    g = hex_grid(n, n, n, stretch_y=kw.pop("ratio", 1.0))
    if kind == "pressure":
        return pressure_system(g, seed, tol=kw.pop("tol", 1e-8), miter=kw.pop("miter", 500),
                               **kw)
    return momentum_system(g, seed, tol=kw.pop("tol", 1e-8), miter=kw.pop("miter", 500), **kw)


def poly_system(n_points, seed, kind="pressure", tol=1e-10, miter=20000, **kw):
    g = poly_dual_grid(n_points, seed)
    if kind == "pressure":
        return pressure_system(g, seed, tol=tol, miter=miter, singular="pin", **kw)
    return momentum_system(g, seed, tol=tol, miter=miter, **kw)


def renumber_rcm(s: System) -> System:
    """The same system with cells renumbered by reverse Cuthill-McKee (a
    symmetric permutation P A P^T): row i' = perm[i] keeps its entries in
    their original storage order with relabelled columns, so every row sum
    is the original row's sum.  `pos` is not carried over."""
    import copy
    import scipy.sparse as sps
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    c = s.csr
    n = c.n
    A = sps.csr_matrix((np.ones(c.nnz), c.col - 1, c.row - 1), shape=(n, n))
    order = reverse_cuthill_mckee(A, symmetric_mode=True)     # new -> old
    inv = np.empty(n, np.int64)
    inv[order] = np.arange(n)                                  # old -> new
    lens = np.diff(c.row)[order]
    row = np.concatenate([[1], 1 + np.cumsum(lens)]).astype(np.int32)
    src = np.concatenate([np.arange(c.row[o] - 1, c.row[o + 1] - 1) for o in order]) \
        if n < 50000 else _gather_rows(c.row, order)
    col = (inv[c.col[src] - 1] + 1).astype(np.int32)
    dia_old = c.dia[order] - 1                                  # entry index in old arrays
    # position of the diagonal within each new row = its offset in the old row
    dia = (row[:-1] + (dia_old - (c.row[order] - 1))).astype(np.int32)
    t = copy.copy(s)
    t.csr = Csr(n=n, row=row, col=col, dia=dia, pos=np.zeros((0, 2), np.int32))
    t.val = s.val[src]
    t.b = s.b[order]
    t.x0 = s.x0[order]
    t.meta = dict(s.meta, renumbered="rcm")
    return t


def _gather_rows(row, order):
    """Entry indices (0-based) of the rows `order`, row after row."""
    starts = row[order].astype(np.int64) - 1
    lens = (row[order + 1] - row[order]).astype(np.int64)
    out_start = np.concatenate([[0], np.cumsum(lens)[:-1]])
    idx = np.arange(lens.sum(), dtype=np.int64)
    return starts.repeat(lens) + (idx - out_start.repeat(lens))
