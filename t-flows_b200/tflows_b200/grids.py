"""Seeded synthetic grids in T-Flows' face/cell conventions.

The reference ships no benchmark meshes for its solver path, so the systems
the solvers are measured on are generated here with the shapes the workloads
name.  Conventions follow T-Flows' Grid_Type:

* cells are numbered 1..n_cells; ``faces_c[s] = (c1, c2)`` with c1 < c2 for
  interior faces (Sort_Cells_By_Coordinates.f90:126 swaps them so) and c2 < 0
  (a boundary-cell index) for boundary faces;
* ``(sx, sy, sz)`` is the face area vector pointing from c1 to c2,
  ``(dx, dy, dz)`` the vector from c1's centre to c2's centre (or to the face
  centre on a boundary), ``fw`` the interpolation weight of c1;
* hexahedral cells are ordered by (x, y, z) as Sort_Cells_By_Coordinates.f90:103
  orders them, so z varies fastest.

The polyhedral grid is the Voronoi dual of a seeded random Delaunay
tetrahedralisation (the dual T-Flows' Convert builds, Convert_Mod/Create_Dual.f90):
one cell per point, one face per Delaunay edge, face area from the dual
polygon, centre distance from the points.
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Grid:
    n_cells: int
    faces_c: np.ndarray          # (n_faces, 2) int32, 1-based, c2 < 0 on boundaries
    sx: np.ndarray
    sy: np.ndarray
    sz: np.ndarray
    dx: np.ndarray
    dy: np.ndarray
    dz: np.ndarray
    fw: np.ndarray               # weight of c1 in face interpolation
    vol: np.ndarray              # (n_cells,)
    h_min: float = 0.0           # smallest cell size (for CFL)
    h_mean: float = 0.0
    kind: str = "hex"
    meta: dict = field(default_factory=dict)

    @property
    def n_faces(self):
        return len(self.faces_c)

    @property
    def interior(self):
        return self.faces_c[:, 1] > 0


def geometric_nodes(n, ratio):
    """n cells on [0, 1], widths growing by `ratio` from both ends to the middle."""
    if ratio == 1.0 or n < 2:
        return np.linspace(0.0, 1.0, n + 1)
    half = n // 2
    w = ratio ** np.arange(half)
    widths = np.concatenate([w, ([w[-1] * ratio] if n % 2 else []), w[::-1]])
    widths = widths / widths.sum()
    nodes = np.concatenate([[0.0], np.cumsum(widths)])
    nodes[-1] = 1.0
    return nodes


def hex_grid(nx, ny, nz, stretch_y=1.0):
    """Block hex grid on the unit cube; y nodes stretched toward both y walls."""
    xn = np.linspace(0.0, 1.0, nx + 1)
    yn = geometric_nodes(ny, stretch_y)
    zn = np.linspace(0.0, 1.0, nz + 1)
    hx, hy, hz = np.diff(xn), np.diff(yn), np.diff(zn)
    xc, yc, zc = 0.5 * (xn[:-1] + xn[1:]), 0.5 * (yn[:-1] + yn[1:]), 0.5 * (zn[:-1] + zn[1:])
    n = nx * ny * nz

    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    cid = (I * ny + J) * nz + K          # 0-based, z fastest

    parts = []   # (c1, c2, sx, sy, sz, dx, dy, dz, fw) per direction

    def interior(axis):
        if axis == 0:
            m = I < nx - 1
            nb = cid[m] + ny * nz
            area = hy[J[m]] * hz[K[m]]
            d = xc[I[m] + 1] - xc[I[m]]
            fw = (xc[I[m] + 1] - xn[I[m] + 1]) / d
        elif axis == 1:
            m = J < ny - 1
            nb = cid[m] + nz
            area = hx[I[m]] * hz[K[m]]
            d = yc[J[m] + 1] - yc[J[m]]
            fw = (yc[J[m] + 1] - yn[J[m] + 1]) / d
        else:
            m = K < nz - 1
            nb = cid[m] + 1
            area = hx[I[m]] * hy[J[m]]
            d = zc[K[m] + 1] - zc[K[m]]
            fw = (zc[K[m] + 1] - zn[K[m] + 1]) / d
        z = np.zeros_like(area)
        s = [z, z, z]
        dd = [z, z, z]
        s[axis] = area
        dd[axis] = d
        return cid[m], nb, s, dd, fw, axis

    keys, cols = [], []
    for ax in (2, 1, 0):                 # per cell: +z, +y, +x faces
        c1, c2, s, dd, fw, a = interior(ax)
        keys.append(c1.astype(np.int64) * 3 + (2 - a))
        cols.append((c1, c2, s[0], s[1], s[2], dd[0], dd[1], dd[2], fw))
    key = np.concatenate(keys)
    order = np.argsort(key, kind="stable")
    cat = [np.concatenate([c[i] for c in cols])[order] for i in range(9)]
    c1, c2, sx, sy, sz, dx, dy, dz, fw = cat

    # Boundary faces: six walls, ordered by cell then wall.
    bparts = []
    for ax, side in ((0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (2, 1)):
        idx = (I, J, K)[ax]
        lim = (nx, ny, nz)[ax] - 1
        m = idx == (0 if side == 0 else lim)
        cc = cid[m]
        if ax == 0:
            area = hy[J[m]] * hz[K[m]]
            d = (xn[0] - xc[0]) if side == 0 else (xn[-1] - xc[-1])
        elif ax == 1:
            area = hx[I[m]] * hz[K[m]]
            d = np.where(side == 0, yn[0] - yc[J[m]], yn[-1] - yc[J[m]])
        else:
            area = hx[I[m]] * hy[J[m]]
            d = (zn[0] - zc[0]) if side == 0 else (zn[-1] - zc[-1])
        sgn = -1.0 if side == 0 else 1.0
        z = np.zeros_like(area)
        s = [z, z, z]
        dd = [z, z, z]
        s[ax] = sgn * area
        dd[ax] = np.broadcast_to(np.asarray(d, dtype=np.float64), area.shape).copy()
        bparts.append((cc, s, dd, ax * 2 + side))
    bkey = np.concatenate([p[0].astype(np.int64) * 6 + p[3] for p in bparts])
    border = np.argsort(bkey, kind="stable")
    bc1 = np.concatenate([p[0] for p in bparts])[border]
    bs = [np.concatenate([p[1][i] for p in bparts])[border] for i in range(3)]
    bd = [np.concatenate([p[2][i] for p in bparts])[border] for i in range(3)]
    nbf = len(bc1)
    bc2 = -(np.arange(nbf) + 1)

    faces_c = np.empty((len(c1) + nbf, 2), dtype=np.int32)
    faces_c[: len(c1), 0] = c1 + 1
    faces_c[: len(c1), 1] = c2 + 1
    faces_c[len(c1):, 0] = bc1 + 1
    faces_c[len(c1):, 1] = bc2
    cat2 = lambda a, b: np.concatenate([a, b])
    vol = (hx[I] * hy[J] * hz[K])
    h = np.cbrt(vol)
    return Grid(n_cells=n, faces_c=faces_c,
                sx=cat2(sx, bs[0]), sy=cat2(sy, bs[1]), sz=cat2(sz, bs[2]),
                dx=cat2(dx, bd[0]), dy=cat2(dy, bd[1]), dz=cat2(dz, bd[2]),
                fw=cat2(fw, np.ones(nbf)), vol=vol,
                h_min=float(min(hx.min(), hy.min(), hz.min())), h_mean=float(h.mean()),
                kind="hex", meta=dict(nx=nx, ny=ny, nz=nz, stretch_y=stretch_y))


def poly_lattice_grid(n_target, seed, jitter=0.25):
    """Median dual of a jittered Freudenthal (Kuhn) tetrahedralisation.

    Lattice vertices (nx*ny*nz ~ n_target, spacing h) are moved by
    U[-jitter, jitter]*h in each direction; every lattice cube is split into
    the 6 tetrahedra along its main diagonal.  Each vertex becomes one
    polyhedral cell whose faces are the median-dual faces of its 14 edges
    (directions (1,0,0), (0,1,0), (0,0,1), (1,1,0), (1,0,1), (0,1,1),
    (1,1,1) and their opposites): interior cells have 14 faces, the face
    normal is not parallel to the centre-to-centre vector (non-orthogonal
    mesh), and the whole construction is O(n) and vectorised, unlike a
    Delaunay dual.  Face area vector of edge (a, b) = sum over its
    tetrahedra of 1/2 (c_T - m_ab) x (c_f1 - c_f2) with m the edge midpoint,
    c_T the tet centroid and c_f the centroids of the tet's two faces that
    contain the edge, oriented along b - a.  Cell volume = 1/4 of every
    incident tet.  No boundary faces (zero-gradient walls).
    """
    m = max(2, int(round(n_target ** (1.0 / 3.0))))
    nx = ny = m
    nz = max(2, int(round(n_target / (m * m))))
    h = 1.0 / max(nx - 1, ny - 1, nz - 1)
    rng = np.random.default_rng(seed)
    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    pts = np.stack([I.ravel(), J.ravel(), K.ravel()], axis=1).astype(np.float64) * h
    pts += rng.uniform(-jitter, jitter, pts.shape) * h
    vid = lambda i, j, k: (i * ny + j) * nz + k  # noqa: E731
    # the 6 tetrahedra of every cube: paths (0,0,0) -> (1,1,1) along axes
    ci, cj, ck = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), np.arange(nz - 1),
                             indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    tets = []
    for pm in perms:
        o = np.zeros((len(ci), 3), dtype=np.int64)
        v = [vid(ci, cj, ck)]
        for ax in pm:
            o[:, ax] += 1
            v.append(vid(ci + o[:, 0], cj + o[:, 1], ck + o[:, 2]))
        tets.append(np.stack(v, axis=1))
    tets = np.concatenate(tets)
    P = pts[tets]
    cT = P.mean(axis=1)
    n = nx * ny * nz
    vol_t = np.abs(np.einsum("ij,ij->i", P[:, 1] - P[:, 0],
                             np.cross(P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]))) / 6.0
    vol = np.bincount(tets.ravel(), weights=np.repeat(vol_t / 4.0, 4), minlength=n)
    # Every tet edge joins a vertex to one of its 7 forward lattice neighbours
    # (the path is monotone), so edge id = vertex * 8 + direction code.
    stride = np.array([ny * nz, nz, 1])
    code_off = np.array([[i >> 2 & 1, i >> 1 & 1, i & 1] for i in range(8)])
    acc = np.zeros((8 * n, 3))
    for (u, w) in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)):
        o1, o2 = [k for k in range(4) if k not in (u, w)]
        mab = 0.5 * (P[:, u] + P[:, w])
        cf1 = (P[:, u] + P[:, w] + P[:, o1]) / 3.0
        cf2 = (P[:, u] + P[:, w] + P[:, o2]) / 3.0
        sv = 0.5 * np.cross(cT - mab, cf1 - cf2)
        a, b = tets[:, u], tets[:, w]            # a precedes b on the path
        e = pts[b] - pts[a]
        sgn = np.sign(np.einsum("ij,ij->i", sv, e))
        sgn[sgn == 0] = 1.0
        sv = sv * sgn[:, None]
        d = b - a
        code = ((d // stride[0]) % 2) * 4 + ((d % stride[0]) // stride[1] % 2) * 2 + (d % nz)
        eid = a * 8 + code
        for c in range(3):
            acc[:, c] += np.bincount(eid, weights=sv[:, c], minlength=8 * n)
    present = np.nonzero(np.any(acc != 0.0, axis=1))[0]
    S = acc[present]
    c1 = present // 8
    off = code_off[present % 8]
    c2 = c1 + off @ stride
    # renumber cells by (x, y, z) like Sort_Cells_By_Coordinates.f90
    order = np.lexsort((pts[:, 2], pts[:, 1], pts[:, 0]))
    new = np.empty(n, dtype=np.int64)
    new[order] = np.arange(n)
    pts, vol = pts[order], vol[order]
    c1, c2 = new[c1], new[c2]
    flip = c1 > c2
    c1, c2 = np.where(flip, c2, c1), np.where(flip, c1, c2)
    S[flip] = -S[flip]
    dvec = pts[c2] - pts[c1]
    faces_c = np.stack([c1 + 1, c2 + 1], axis=1).astype(np.int32)
    deg = np.bincount(c1, minlength=n) + np.bincount(c2, minlength=n)
    dist = np.linalg.norm(dvec, axis=1)
    return Grid(n_cells=n, faces_c=faces_c, sx=S[:, 0].copy(), sy=S[:, 1].copy(),
                sz=S[:, 2].copy(), dx=dvec[:, 0].copy(), dy=dvec[:, 1].copy(),
                dz=dvec[:, 2].copy(), fw=np.full(len(c1), 0.5), vol=vol,
                h_min=float(dist.min()), h_mean=float(np.cbrt(vol).mean()), kind="poly-lattice",
                meta=dict(seed=seed, dims=(nx, ny, nz), jitter=jitter,
                          faces_per_cell_mean=float(deg.mean()),
                          faces_per_cell_max=int(deg.max())))


def poly_dual_grid(n_points, seed):
    """Voronoi dual of a seeded random Delaunay tetrahedralisation of [0,1]^3.

    One cell per point; one face per Delaunay edge with area = area of the
    dual polygon (sum over the edge's tetrahedra of the two triangles
    (edge midpoint, facet circumcentre, tet circumcentre), signed along the
    edge direction so obtuse configurations cancel correctly); d = edge
    vector.  Edges on the hull give open dual faces; their area is the same
    sum over the tetrahedra that exist (a truncated face).  Boundary faces
    are not created: the cube walls act as zero-gradient boundaries, which
    contribute nothing to the pressure matrix.  Cells are renumbered by
    (x, y, z) like Sort_Cells_By_Coordinates.f90.
    """
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    pts = rng.random((n_points, 3))
    order = np.lexsort((pts[:, 2], pts[:, 1], pts[:, 0]))
    pts = pts[order]
    tri = Delaunay(pts)
    tets = tri.simplices.astype(np.int64)
    P = pts[tets]                                   # (T, 4, 3)

    def circumcentre(A, B, C, D=None):
        # 3D circumcentre of a triangle (D is None) or tetrahedron.
        if D is None:
            a, b = B - A, C - A
            axb = np.cross(a, b)
            num = (np.sum(a * a, -1)[:, None] * np.cross(b, axb)
                   + np.sum(b * b, -1)[:, None] * np.cross(axb, a))
            den = 2.0 * np.sum(axb * axb, -1)[:, None]
            return A + num / den
        a, b, c = B - A, C - A, D - A
        num = (np.sum(a * a, -1)[:, None] * np.cross(b, c)
               + np.sum(b * b, -1)[:, None] * np.cross(c, a)
               + np.sum(c * c, -1)[:, None] * np.cross(a, b))
        den = 2.0 * np.sum(a * np.cross(b, c), -1)[:, None]
        return A + num / den

    cT = circumcentre(P[:, 0], P[:, 1], P[:, 2], P[:, 3])
    # facet k is opposite vertex k
    opp = [(1, 2, 3), (0, 2, 3), (0, 1, 3), (0, 1, 2)]
    cF = [circumcentre(P[:, i], P[:, j], P[:, k]) for i, j, k in opp]

    edges_i, edges_j, areas = [], [], []
    for (u, v) in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)):
        w1, w2 = [k for k in range(4) if k not in (u, v)]
        # the two facets containing edge (u, v) are opposite w1 and w2
        m = 0.5 * (P[:, u] + P[:, v])
        e = P[:, v] - P[:, u]
        e = e / np.linalg.norm(e, axis=1)[:, None]
        a1 = 0.5 * np.sum(np.cross(cF[w1] - m, cT - m) * e, -1)
        a2 = 0.5 * np.sum(np.cross(cT - m, cF[w2] - m) * e, -1)
        edges_i.append(tets[:, u])
        edges_j.append(tets[:, v])
        areas.append(a1 + a2)
    ei = np.concatenate(edges_i)
    ej = np.concatenate(edges_j)
    ar = np.concatenate(areas)
    lo, hi = np.minimum(ei, ej), np.maximum(ei, ej)
    # orient each contribution with the edge lo -> hi
    ar = np.where(ei < ej, ar, -ar)
    key = lo * n_points + hi
    uk, inv = np.unique(key, return_inverse=True)
    area = np.abs(np.bincount(inv, weights=ar, minlength=len(uk)))
    c1 = (uk // n_points).astype(np.int64)
    c2 = (uk % n_points).astype(np.int64)
    # Guard against degenerate slivers: a face needs a positive area.
    area = np.maximum(area, 1e-12 * np.median(area))
    dvec = pts[c2] - pts[c1]
    dist = np.linalg.norm(dvec, axis=1)
    nrm = dvec / dist[:, None]
    s = nrm * area[:, None]
    faces_c = np.stack([c1 + 1, c2 + 1], axis=1).astype(np.int32)
    # cell volumes: 1/3 * sum over faces of area * (distance to face) = d/2
    vol = np.bincount(c1, weights=area * dist / 6.0, minlength=n_points) + \
        np.bincount(c2, weights=area * dist / 6.0, minlength=n_points)
    vol = np.maximum(vol, 1e-12)
    deg = np.bincount(c1, minlength=n_points) + np.bincount(c2, minlength=n_points)
    h = np.cbrt(vol)
    return Grid(n_cells=n_points, faces_c=faces_c,
                sx=s[:, 0].copy(), sy=s[:, 1].copy(), sz=s[:, 2].copy(),
                dx=dvec[:, 0].copy(), dy=dvec[:, 1].copy(), dz=dvec[:, 2].copy(),
                fw=np.full(len(c1), 0.5), vol=vol,
                h_min=float(dist.min()), h_mean=float(h.mean()),
                kind="poly", meta=dict(seed=seed, faces_per_cell_mean=float(deg.mean()),
                                       faces_per_cell_min=int(deg.min()),
                                       faces_per_cell_max=int(deg.max())))
