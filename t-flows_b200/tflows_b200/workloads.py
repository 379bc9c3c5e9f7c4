"""Seeded synthetic workloads for the batched and served solvers.

The reference ships no benchmark suite, so these stand in for it with the
shapes the workloads name:

* batched: `count` independent systems, sizes log-uniform in [nmin, nmax];
  even entries are hex pressure-Poisson systems (Cg; one grid per distinct
  edge length m = round(n^(1/3)), per-system seeded RHS), odd entries are
  polyhedral upwind convection-diffusion systems (Bicg; Peclet uniform in
  [1, 50], per-system seeded face velocities and RHS) on a pool of
  `n_poly_grids` log-spaced jittered-lattice polyhedral grids.  The time
  step is CFL 0.1: at CFL 0.5 the reference's Bicg (the Cg recurrence on
  a non-symmetric matrix) diverges for Pe >~ 3 on these meshes, at 0.1 it
  converges for every Pe in [1, 50].
* served: a pool of systems of both kinds with sizes log-uniform in
  [nmin, nmax]; each request draws a pool member and gets its own seeded RHS.
"""
import concurrent.futures as cf
import math

import numpy as np

from . import grids, systems


def _hex_pressure(m, seeds):
    g = grids.hex_grid(m, m, m)
    csr = systems.create_matrix(g)
    out = []
    for sd in seeds:
        s = systems.pressure_system(g, sd, tol=1e-10, miter=50000, singular="pin", norm=1.0,
                                    csr=csr, name=f"hex-poisson-{m}^3-s{sd}")
        out.append(s)
    return out


def _poly_momentum(n, grid_seed, items):
    g = grids.poly_lattice_grid(n, grid_seed)
    csr = systems.create_matrix(g)
    out = []
    for sd, pe in items:
        s = systems.momentum_system(g, sd, tol=1e-10, miter=50000, peclet=pe, cfl=0.1,
                                    csr=csr, name=f"poly-cd-{g.n_cells}-pe{pe:.1f}-s{sd}")
        out.append(s)
    return out


def batched(count=512, seed=4, nmin=1e3, nmax=1e6, n_poly_grids=16, threads=16):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(nmin), math.log(nmax), count))
    pes = rng.uniform(1.0, 50.0, count)
    hex_jobs, poly_jobs = {}, {}
    grid_sizes = np.exp(np.linspace(math.log(nmin), math.log(nmax), n_poly_grids))
    order = []
    for k in range(count):
        sd = seed * 100000 + k
        if k % 2 == 0:
            m = max(4, int(round(sizes[k] ** (1.0 / 3.0))))
            hex_jobs.setdefault(m, []).append(sd)
            order.append(("hex", m, sd))
        else:
            gi = int(np.argmin(np.abs(np.log(grid_sizes) - math.log(sizes[k]))))
            poly_jobs.setdefault(gi, []).append((sd, float(pes[k])))
            order.append(("poly", gi, sd))
    built = {}
    with cf.ThreadPoolExecutor(threads) as ex:
        futs = {ex.submit(_hex_pressure, m, sds): ("hex", m) for m, sds in hex_jobs.items()}
        futs.update({ex.submit(_poly_momentum, int(grid_sizes[gi]), seed * 1000 + gi, it):
                     ("poly", gi) for gi, it in poly_jobs.items()})
        for f in cf.as_completed(futs):
            kind, key = futs[f]
            for s in f.result():
                built[(kind, key, int(s.name.rsplit("-s", 1)[1]))] = s
    return [built[o] for o in order]


def served_pool(seed=5, nmin=1e4, nmax=4e6, per_kind=12, threads=16):
    """Pool of systems for the served stream: sizes log-spaced over
    [nmin, nmax], half hex Poisson (Cg), half polyhedral convection-diffusion
    (Bicg, Peclet drawn uniform in [1, 50])."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(np.linspace(math.log(nmin), math.log(nmax), per_kind))
    jobs = []
    with cf.ThreadPoolExecutor(threads) as ex:
        for k, n in enumerate(sizes):
            m = max(4, int(round(n ** (1.0 / 3.0))))
            jobs.append(ex.submit(_hex_pressure, m, [seed * 100000 + k]))
            jobs.append(ex.submit(_poly_momentum, int(n), seed * 1000 + k,
                                  [(seed * 100000 + 500 + k, float(rng.uniform(1, 50)))]))
        pool = [s for f in jobs for s in f.result()]
    pool.sort(key=lambda s: s.n)
    return pool


def with_rhs(s, seed):
    """Same system, fresh seeded right-hand side (zero mean for Poisson)."""
    import copy
    t = copy.copy(s)
    t.b = systems.uniform_rhs(s.n, seed, zero_mean=(s.solver == "cg"))
    return t


def nrms_b(s):
    """NRMS of b with norm = 1 (Normalized_Root_Mean_Square.f90): the
    reference's residual measure at x = 0."""
    a = s.val[s.csr.dia - 1]
    return float(np.sqrt(np.sum((s.b / a) ** 2)))
