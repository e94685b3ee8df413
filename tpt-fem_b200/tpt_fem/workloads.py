"""Seeded synthetic inputs for the benchmark configurations.

No dataset exists for this path; every input is generated here with a fixed
seed, with the shapes and value distributions the benchmark configurations
name:
  * elasticity cantilever on box_mesh [0,L]x[0,1]x[0,1]: per-brick density
    rho ~ U[0,1], 3x3x3 box-filter mean truncated at the boundary,
    E = 1e-3 + (1 - 1e-3) * rho^3 per tet (6 tets per brick), nu = 0.3,
    x = 0 clamped, uniform traction (0, 0, -1e-3) on x = L;
  * the unit-cube elasticity case (E = 1) with the same clamp and traction.
"""
from __future__ import annotations

import numpy as np


def smoothed_density(n, seed):
    """rho ~ U[0,1] per brick, then the mean over the 3x3x3 neighbourhood that lies inside the box."""
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.0, 1.0, size=(nx, ny, nz))
    pad = np.pad(r, 1)
    one = np.pad(np.ones_like(r), 1)
    s = np.zeros_like(r)
    c = np.zeros_like(r)
    for di in range(3):
        for dj in range(3):
            for dk in range(3):
                s += pad[di:di + nx, dj:dj + ny, dk:dk + nz]
                c += one[di:di + nx, dj:dj + ny, dk:dk + nz]
    return s / c


def simp_young(rho, emin=1e-3, p=3.0):
    return emin + (1.0 - emin) * rho ** p


def per_tet(brick_values):
    """box_mesh numbers bricks (i, j, k) with k fastest and emits 6 tets per brick in order."""
    return np.repeat(brick_values.reshape(-1), 6)


def cantilever_young(n, seed=2024):
    return per_tet(simp_young(smoothed_density(n, seed)))


def clamp_x0_bcs(coords, dpn=3, tol=1e-9):
    nodes = np.nonzero(np.abs(coords[:, 0]) <= tol)[0]
    dof = (nodes[:, None] * dpn + np.arange(dpn)[None, :]).reshape(-1).astype(np.int64)
    return dof, np.zeros(len(dof))


def box_coords(mn, mx, n):
    """box_mesh node coordinates (k fastest), the same values the device mesher writes."""
    nx, ny, nz = n
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    t = i.reshape(-1) / nx
    u = j.reshape(-1) / ny
    w = k.reshape(-1) / nz
    return np.stack([mn[0] + t * (mx[0] - mn[0]), mn[1] + u * (mx[1] - mn[1]), mn[2] + w * (mx[2] - mn[2])], axis=1)


def tet_centroids(coords, conn):
    return coords[conn].mean(axis=1)


def grf_at_centroids(coords, conn, seed, ctx=None, length=0.1, n_features=1024):
    """grf_log_conductivity at the element centroids (mean of the element's
    nodes, numpy)."""
    return grf_log_conductivity(tet_centroids(coords, conn), seed, ctx, length, n_features)


class GrfPoisson:
    """Heterogeneous Poisson on the unit cube, box_mesh [n, n, n]: k = exp(g) per
    tet with g the seeded Gaussian random field at its centroid, f = 1,
    u = 0 on all six faces, quadrature order 2.  One mesh; matrix() assembles
    the operator of a field, system() reduces it."""

    def __init__(self, ctx, n):
        import tpt_fem as F
        self.F = F
        self.mesh = F.Mesh.box_mesh([0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [n, n, n], ctx=ctx)
        c = self.mesh.coords_array
        self.coords, self.conn = c, self.mesh.conn_array
        self.rhs = F.load_poisson_source(self.mesh, 1.0, 2)
        on_b = np.nonzero(np.any((c < 1e-9) | (c > 1 - 1e-9), axis=1))[0]
        self.bcs = [(int(i), 0.0) for i in on_b]

    def matrix(self, seed):
        k = np.exp(grf_at_centroids(self.coords, self.conn, seed, self.mesh.ctx))
        return self.F.assemble_poisson(self.mesh, k, 2)

    def system(self, seed):
        return self.F.reduce_system(self.matrix(seed), self.rhs, self.bcs)


def grf_poisson_system(ctx, n, seed):
    """The reduced GrfPoisson system of one field on a fresh mesh."""
    return GrfPoisson(ctx, n).system(seed)


def grf_log_conductivity(points, seed, ctx=None, length=0.1, n_features=1024):
    """Seeded Gaussian random field (mean 0, variance 1, squared-exponential
    correlation of length `length`) by random Fourier features:
    g(x) = sqrt(2/M) sum_m cos(w_m . x + phi_m), w_m ~ N(0, length^-2 I),
    phi_m ~ U[0, 2 pi) drawn from numpy's PCG64 stream of `seed`.  The sum is
    evaluated by the library (tptfem_grf_eval, one fixed operation order), so
    a seed gives the same field on every host."""
    import tpt_fem as F
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((3, n_features)) / length
    phi = rng.uniform(0.0, 2.0 * np.pi, n_features)
    return F.grf_eval(points, w, phi, np.sqrt(2.0 / n_features), ctx=ctx)


CANTILEVERS = {
    "cantilever_200x50x50": ([0.0, 0.0, 0.0], [4.0, 1.0, 1.0], [200, 50, 50]),
    "cantilever_280x70x70": ([0.0, 0.0, 0.0], [4.0, 1.0, 1.0], [280, 70, 70]),
    "cantilever_400x100x100": ([0.0, 0.0, 0.0], [4.0, 1.0, 1.0], [400, 100, 100]),
    "cube_elasticity_64": ([0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [64, 64, 64]),
}


TOPOPT_SIZES = [(60, 20), (90, 30), (120, 40), (180, 60), (240, 80)]


def topopt_batch_problems(n=512, seed=7, max_iter=100):
    """The batched 2-D SIMP workload: n plane-stress Q1 cantilevers, (nelx, nely)
    drawn uniformly from TOPOPT_SIZES, vol_frac ~ U[0.3, 0.5], E0 = 1,
    Emin = 1e-9, nu = 0.3, penalty 3, density filter radius 1.5 (h = 1), move
    limit 0.2, left edge clamped, unit -y load at the mid-right node
    (i = nelx, j = nely / 2), max_iter OC iterations.  Returns
    [(TopOptParams, f, bcs), ...] for tpt_fem.topopt.topopt_batch."""
    from .topopt import Grid, TopOptParams, cantilever_load
    rng = np.random.default_rng(seed)
    sizes = rng.integers(0, len(TOPOPT_SIZES), size=n)
    vfs = rng.uniform(0.3, 0.5, size=n)
    out = []
    for k in range(n):
        nelx, nely = TOPOPT_SIZES[sizes[k]]
        g = Grid(nelx + 1, nely + 1, 1.0)
        P = TopOptParams(grid=g, e0=1.0, nu=0.3, vol_frac=float(vfs[k]), penal=3.0, filter_radius=1.5,
                         max_iter=max_iter, move_limit=0.2, emin=1e-9, density_filter=True)
        f, bcs = cantilever_load(g, 1.0, node=g.nx * (nely // 2) + nelx)
        out.append((P, f, bcs))
    return out
