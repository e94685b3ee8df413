"""Batched 2-D SIMP topology optimisation on the GPU (csrc/topopt.cu).

Mirrors the reference's ``tpt_fem_topopt`` crate (crates/tpt-fem-topopt/src/lib.rs):
``Grid``, ``TopOptParams``, ``cantilever_load`` and ``topopt_simp`` keep the
reference's names and meaning; ``topopt_batch`` runs many instances in one
call (one CTA per instance, all optimality-criteria iterations in one CUDA
graph).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

E_MIN_FACTOR = 1e-3  # topopt:54


@dataclass
class Grid:
    """Grid::new(nx, ny, h) (topopt:89-116): nx * ny nodes, (nx-1)(ny-1) Quad4 elements."""
    nx: int
    ny: int
    h: float = 1.0

    @property
    def nelx(self):
        return self.nx - 1

    @property
    def nely(self):
        return self.ny - 1

    def n_nodes(self):
        return self.nx * self.ny

    def n_elem(self):
        return (self.nx - 1) * (self.ny - 1)


@dataclass
class TopOptParams:
    """TopOptParams (topopt:130-147); emin defaults to E_MIN_FACTOR * e0 as the reference fixes it.
    density_filter=True selects the 88-line code's density filter (not in the reference)."""
    grid: Grid
    e0: float = 1.0
    nu: float = 0.3
    vol_frac: float = 0.5
    penal: float = 3.0
    filter_radius: float = 1.5
    max_iter: int = 100
    move_limit: float = 0.2
    emin: float | None = None
    density_filter: bool = False


@dataclass
class TopOptResult:
    densities: np.ndarray
    compliance: np.ndarray
    iterations: int
    stats: dict = field(default_factory=dict)


def cantilever_load(grid, load=1.0, node=None):
    """cantilever_load (topopt:398-415): left edge clamped, -y point load at the
    bottom-right node (or at `node`)."""
    f = np.zeros(2 * grid.n_nodes())
    bcs = []
    for j in range(grid.ny):
        n = j * grid.nx
        bcs += [(2 * n, 0.0), (2 * n + 1, 0.0)]
    f[2 * (grid.nx - 1 if node is None else node) + 1] = -load
    return f, bcs


def element_stiffness_unit(nu, h):
    ke = np.zeros(64)
    rc = N.load().tptfem_topopt_element_stiffness(float(nu), float(h), N.ptr(ke))
    if rc != N.OK:
        raise ValueError("invalid nu or h")
    return ke.reshape(8, 8)


def topopt_batch(ctx, problems, rel_tol=1e-10, max_pcg_iter=0, block_threads=0, use_graph=True, plain_jacobi=False,
                 pcg_only=False):
    """Run [(TopOptParams, f, bcs), ...] (f/bcs None: cantilever_load) on ctx's GPU.

    Displacement solves: banded Cholesky per instance (grids at most 110 nodes
    across), PCG otherwise or with pcg_only.

    Returns ([TopOptResult, ...], stats dict)."""
    n = len(problems)
    arr = (N.TopoptInstance * n)()
    keep = []
    for k, (P, f, bcs) in enumerate(problems):
        g = P.grid
        I = arr[k]
        I.nelx, I.nely, I.max_iter, I.density_filter = g.nelx, g.nely, int(P.max_iter), int(bool(P.density_filter))
        I.h, I.e0, I.nu, I.vol_frac, I.penal = g.h, P.e0, P.nu, P.vol_frac, P.penal
        I.filter_radius, I.move_limit = P.filter_radius, P.move_limit
        I.emin = E_MIN_FACTOR * P.e0 if P.emin is None else P.emin
        if f is None:
            f, bcs_default = cantilever_load(g)
            bcs = bcs_default if bcs is None else bcs
        fv = np.ascontiguousarray(f, dtype=np.float64)
        if fv.size != 2 * g.n_nodes():
            raise ValueError("load vector must have 2 * n_nodes entries")
        keep.append(fv)
        I.f = fv.ctypes.data
        if bcs is not None:
            if len(bcs) == 0:
                raise ValueError("at least one Dirichlet condition is required")
            dof = np.ascontiguousarray([int(b[0]) for b in bcs], dtype=np.int64)
            val = np.ascontiguousarray([float(b[1]) for b in bcs], dtype=np.float64)
            keep += [dof, val]
            I.bc_dof = dof.ctypes.data
            I.bc_val = val.ctypes.data
            I.nbc = dof.size
    ncomp = sum(int(P.max_iter) + 1 for P, _, _ in problems)
    nden = sum(P.grid.n_elem() for P, _, _ in problems)
    comp = np.zeros(ncomp)
    dens = np.zeros(nden)
    opts = N.TopoptOpts(float(rel_tol), int(max_pcg_iter), int(block_threads), int(bool(use_graph)),
                        int(bool(plain_jacobi)), int(bool(pcg_only)))
    st = N.TopoptStats()
    ctx.check(ctx.lib.tptfem_topopt_batch(ctx.h, C.cast(arr, C.c_void_p), n, C.byref(opts), N.ptr(comp), N.ptr(dens),
                                          C.byref(st)))
    out, a, b = [], 0, 0
    for P, _, _ in problems:
        m, ne = int(P.max_iter) + 1, P.grid.n_elem()
        out.append(TopOptResult(densities=dens[b:b + ne].copy(), compliance=comp[a:a + m].copy(),
                                iterations=int(P.max_iter)))
        a += m
        b += ne
    return out, st.as_dict()


def topopt_simp(params, f, bcs, ctx=None, **kw):
    """topopt_simp (topopt:342-385) for one instance on the GPU."""
    from . import Context
    ctx = ctx or Context.default()
    res, stats = topopt_batch(ctx, [(params, f, bcs)], **kw)
    res[0].stats = stats
    return res[0]
