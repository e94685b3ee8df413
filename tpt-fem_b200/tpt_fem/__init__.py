"""tpt_fem -- Python front end of the B200 finite-element hot path.

Mirrors the reference's pyo3 module (crates/tpt-fem-py/src/lib.rs): a
``Mesh`` class with ``box_mesh`` / ``node_count`` / ``coords`` /
``nodes_on_plane`` / ``nodes_in_box`` and the solver functions
``solve_poisson`` / ``solve_elasticity`` returning result objects with
``values`` and ``to_numpy()``.  Below that it exposes the drop-in pieces of
the path -- ``assemble_poisson``, ``assemble_elasticity``, ``Matrix.to_csr``,
``reduce_system``, ``solve_with_dirichlet`` -- each a thin call through the C
ABI of ``libtptfem.so`` (include/tptfem.h).  Every computation runs on the GPU;
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from ._native import (CELL_QUAD4, CELL_TET4, CELL_TRI3, MODEL_BAR_AXIAL, MODEL_CONTINUUM_3D, MODEL_PLANE_STRAIN,
                      MODEL_PLANE_STRESS, SOLVER_FSAI_MP_PCG, SOLVER_JACOBI_PCG, SOLVER_LEARNED_FSAI_PCG,
                      SOLVER_MP_PCG, SolverOpts,
                      SolveStats)

__all__ = [
    "TptFemError", "Context", "Mesh", "Matrix", "System", "assemble_poisson", "assemble_elasticity",
    "load_poisson_source", "load_body", "apply_traction", "reduce_system", "solve_with_dirichlet",
    "solve_poisson", "solve_elasticity", "SolverOpts", "SolveStats", "CELL_TET4", "CELL_QUAD4", "CELL_TRI3",
    "MODEL_CONTINUUM_3D", "MODEL_PLANE_STRESS", "MODEL_PLANE_STRAIN", "SOLVER_JACOBI_PCG", "SOLVER_MP_PCG",
    "SOLVER_FSAI_MP_PCG", "SOLVER_LEARNED_FSAI_PCG",
]


class TptFemError(RuntimeError):
    """A non-OK tptfem_status, with the context's message."""

    def __init__(self, status, message):
        self.status = status
        self.name = N.STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.name}: {message}")


class Context:
    """One device + one CUDA stream (tptfem_context)."""

    _default = {}

    def __init__(self, device=0):
        self.lib = N.load()
        h = C.c_void_p()
        rc = self.lib.tptfem_create(device, C.byref(h))
        if rc != N.OK:
            raise TptFemError(rc, f"tptfem_create(device={device}) failed (no usable sm_100 GPU?)")
        self.h = h
        self.device = device

    @classmethod
    def default(cls, device=0):
        if device not in cls._default:
            cls._default[device] = Context(device)
        return cls._default[device]

    def check(self, rc):
        if rc != N.OK:
            buf = C.create_string_buffer(4096)
            self.lib.tptfem_last_error(self.h, buf, len(buf))
            raise TptFemError(rc, buf.value.decode(errors="replace"))

    def synchronize(self):
        self.check(self.lib.tptfem_synchronize(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.tptfem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ctx(ctx):
    return ctx if ctx is not None else Context.default()


class Mesh:
    """A device-resident mesh (tptfem_mesh).  Mirrors tpt_fem.Mesh of the reference bindings."""

    def __init__(self, handle, ctx):
        self.h = handle
        self.ctx = ctx
        nn, ne = C.c_int64(), C.c_int64()
        cell, cdim = C.c_int(), C.c_int()
        ctx.check(ctx.lib.tptfem_mesh_sizes(handle, C.byref(nn), C.byref(ne), C.byref(cell), C.byref(cdim)))
        self.n_nodes, self.n_elems, self.cell, self.cdim = nn.value, ne.value, cell.value, cdim.value
        self._coords = None
        self._conn = None

    @staticmethod
    def box_mesh(min, max, n, ctx=None):
        """box_mesh(min, max, n) built on the device (crates/tpt-fem-mesh-gen/src/lib.rs:422-495)."""
        ctx = _ctx(ctx)
        h = C.c_void_p()
        mn, mx, nn = N.f64(min), N.f64(max), N.i64(n)
        ctx.check(ctx.lib.tptfem_mesh_box(ctx.h, N.ptr(mn), N.ptr(mx), N.ptr(nn), C.byref(h)))
        return Mesh(h, ctx)

    @staticmethod
    def from_arrays(cell_type, coords, conn, ctx=None):
        ctx = _ctx(ctx)
        coords = N.f64(coords)
        conn = N.i64(conn)
        h = C.c_void_p()
        ctx.check(ctx.lib.tptfem_mesh_upload(ctx.h, cell_type, coords.shape[1], N.ptr(coords), coords.shape[0],
                                             N.ptr(conn), conn.shape[0], C.byref(h)))
        m = Mesh(h, ctx)
        m._coords, m._conn = coords, conn
        return m

    def _download(self):
        if self._coords is None:
            c = np.zeros((self.n_nodes, self.cdim))
            e = np.zeros((self.n_elems, 3 if self.cell == CELL_TRI3 else 4), dtype=np.int64)
            self.ctx.check(self.ctx.lib.tptfem_mesh_download(self.ctx.h, self.h, N.ptr(c), N.ptr(e)))
            self._coords, self._conn = c, e

    @property
    def coords_array(self):
        self._download()
        return self._coords

    @property
    def conn_array(self):
        self._download()
        return self._conn

    @property
    def dim(self):
        return 3 if self.cell == CELL_TET4 else 2

    def node_count(self):
        return self.n_nodes

    def element_count(self):
        return self.n_elems

    def coords(self, i):
        return [float(v) for v in self.coords_array[i]]

    def write_vtk(self, path, fields=None, title=None):
        """write_vtk / write_vtk_with_data (io-vtk/src/lib.rs:117-196): legacy binary
        .vtk with per-node scalar fields {name: values}, in the given order."""
        fields = dict(fields or {})
        names = (C.c_char_p * max(1, len(fields)))(*[k.encode() for k in fields])
        arrs = [N.f64(v) for v in fields.values()]
        for a in arrs:
            if a.shape != (self.n_nodes,):
                raise ValueError("each field needs one value per node")
        ptrs = (C.c_void_p * max(1, len(arrs)))(*[a.ctypes.data for a in arrs])
        self.ctx.check(self.ctx.lib.tptfem_mesh_write_vtk(self.ctx.h, self.h, str(path).encode(),
                                                          title.encode() if title else None, len(arrs),
                                                          C.cast(names, C.c_void_p), C.cast(ptrs, C.c_void_p)))

    def write_exodus(self, path):
        """write_exodus (io-exodus/src/lib.rs:384-563): NetCDF-3 classic Exodus II file."""
        self.ctx.check(self.ctx.lib.tptfem_mesh_write_exodus(self.ctx.h, self.h, str(path).encode()))

    def nodes_on_plane(self, axis, coord, tol):
        """Mesh::nodes_on_plane (crates/tpt-fem-mesh/src/lib.rs:425-431)."""
        c = self.coords_array
        col = c[:, axis] if axis < c.shape[1] else np.zeros(len(c))
        return [int(i) for i in np.nonzero(np.abs(col - coord) <= tol)[0]]

    def nodes_in_box(self, min, max):
        """Mesh::nodes_in_box (crates/tpt-fem-mesh/src/lib.rs:435-447), tolerance 1e-12."""
        c = self.coords_array
        tol = 1e-12
        ok = np.ones(len(c), dtype=bool)
        for d in range(3):
            v = c[:, d] if d < c.shape[1] else np.zeros(len(c))
            ok &= (v >= min[d] - tol) & (v <= max[d] + tol)
        return [int(i) for i in np.nonzero(ok)[0]]

    def __del__(self):
        if getattr(self, "h", None) is not None and self.ctx.h:
            self.ctx.lib.tptfem_mesh_free(self.h)
            self.h = None


class Matrix:
    """A device-resident CSR matrix (tptfem_matrix), equal to Coo::to_csr(assemble(...))."""

    def __init__(self, handle, mesh):
        self.h = handle
        self.mesh = mesh
        self.ctx = mesh.ctx
        nr, nc, nz = C.c_int64(), C.c_int64(), C.c_int64()
        self.ctx.check(self.ctx.lib.tptfem_matrix_sizes(handle, C.byref(nr), C.byref(nc), C.byref(nz)))
        self.nrows, self.ncols, self.nnz = nr.value, nc.value, nz.value

    def _refresh(self):
        nr, nc, nz = C.c_int64(), C.c_int64(), C.c_int64()
        self.ctx.check(self.ctx.lib.tptfem_matrix_sizes(self.h, C.byref(nr), C.byref(nc), C.byref(nz)))
        self.nrows, self.ncols, self.nnz = nr.value, nc.value, nz.value

    def to_csr(self):
        """(row_ptrs, col_ind, values) as int64/int64/float64 numpy arrays."""
        rp = np.zeros(self.nrows + 1, np.int64)
        ci = np.zeros(self.nnz, np.int64)
        va = np.zeros(self.nnz)
        self.ctx.check(self.ctx.lib.tptfem_matrix_download(self.ctx.h, self.h, N.ptr(rp), N.ptr(ci), N.ptr(va)))
        return rp, ci, va

    def matvec(self, x):
        """Csr::matvec (crates/tpt-fem-sparse/src/lib.rs:195-205), bit-exact."""
        x = N.f64(x)
        y = np.zeros(max(self.nrows, len(x)))
        self.ctx.check(self.ctx.lib.tptfem_csr_matvec(self.ctx.h, self.h, N.ptr(x), len(x), N.ptr(y)))
        return y

    def lanczos_eigs(self, num, which="smallest", lanczos_dim=None, vectors=True):
        """lanczos_eigs (eigen/src/lib.rs:223-262) on the device -> [(value, unit vector or None)]."""
        dim = lanczos_dim or self.nrows
        vals = np.zeros(max(num, 1))
        vecs = np.zeros((max(num, 1), self.nrows)) if vectors else None
        found = C.c_int()
        w = 1 if which == "largest" else 0
        self.ctx.check(self.ctx.lib.tptfem_lanczos_eigs(self.ctx.h, self.h, num, w, dim, N.ptr(vals),
                                                        N.ptr(vecs) if vectors else None, C.byref(found)))
        return [(float(vals[i]), vecs[i].copy() if vectors else None) for i in range(found.value)]

    def power_iteration(self, max_iter=200, tol=1e-12):
        """power_iteration (eigen/src/lib.rs:62-88) on the device -> (lambda, x, iterations)."""
        lam, it = C.c_double(), C.c_int()
        x = np.zeros(self.nrows)
        self.ctx.check(self.ctx.lib.tptfem_power_iteration(self.ctx.h, self.h, max_iter, tol, C.byref(lam),
                                                           N.ptr(x), C.byref(it)))
        return lam.value, x, it.value

    def profile_assembly(self, reps=10):
        """Average device time (ms) of a numeric re-assembly with resident coefficients (CUDA events)."""
        ms = C.c_double()
        self.ctx.check(self.ctx.lib.tptfem_matrix_profile_assembly(self.ctx.h, self.h, int(reps), C.byref(ms)))
        return ms.value

    def reassemble(self, coef):
        """New per-element (or constant) coefficients on the same mesh; pattern revalidated."""
        coef = np.atleast_1d(N.f64(coef))
        per = 1 if len(coef) > 1 or self.mesh.n_elems == 1 else 0
        self.ctx.check(self.ctx.lib.tptfem_reassemble(self.ctx.h, self.h, N.ptr(coef), per))
        self._refresh()

    def __del__(self):
        if getattr(self, "h", None) is not None and self.ctx.h:
            self.ctx.lib.tptfem_matrix_free(self.h)
            self.h = None


def _coef(mesh, coef):
    c = np.atleast_1d(N.f64(coef))
    if len(c) == 1:
        return c, 0
    if len(c) != mesh.n_elems:
        raise ValueError("coefficient array must hold one value per element or a single value")
    return c, 1


def assemble_poisson(mesh, conductivity, quad_order=2, robin=None):
    """assemble(mesh, 1, poisson_element_matrix) -> Matrix (thermal/src/lib.rs:132-160).

    robin adds apply_robin (assembly/src/lib.rs:674-753), as solve_poisson's
    `robin` argument does (thermal/src/lib.rs:235-237): a callable h(x, n) of
    the boundary point and its outward unit normal (numpy arrays), or
    (axis, sign, h) for the constant h on the boundary faces whose outward
    normal n has sign * n[axis] > 0.5 (axis=-1: every boundary face)."""
    ctx = mesh.ctx
    c, per = _coef(mesh, conductivity)
    h = C.c_void_p()
    if robin is None:
        ctx.check(ctx.lib.tptfem_assemble_poisson(ctx.h, mesh.h, N.ptr(c), per, quad_order, C.byref(h)))
    elif callable(robin):  # h(x, n) at every boundary-face quadrature point
        hv = _eval_flux(mesh, robin)
        ctx.check(ctx.lib.tptfem_assemble_poisson_robin_points(ctx.h, mesh.h, N.ptr(c), per, quad_order, N.ptr(hv),
                                                               C.byref(h)))
    else:
        axis, sign, coef = robin
        ctx.check(ctx.lib.tptfem_assemble_poisson_robin(ctx.h, mesh.h, N.ptr(c), per, quad_order, int(axis),
                                                        float(sign), float(coef), C.byref(h)))
    return Matrix(h, mesh)


_MODELS = {"bar": MODEL_BAR_AXIAL, "baraxial": MODEL_BAR_AXIAL, "planestress": MODEL_PLANE_STRESS,
           "planestrain": MODEL_PLANE_STRAIN, "3d": MODEL_CONTINUUM_3D, "continuum": MODEL_CONTINUUM_3D,
           "continuum3d": MODEL_CONTINUUM_3D}


def parse_model(model):
    """parse_model of the reference bindings (crates/tpt-fem-py/src/lib.rs:201-211)."""
    if isinstance(model, int):
        return model
    key = model.lower().replace("-", "").replace("_", "")
    if key not in _MODELS:
        raise TptFemError(9, f"unknown elasticity model '{key}' (bar | plane-stress | plane-strain | 3d)")
    return _MODELS[key]


def assemble_elasticity(mesh, model, young, poisson, quad_order=2):
    """try_assemble(mesh, dim, elasticity_element_matrix) -> Matrix (elasticity/src/lib.rs:262-309)."""
    ctx = mesh.ctx
    c, per = _coef(mesh, young)
    h = C.c_void_p()
    ctx.check(ctx.lib.tptfem_assemble_elasticity(ctx.h, mesh.h, parse_model(model), N.ptr(c), per, float(poisson),
                                                 quad_order, C.byref(h)))
    return Matrix(h, mesh)


def quadrature_points(mesh, quad_order=2):
    """Physical quadrature points of every element, (n_elems, nq, coord_dim):
    where the reference calls the source / body-force closure
    (thermal/src/lib.rs:163-196, elasticity/src/lib.rs:312-348)."""
    ctx = mesh.ctx
    nq = C.c_int32()
    ctx.check(ctx.lib.tptfem_mesh_quadrature_points(ctx.h, mesh.h, quad_order, C.byref(nq), None))
    pts = np.zeros((mesh.n_elems, nq.value, mesh.cdim))
    ctx.check(ctx.lib.tptfem_mesh_quadrature_points(ctx.h, mesh.h, quad_order, C.byref(nq), N.ptr(pts)))
    return pts


def boundary_points(mesh):
    """(x, normal): every boundary face's quadrature points and outward unit
    normals, (n_points, dim) each, faces in boundary_faces order
    (assembly/src/lib.rs:563-583): where apply_neumann / apply_robin call their
    closures."""
    ctx = mesh.ctx
    n = C.c_int64()
    ctx.check(ctx.lib.tptfem_mesh_boundary_points(ctx.h, mesh.h, C.byref(n), None, None))
    x = np.zeros((n.value, mesh.dim))
    nrm = np.zeros((n.value, mesh.dim))
    ctx.check(ctx.lib.tptfem_mesh_boundary_points(ctx.h, mesh.h, C.byref(n), N.ptr(x), N.ptr(nrm)))
    return x, nrm


def _xyz(x):
    """The reference bindings call a source as f(x, y, z), missing coordinates 0.0."""
    return (float(x[0]) if len(x) > 0 else 0.0, float(x[1]) if len(x) > 1 else 0.0,
            float(x[2]) if len(x) > 2 else 0.0)


def _eval_flux(mesh, fn):
    x, nrm = boundary_points(mesh)
    return np.array([float(fn(xp, n)) for xp, n in zip(x, nrm)], dtype=np.float64)


def load_poisson_source(mesh, source, quad_order=2):
    """The Poisson load loop of solve_poisson (thermal/src/lib.rs:224-230):
    source is a float or a callable f(x, y, z) evaluated at every quadrature point."""
    rhs = np.zeros(mesh.n_nodes)
    ctx = mesh.ctx
    if callable(source):
        pts = quadrature_points(mesh, quad_order).reshape(-1, mesh.cdim)
        sv = np.array([float(source(*_xyz(x))) for x in pts], dtype=np.float64)
        ctx.check(ctx.lib.tptfem_load_poisson_source_points(ctx.h, mesh.h, N.ptr(sv), quad_order, N.ptr(rhs)))
    else:
        ctx.check(ctx.lib.tptfem_load_poisson_source(ctx.h, mesh.h, float(source), quad_order, N.ptr(rhs)))
    return rhs


def load_body(mesh, body, quad_order=2):
    """The body-force loop of solve_elasticity (elasticity/src/lib.rs:371-379):
    body is a constant vector or a callable b(x, y, z) -> dim values."""
    rhs = np.zeros(mesh.n_nodes * mesh.dim)
    ctx = mesh.ctx
    if callable(body):
        pts = quadrature_points(mesh, quad_order).reshape(-1, mesh.cdim)
        bv = np.array([[float(v) for v in list(body(*_xyz(x)))[:mesh.dim]] for x in pts], dtype=np.float64)
        ctx.check(ctx.lib.tptfem_load_body_points(ctx.h, mesh.h, N.ptr(bv), quad_order, N.ptr(rhs)))
    else:
        b = N.f64(body)
        ctx.check(ctx.lib.tptfem_load_body(ctx.h, mesh.h, N.ptr(b), quad_order, N.ptr(rhs)))
    return rhs


def apply_neumann(mesh, dofs_per_node, flux, rhs, comp_mask=0xFFFFFFFF):
    """rhs += apply_neumann (assembly/src/lib.rs:591-667) with the flux g(x, n)
    of the boundary point and its outward unit normal (numpy arrays), applied
    to every component in comp_mask (in place)."""
    assert rhs.dtype == np.float64 and rhs.flags["C_CONTIGUOUS"]
    g = _eval_flux(mesh, flux)
    ctx = mesh.ctx
    ctx.check(ctx.lib.tptfem_apply_neumann_points(ctx.h, mesh.h, dofs_per_node, N.ptr(g), comp_mask, N.ptr(rhs)))
    return rhs


def apply_traction(mesh, dofs_per_node, axis, sign, traction, rhs):
    """rhs += apply_neumann with flux traction[c] on faces where sign*n[axis] > 0.5 (in place)."""
    t = N.f64(traction)
    assert rhs.dtype == np.float64 and rhs.flags["C_CONTIGUOUS"]
    mesh.ctx.check(mesh.ctx.lib.tptfem_apply_traction(mesh.ctx.h, mesh.h, dofs_per_node, axis, float(sign),
                                                      N.ptr(t), N.ptr(rhs)))
    return rhs


def _bcs(bcs):
    if len(bcs) == 0:
        return np.zeros(0, np.int64), np.zeros(0)
    arr = list(bcs)
    return N.i64([b[0] for b in arr]), N.f64([b[1] for b in arr])


def _opts(solver=SOLVER_JACOBI_PCG, tol=1e-10, inner_tol=0.0, max_iter=0, max_outer=0, batch=0, fresh_setup=False,
          csr_only=False, full_operator=False, coarse=False, coarse_aggregates=0):
    o = SolverOpts()
    o.solver, o.rel_tol, o.inner_rel_tol, o.max_iter, o.max_outer, o.batch = solver, tol, inner_tol, max_iter, \
        max_outer, batch
    o.flags = (N.SOLVE_FRESH_SETUP if fresh_setup else 0) | (N.SOLVE_CSR_ONLY if csr_only else 0) | \
        (N.SOLVE_FULL_OPERATOR if full_operator else 0) | (N.SOLVE_COARSE if coarse else 0)
    o.coarse_aggregates = coarse_aggregates
    return o


class System:
    """Device-resident ReducedSystem (assembly/src/lib.rs:488-535) plus its solution."""

    def __init__(self, handle, ctx, n):
        self.h, self.ctx, self.n = handle, ctx, n
        nf, nz = C.c_int64(), C.c_int64()
        ctx.check(ctx.lib.tptfem_system_sizes(handle, C.byref(nf), C.byref(nz)))
        self.n_free, self.nnz = nf.value, nz.value

    def download(self):
        """(row_ptrs, col_ind, values, fred, free)."""
        rp = np.zeros(self.n_free + 1, np.int64)
        ci = np.zeros(self.nnz, np.int64)
        va = np.zeros(self.nnz)
        fred = np.zeros(self.n_free)
        free = np.zeros(self.n_free, np.int64)
        self.ctx.check(self.ctx.lib.tptfem_system_download(self.ctx.h, self.h, N.ptr(rp), N.ptr(ci), N.ptr(va),
                                                           N.ptr(fred), N.ptr(free)))
        return rp, ci, va, fred, free

    def solve(self, **kw):
        o = _opts(**kw)
        st = SolveStats()
        rc = self.ctx.lib.tptfem_system_solve(self.ctx.h, self.h, C.byref(o), C.byref(st))
        self.ctx.check(rc)
        return st.as_dict()

    def refresh(self, mat, rhs):
        """New values (same mesh, same pattern, same Dirichlet set) for this system; structures are kept."""
        rhs = N.f64(rhs)
        self.ctx.check(self.ctx.lib.tptfem_system_refresh(self.ctx.h, self.h, mat.h, N.ptr(rhs), len(rhs)))

    def coarse(self, with_inverse=False):
        """The coarse space of the last coarse solve: dict(na, nm, bins[, ainv])."""
        na, nm = C.c_int32(), C.c_int32()
        bins = np.zeros(3, np.int32)
        self.ctx.check(self.ctx.lib.tptfem_system_coarse(self.ctx.h, self.h, C.byref(na), C.byref(nm), N.ptr(bins),
                                                         None))
        out = {"na": na.value, "nm": nm.value, "bins": bins.tolist()}
        if with_inverse and na.value:
            nc = na.value * nm.value
            a = np.zeros((nc, nc))
            self.ctx.check(self.ctx.lib.tptfem_system_coarse(self.ctx.h, self.h, C.byref(na), C.byref(nm),
                                                             N.ptr(bins), N.ptr(a)))
            out["ainv"] = a
        return out

    def profile_spmv(self, reps=20):
        """Average device ms of the solver's SpMV kernels as a dict: FP64 CSR, FP32 CSR, FP64 node-block
        full storage and symmetric half storage (with the bytes those layouts move per launch)."""
        v = [C.c_double() for _ in range(6)]
        self.ctx.check(self.ctx.lib.tptfem_system_profile_spmv(self.ctx.h, self.h, reps, *[C.byref(x) for x in v]))
        a, b, c, d, e, f = (x.value for x in v)
        return {"csr_f64_ms": a, "csr_f32_ms": b, "nb_ms": c, "nb_bytes": d, "nbs_ms": e, "nbs_bytes": f}

    def fsai(self):
        """Classic FSAI factor: (L row_ptrs, L cols, L values, sigma^2); G = diag(sigma)(I + L)."""
        nnz = C.c_int64()
        self.ctx.check(self.ctx.lib.tptfem_system_fsai(self.ctx.h, self.h, C.byref(nnz)))
        rp = np.zeros(self.n_free + 1, np.int64)
        ci = np.zeros(nnz.value, np.int64)
        va = np.zeros(nnz.value)
        s2 = np.zeros(self.n_free)
        self.ctx.check(self.ctx.lib.tptfem_system_fsai_download(self.ctx.h, self.h, N.ptr(rp), N.ptr(ci), N.ptr(va),
                                                                N.ptr(s2)))
        return rp, ci, va, s2

    def solution(self):
        u = np.zeros(self.n)
        self.ctx.check(self.ctx.lib.tptfem_system_solution(self.ctx.h, self.h, N.ptr(u)))
        return u

    def __del__(self):
        if getattr(self, "h", None) is not None and self.ctx.h:
            self.ctx.lib.tptfem_system_free(self.h)
            self.h = None


def reduce_system(mat, rhs, bcs):
    ctx = mat.ctx
    rhs = N.f64(rhs)
    dof, val = _bcs(bcs)
    h = C.c_void_p()
    ctx.check(ctx.lib.tptfem_reduce_system(ctx.h, mat.h, N.ptr(rhs), len(rhs), N.ptr(dof), N.ptr(val), len(dof),
                                           C.byref(h)))
    return System(h, ctx, len(rhs))


def solve_with_dirichlet(mat, rhs, bcs, **kw):
    """solve_with_dirichlet (assembly/src/lib.rs:543-559) -> (u, stats dict)."""
    ctx = mat.ctx
    rhs = N.f64(rhs)
    dof, val = _bcs(bcs)
    u = np.zeros(len(rhs))
    o = _opts(**kw)
    st = SolveStats()
    ctx.check(ctx.lib.tptfem_solve_with_dirichlet(ctx.h, mat.h, N.ptr(rhs), len(rhs), N.ptr(dof), N.ptr(val),
                                                  len(dof), C.byref(o), N.ptr(u), C.byref(st)))
    return u, st.as_dict()


def grf_eval(points, w, phi, scale, ctx=None):
    """scale * sum_m cos(w[:, m] . x + phi[m]) at each row x of points (n x 3),
    evaluated on the GPU in a fixed operation order (tptfem_grf_eval)."""
    ctx = _ctx(ctx)
    pts = N.f64(points).reshape(-1, 3)
    w = N.f64(w).reshape(3, -1)
    phi = N.f64(phi)
    assert w.shape[1] == len(phi)
    out = np.zeros(len(pts))
    ctx.check(ctx.lib.tptfem_grf_eval(ctx.h, N.ptr(pts), len(pts), N.ptr(w), N.ptr(phi), len(phi), float(scale),
                                      N.ptr(out)))
    return out


class PoissonSolution:
    def __init__(self, mesh, values, stats):
        self.mesh, self.values, self.stats = mesh, values, stats

    def __len__(self):
        return len(self.values)

    def to_numpy(self):
        return np.asarray(self.values, dtype=np.float64).reshape(self.mesh.node_count())


class ElasticitySolution:
    def __init__(self, mesh, values, dim, stats):
        self.mesh, self.values, self.dim, self.stats = mesh, values, dim, stats

    def __len__(self):
        return len(self.values)

    def to_numpy(self):
        return np.asarray(self.values, dtype=np.float64).reshape(self.mesh.node_count(), self.dim)


def solve_poisson(mesh, conductivity, quad_order, source, bcs, neumann=None, robin=None, **kw):
    """solve_poisson of the reference bindings (crates/tpt-fem-py/src/lib.rs:102-199):
    source is a float or a callable f(x, y, z); neumann and robin are the
    optional flux g(x, n) and Robin coefficient h(x, n) of the Rust function
    (crates/tpt-fem-thermal/src/lib.rs:206-240), each a callable of the boundary
    point and its outward unit normal."""
    if callable(source) or neumann is not None or robin is not None:
        K = assemble_poisson(mesh, conductivity, quad_order, robin=robin)
        rhs = load_poisson_source(mesh, source, quad_order)
        if neumann is not None:
            apply_neumann(mesh, 1, neumann, rhs)
        u, st = solve_with_dirichlet(K, rhs, bcs, **kw)
        return PoissonSolution(mesh, [float(v) for v in u], st)
    ctx = mesh.ctx
    dof, val = _bcs(bcs)
    u = np.zeros(mesh.n_nodes)
    o = _opts(**kw)
    st = SolveStats()
    ctx.check(ctx.lib.tptfem_solve_poisson(ctx.h, mesh.h, float(conductivity), quad_order, float(source),
                                           N.ptr(dof), N.ptr(val), len(dof), C.byref(o), N.ptr(u), C.byref(st)))
    return PoissonSolution(mesh, [float(v) for v in u], st.as_dict())


def solve_elasticity(mesh, model, young, poisson, quad_order, bcs, body=None, **kw):
    """solve_elasticity of the reference bindings (crates/tpt-fem-py/src/lib.rs:213-252).

    ``bcs`` are (node_id, component, value) triples; zero body force unless
    ``body`` is given, as a constant vector or a callable b(x, y, z) -> dim values.
    """
    ctx = mesh.ctx
    dim = mesh.dim
    dofs = [(int(n) * dim + int(c), float(v)) for n, c, v in bcs]
    if callable(body):
        K = assemble_elasticity(mesh, model, young, poisson, quad_order)
        u, st = solve_with_dirichlet(K, load_body(mesh, body, quad_order), dofs, **kw)
        return ElasticitySolution(mesh, [float(v) for v in u], dim, st)
    dof, val = _bcs(dofs)
    b = N.f64(body if body is not None else np.zeros(dim))
    u = np.zeros(mesh.n_nodes * dim)
    o = _opts(**kw)
    st = SolveStats()
    ctx.check(ctx.lib.tptfem_solve_elasticity(ctx.h, mesh.h, parse_model(model), float(young), float(poisson),
                                              quad_order, N.ptr(b), N.ptr(dof), N.ptr(val), len(dof), C.byref(o),
                                              N.ptr(u), C.byref(st)))
    return ElasticitySolution(mesh, [float(v) for v in u], dim, st.as_dict())
