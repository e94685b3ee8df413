"""ctypes front end of the CPU parity oracle (``oracle/liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``, always as the checker, never as the
product.  Every function restates a reference function; the C++ source
``oracle/oracle.cpp`` cites the file:line it follows.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

CELL_LINE, CELL_TRI, CELL_QUAD, CELL_TET = 1, 2, 3, 4
MODEL_BAR, MODEL_PLANE_STRESS, MODEL_PLANE_STRAIN, MODEL_3D = 0, 1, 2, 3
NODES_PER_CELL = {CELL_LINE: 2, CELL_TRI: 3, CELL_QUAD: 4, CELL_TET: 4}
DIM_OF_CELL = {CELL_LINE: 1, CELL_TRI: 2, CELL_QUAD: 2, CELL_TET: 3}

_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_vp = C.c_void_p
_i64 = C.c_int64

SOURCE_CB = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_int, C.c_void_p)
FLUX_CB = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_void_p)
BODY_CB = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.c_void_p)


def build() -> str:
    """Compile liboracle.so with the committed Makefile (no-op when fresh)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    sig = {
        "orc_last_error": (C.c_char_p, []),
        "orc_box_mesh_sizes": (None, [_i64p, C.POINTER(_i64), C.POINTER(_i64)]),
        "orc_box_mesh": (None, [_f64p, _f64p, _i64p, _f64p, _i64p]),
        "orc_mesh_new": (_vp, [C.c_int, C.c_int, _f64p, _i64, _i64p, _i64, C.c_int]),
        "orc_mesh_free": (None, [_vp]),
        "orc_poisson_element_matrix": (C.c_int, [_vp, _i64, C.c_double, C.c_int, _f64p]),
        "orc_elasticity_element_matrix": (C.c_int, [_vp, _i64, C.c_int, C.c_double, C.c_double, C.c_int, _f64p]),
        "orc_assemble_poisson": (_vp, [_vp, _f64p, C.c_int, C.c_int]),
        "orc_assemble_elasticity": (_vp, [_vp, C.c_int, _f64p, C.c_int, C.c_double, C.c_int]),
        "orc_assemble_given": (_vp, [_vp, C.c_int, _f64p]),
        "orc_csr_rows": (_vp, [_vp, C.c_int, C.c_int, _f64p, C.c_int, C.c_double, C.c_int, _i64p, _i64]),
        "orc_rows_nnz": (_i64, [_vp]),
        "orc_rows_copy": (None, [_vp, _i64p, _i64p, _f64p]),
        "orc_rows_free": (None, [_vp]),
        "orc_load_poisson_rows": (C.c_int, [_vp, C.c_double, C.c_int, _i64p, _i64, _f64p]),
        "orc_coo_new": (_vp, []),
        "orc_coo_push": (None, [_vp, _i64, _i64, C.c_double]),
        "orc_coo_len": (_i64, [_vp]),
        "orc_coo_copy": (None, [_vp, _i64p, _i64p, _f64p]),
        "orc_coo_free": (None, [_vp]),
        "orc_to_csr": (_vp, [_vp]),
        "orc_csr_dims": (None, [_vp, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
        "orc_csr_copy": (None, [_vp, _i64p, _i64p, _f64p]),
        "orc_csr_from_arrays": (_vp, [_i64, _i64, _i64p, _i64p, _f64p]),
        "orc_csr_free": (None, [_vp]),
        "orc_csr_matvec": (None, [_vp, _f64p, _i64, _f64p]),
        "orc_load_poisson_source": (C.c_int, [_vp, C.c_double, C.c_int, _f64p]),
        "orc_load_poisson_source_cb": (C.c_int, [_vp, SOURCE_CB, _vp, C.c_int, _f64p]),
        "orc_load_body": (C.c_int, [_vp, _f64p, C.c_int, _f64p]),
        "orc_load_body_cb": (C.c_int, [_vp, BODY_CB, _vp, C.c_int, _f64p]),
        "orc_apply_neumann_cb": (None, [_vp, C.c_int, FLUX_CB, _vp, C.c_int, C.c_uint, _f64p]),
        "orc_apply_robin": (None, [_vp, _vp, C.c_int, C.c_int, C.c_double, C.c_double]),
        "orc_apply_robin_cb": (None, [_vp, _vp, C.c_int, FLUX_CB, _vp, C.c_int]),
        "orc_apply_traction": (None, [_vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint, _f64p]),
        "orc_boundary_face_count": (_i64, [_vp]),
        "orc_reduce_system": (_vp, [_vp, _f64p, _i64, _i64p, _f64p, _i64]),
        "orc_reduced_nfree": (_i64, [_vp]),
        "orc_reduced_kred": (_vp, [_vp]),
        "orc_reduced_copy": (None, [_vp, _f64p, _i64p]),
        "orc_reduced_free": (None, [_vp]),
        "orc_solve": (C.c_int, [_vp, _f64p, _i64, _f64p]),
        "orc_solve_with_dirichlet": (C.c_int, [_vp, _f64p, _i64, _i64p, _f64p, _i64, _f64p]),
        "orc_pcg_jacobi": (_i64, [_i64, _i64p, _i64p, _f64p, _f64p, _f64p, C.c_double, _i64, C.c_int,
                                  C.POINTER(C.c_double)]),
        "orc_pcg_jacobi_i32": (_i64, [_i64, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_double, _i64, C.c_int,
                                      C.POINTER(C.c_double)]),
        "orc_max_threads": (C.c_int, []),
        "orc_map": (None, [C.c_int, _f64p, C.c_int, C.c_int, _f64p, _f64p, C.POINTER(C.c_double), _f64p]),
        "orc_cell_quad": (C.c_int, [C.c_int, C.c_int, _f64p, _f64p]),
        "orc_fsai": (_vp, [_i64, _i64p, _i64p, _f64p, _vp, _vp]),
        "orc_topopt_ke0": (None, [C.c_double, C.c_double, _f64p]),
        "orc_topopt_filter_sensitivity": (None, [_i64, _i64, C.c_double, _f64p, C.c_double, _f64p]),
        "orc_topopt_oc_update": (None, [_i64, _f64p, _f64p, C.c_double, C.c_double, _f64p]),
        "orc_topopt": (C.c_int, [_i64, _i64, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_double, _i64, C.c_int, C.c_int, _f64p, _i64p, _f64p,
                                 _i64, _f64p, _f64p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class OracleError(RuntimeError):
    pass


def _err():
    return lib().orc_last_error().decode()


# ---- mesh -------------------------------------------------------------------

def box_mesh(mn, mx, n):
    """box_mesh (mesh-gen/src/lib.rs:422-495): coords (N,3) f64, conn (E,4) i64."""
    n = np.ascontiguousarray(n, dtype=np.int64)
    nn, ne = _i64(), _i64()
    lib().orc_box_mesh_sizes(n, C.byref(nn), C.byref(ne))
    coords = np.zeros((nn.value, 3))
    conn = np.zeros((ne.value, 4), dtype=np.int64)
    lib().orc_box_mesh(np.ascontiguousarray(mn, dtype=np.float64), np.ascontiguousarray(mx, dtype=np.float64),
                       n, coords, conn)
    return coords, conn


def nodes_on_plane(coords, axis, coord, tol):
    """Mesh::nodes_on_plane (mesh/src/lib.rs:425-431)."""
    c = coords[:, axis] if coords.shape[1] > axis else np.zeros(len(coords))
    return np.nonzero(np.abs(c - coord) <= tol)[0].astype(np.int64)


class Mesh:
    def __init__(self, cell, coords, conn):
        self.cell = cell
        self.coords = np.ascontiguousarray(coords, dtype=np.float64)
        self.conn = np.ascontiguousarray(conn, dtype=np.int64)
        if self.coords.ndim == 1:
            self.coords = self.coords[:, None].copy()
        self.cdim = self.coords.shape[1]
        self.npe = self.conn.shape[1]
        self.h = lib().orc_mesh_new(cell, self.cdim, self.coords, len(self.coords), self.conn, len(self.conn),
                                    self.npe)

    @property
    def n_nodes(self):
        return len(self.coords)

    @property
    def n_elems(self):
        return len(self.conn)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_mesh_free(self.h)
            self.h = None


# ---- sparse -----------------------------------------------------------------

class Coo:
    """Coo (sparse/src/lib.rs:40-118)."""

    def __init__(self, h=None):
        self.h = h if h is not None else lib().orc_coo_new()

    def push(self, r, c, v):
        lib().orc_coo_push(self.h, int(r), int(c), float(v))

    def __len__(self):
        return lib().orc_coo_len(self.h)

    def triplets(self):
        n = len(self)
        r = np.zeros(n, np.int64); c = np.zeros(n, np.int64); v = np.zeros(n)
        if n:
            lib().orc_coo_copy(self.h, r, c, v)
        return r, c, v

    def to_csr(self):
        h = lib().orc_to_csr(self.h)
        try:
            return Csr._from_handle(h)
        finally:
            lib().orc_csr_free(h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_coo_free(self.h)
            self.h = None


class Csr:
    """Csr (sparse/src/lib.rs:51-63) with numpy arrays."""

    def __init__(self, nrows, ncols, row_ptrs, col_ind, values):
        self.nrows, self.ncols = int(nrows), int(ncols)
        self.row_ptrs = np.ascontiguousarray(row_ptrs, dtype=np.int64)
        self.col_ind = np.ascontiguousarray(col_ind, dtype=np.int64)
        self.values = np.ascontiguousarray(values, dtype=np.float64)

    @classmethod
    def _from_handle(cls, h):
        nr, nc, nnz = _i64(), _i64(), _i64()
        lib().orc_csr_dims(h, C.byref(nr), C.byref(nc), C.byref(nnz))
        rp = np.zeros(nr.value + 1, np.int64)
        ci = np.zeros(nnz.value, np.int64)
        va = np.zeros(nnz.value)
        lib().orc_csr_copy(h, rp, ci, va)
        return cls(nr.value, nc.value, rp, ci, va)

    @property
    def nnz(self):
        return len(self.values)

    def matvec(self, x):
        """Csr::matvec (sparse/src/lib.rs:195-205)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        h = lib().orc_csr_from_arrays(self.nrows, self.ncols, self.row_ptrs, self.col_ind, self.values)
        try:
            y = np.zeros(max(self.nrows, len(x)))
            lib().orc_csr_matvec(h, x, len(x), y)
            return y
        finally:
            lib().orc_csr_free(h)


# ---- element kernels and assembly -----------------------------------------------

def poisson_element_matrix(mesh, eid, k, quad_order):
    n = mesh.npe
    out = np.zeros(n * n)
    if lib().orc_poisson_element_matrix(mesh.h, eid, k, quad_order, out):
        raise OracleError("poisson_element_matrix failed")
    return out.reshape(n, n)


def elasticity_element_matrix(mesh, eid, model, young, nu, quad_order):
    dim = DIM_OF_CELL[mesh.cell]
    n = mesh.npe * dim
    out = np.zeros(n * n)
    if lib().orc_elasticity_element_matrix(mesh.h, eid, model, young, nu, quad_order, out):
        raise OracleError("elasticity model/dimension mismatch")
    return out.reshape(n, n)


def assemble_poisson(mesh, k, quad_order):
    k = np.atleast_1d(np.asarray(k, dtype=np.float64)).copy()
    per = 1 if (len(k) == mesh.n_elems and len(k) > 1) else 0
    h = lib().orc_assemble_poisson(mesh.h, k, per, quad_order)
    if not h:
        raise OracleError(_err())
    return Coo(h)


def assemble_elasticity(mesh, model, young, nu, quad_order):
    E = np.atleast_1d(np.asarray(young, dtype=np.float64)).copy()
    per = 1 if (len(E) == mesh.n_elems and len(E) > 1) else 0
    h = lib().orc_assemble_elasticity(mesh.h, model, E, per, nu, quad_order)
    if not h:
        raise OracleError(_err())
    return Coo(h)


def csr_rows(mesh, kind, coef, rows, model=MODEL_3D, nu=0.3, quad_order=2):
    """Rows `rows` of Coo::to_csr(assemble(...)) (sparse:122-175 over
    assembly:428-480) without the whole COO: kind "poisson" (coef = k) or
    "elasticity" (coef = E).  Returns (ptr, cols, vals) with row k of the
    sample in cols[ptr[k]:ptr[k+1]]."""
    c = np.atleast_1d(np.asarray(coef, dtype=np.float64)).copy()
    per = 1 if (len(c) == mesh.n_elems and len(c) > 1) else 0
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    h = lib().orc_csr_rows(mesh.h, 0 if kind == "poisson" else 1, model, c, per, float(nu), quad_order, rows,
                           len(rows))
    if not h:
        raise OracleError(_err())
    try:
        nnz = lib().orc_rows_nnz(h)
        ptr = np.zeros(len(rows) + 1, np.int64)
        cols = np.zeros(nnz, np.int64)
        vals = np.zeros(nnz)
        lib().orc_rows_copy(h, ptr, cols, vals)
        return ptr, cols, vals
    finally:
        lib().orc_rows_free(h)


def load_poisson_rows(mesh, source, nodes, quad_order=2):
    """Entries `nodes` of the constant-source Poisson load (thermal:224-230)."""
    nodes = np.ascontiguousarray(nodes, dtype=np.int64)
    out = np.zeros(len(nodes))
    if lib().orc_load_poisson_rows(mesh.h, float(source), quad_order, nodes, len(nodes), out):
        raise OracleError(_err())
    return out


def reduced_rows(ptr, cols, vals, rhs_rows, bcs, free_index):
    """reduce_system (assembly/src/lib.rs:504-535) restricted to the free rows
    whose full CSR rows are given (ptr/cols/vals as csr_rows returns them, and
    their right-hand-side entries rhs_rows).  For each row: fred = rhs minus
    v * value of every fixed column, value from the FIRST bcs entry of that
    column (assembly:525), subtracted in column order; the free columns keep
    their values under the reduced numbering free_index[col] (ascending, so
    the later to_csr keeps their order and has no duplicates to sum).
    Returns (ptr, cols, vals, fred)."""
    first = {}
    for d, v in bcs:
        first.setdefault(int(d), float(v))
    optr, ocols, ovals, fred = [0], [], [], []
    for k in range(len(ptr) - 1):
        r = float(rhs_rows[k])
        for c, v in zip(cols[ptr[k]:ptr[k + 1]], vals[ptr[k]:ptr[k + 1]]):
            c = int(c)
            if c in first:
                r -= float(v) * first[c]
            else:
                ocols.append(int(free_index[c]))
                ovals.append(float(v))
        optr.append(len(ocols))
        fred.append(r)
    return (np.asarray(optr, np.int64), np.asarray(ocols, np.int64), np.asarray(ovals, np.float64),
            np.asarray(fred, np.float64))


def assemble_given(mesh, dpn, mats):
    mats = np.ascontiguousarray(mats, dtype=np.float64)
    return Coo(lib().orc_assemble_given(mesh.h, dpn, mats))


def load_poisson_source(mesh, source, quad_order):
    rhs = np.zeros(mesh.n_nodes)
    if callable(source):
        def cb(xp, dim, _ud):
            return float(source(*[xp[i] for i in range(dim)]))
        ccb = SOURCE_CB(cb)
        rc = lib().orc_load_poisson_source_cb(mesh.h, ccb, None, quad_order, rhs)
    else:
        rc = lib().orc_load_poisson_source(mesh.h, float(source), quad_order, rhs)
    if rc:
        raise OracleError("bad quadrature order")
    return rhs


def load_body(mesh, body, quad_order):
    """Body-force load loop of solve_elasticity (elasticity:371-379); body is a
    constant vector or a callable body(*x) -> sequence of dim values, called
    with the point's coordinates as arguments (like the source callbacks)."""
    dim = DIM_OF_CELL[mesh.cell]
    rhs = np.zeros(mesh.n_nodes * dim)
    if callable(body):
        def cb(xp, cdim, out, _ud):
            v = body(*[xp[i] for i in range(cdim)])
            for a in range(dim):
                out[a] = float(v[a])
        rc = lib().orc_load_body_cb(mesh.h, BODY_CB(cb), None, quad_order, rhs)
    else:
        rc = lib().orc_load_body(mesh.h, np.ascontiguousarray(body, dtype=np.float64), quad_order, rhs)
    if rc:
        raise OracleError("bad quadrature order")
    return rhs


def apply_neumann(mesh, dpn, flux, rhs, order=2, comp_mask=0xFFFFFFFF):
    """apply_neumann_order (assembly/src/lib.rs:601-667); flux(x, n) -> float."""
    def cb(xp, nrm, dim, _ud):
        return float(flux([xp[i] for i in range(dim)], [nrm[i] for i in range(dim)]))
    ccb = FLUX_CB(cb)
    lib().orc_apply_neumann_cb(mesh.h, dpn, ccb, None, order, comp_mask, rhs)
    return rhs


def apply_traction(mesh, dpn, axis, sign, value, comp_mask, rhs):
    lib().orc_apply_traction(mesh.h, dpn, axis, sign, value, comp_mask, rhs)
    return rhs


def apply_robin(coo, mesh, dpn, coeff, order=2):
    """apply_robin_order (assembly/src/lib.rs:684-753) onto `coo`; coeff(x, n) -> float."""
    def cb(xp, nrm, dim, _ud):
        return float(coeff([xp[i] for i in range(dim)], [nrm[i] for i in range(dim)]))
    ccb = FLUX_CB(cb)
    lib().orc_apply_robin_cb(coo.h, mesh.h, dpn, ccb, None, order)
    return coo


def apply_robin_selected(coo, mesh, dpn, axis, sign, h):
    """apply_robin with h on the faces whose outward normal n has sign*n[axis] > 0.5
    (axis < 0: every boundary face), zero elsewhere."""
    lib().orc_apply_robin(coo.h, mesh.h, dpn, axis, sign, h)
    return coo


def boundary_face_count(mesh):
    return lib().orc_boundary_face_count(mesh.h)


def _bcs(bcs):
    if len(bcs) == 0:
        return np.zeros(0, np.int64), np.zeros(0)
    dof = np.ascontiguousarray([int(b[0]) for b in bcs], dtype=np.int64)
    val = np.ascontiguousarray([float(b[1]) for b in bcs], dtype=np.float64)
    return dof, val


def reduce_system(coo, rhs, bcs):
    """reduce_system (assembly/src/lib.rs:504-535) -> (kred Coo, fred, free)."""
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    dof, val = _bcs(bcs)
    h = lib().orc_reduce_system(coo.h, rhs, len(rhs), dof, val, len(dof))
    try:
        nf = lib().orc_reduced_nfree(h)
        fred = np.zeros(nf); free = np.zeros(nf, np.int64)
        lib().orc_reduced_copy(h, fred, free)
        kred = Coo(lib().orc_reduced_kred(h))
        return kred, fred, free
    finally:
        lib().orc_reduced_free(h)


def solve(coo, rhs):
    """solve (sparse/src/lib.rs:225-278) with a partial-pivot dense LU."""
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.zeros(len(rhs))
    if lib().orc_solve(coo.h, rhs, len(rhs), x):
        raise OracleError(_err())
    return x


def solve_with_dirichlet(coo, rhs, bcs):
    """solve_with_dirichlet (assembly/src/lib.rs:543-559)."""
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    dof, val = _bcs(bcs)
    u = np.zeros(len(rhs))
    if lib().orc_solve_with_dirichlet(coo.h, rhs, len(rhs), dof, val, len(dof), u):
        raise OracleError(_err())
    return u


def pcg_jacobi(csr, b, tol=1e-10, max_it=100000, nthreads=0):
    """CPU FP64 Jacobi-PCG (not reference code; see oracle.cpp), stopping on
    the true relative residual.

    Returns (x, iterations, true relative residual); iterations < 0 means
    max_it was reached first.
    """
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(csr.nrows)
    rel = C.c_double()
    it = lib().orc_pcg_jacobi(csr.nrows, csr.row_ptrs, csr.col_ind, csr.values, b, x, tol, max_it, nthreads,
                              C.byref(rel))
    return x, int(it), rel.value


def pcg_jacobi_i32(n, row_ptrs, col_ind, values, b, tol=1e-10, max_it=100000, nthreads=0):
    """pcg_jacobi on int32 CSR arrays (12 bytes per stored entry).
    Returns (x, iterations, true relative residual)."""
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n)
    rel = C.c_double()
    it = lib().orc_pcg_jacobi_i32(n, np.ascontiguousarray(row_ptrs, dtype=np.int32),
                                  np.ascontiguousarray(col_ind, dtype=np.int32),
                                  np.ascontiguousarray(values, dtype=np.float64), b, x, tol, max_it, nthreads,
                                  C.byref(rel))
    return x, int(it), rel.value


def map_at(cell, X, xi):
    """Map::from_nodes_and_grad (element/src/lib.rs:702-724) -> (jac, signed det, inv)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    rd = DIM_OF_CELL[cell]
    jac = np.zeros(rd * rd); inv = np.zeros(rd * rd); det = C.c_double()
    lib().orc_map(cell, X, X.shape[0], X.shape[1], np.ascontiguousarray(xi, dtype=np.float64), jac, C.byref(det), inv)
    return jac.reshape(rd, rd), det.value, inv.reshape(rd, rd)


def cell_quad(cell, order):
    rd = DIM_OF_CELL[cell]
    pts = np.zeros((64, rd)); w = np.zeros(64)
    nq = lib().orc_cell_quad(cell, order, pts, w)
    return pts[:nq].copy(), w[:nq].copy()


def node_block_lower_pattern(csr, free, dpn):
    """Strictly-lower node-block pattern of a reduced matrix (not reference code).

    Row i may use every free dof j < i of every mesh node coupled in `csr` to
    the node of i (nodes = full dof // dpn; `free` maps reduced -> full dof).
    Returns (row_ptrs, col_ind) int64.
    """
    n = csr.nrows
    node = np.asarray(free) // dpn
    red = {int(g): i for i, g in enumerate(free)}
    rows = []
    i = 0
    while i < n:
        g1 = i
        while g1 < n and node[g1] == node[i]:
            g1 += 1
        nodes = set()
        for g in range(i, g1):
            nodes |= set(int(v) for v in node[csr.col_ind[csr.row_ptrs[g]:csr.row_ptrs[g + 1]]])
        cand = sorted(red[m * dpn + c] for m in nodes for c in range(dpn) if (m * dpn + c) in red)
        for g in range(i, g1):
            rows.append([j for j in cand if j < g])
        i = g1
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    ci = np.array([j for r in rows for j in r], dtype=np.int64)
    return rp, ci


def fsai(csr, pattern=None):
    """Classic FSAI factor G (CSR incl. diagonal) of an SPD CSR matrix (not reference code).

    pattern: optional (row_ptrs, col_ind) of the strictly-lower pattern; default tril(A).
    """
    if pattern is None:
        h = lib().orc_fsai(csr.nrows, csr.row_ptrs, csr.col_ind, csr.values, None, None)
    else:
        lrp = np.ascontiguousarray(pattern[0], dtype=np.int64)
        lci = np.ascontiguousarray(pattern[1], dtype=np.int64)
        h = lib().orc_fsai(csr.nrows, csr.row_ptrs, csr.col_ind, csr.values, lrp.ctypes.data_as(C.c_void_p),
                           lci.ctypes.data_as(C.c_void_p))
    if not h:
        raise OracleError(_err())
    try:
        return Csr._from_handle(h)
    finally:
        lib().orc_csr_free(h)


def max_threads():
    return lib().orc_max_threads()


# ---- topology optimisation (crates/tpt-fem-topopt/src/lib.rs) ----------------

TOPO_E_MIN_FACTOR = 1e-3  # topopt:54


def topopt_ke0(nu, h):
    """element_stiffness_unit (topopt:166-217) -> 8x8."""
    out = np.zeros(64)
    lib().orc_topopt_ke0(float(nu), float(h), out)
    return out.reshape(8, 8)


def topopt_filter_sensitivity(nelx, nely, h, raw, radius):
    """filter_sensitivity (topopt:259-279) on Grid::new(nelx + 1, nely + 1, h)."""
    raw = np.ascontiguousarray(raw, dtype=np.float64)
    out = np.zeros(nelx * nely)
    lib().orc_topopt_filter_sensitivity(nelx, nely, float(h), raw, float(radius), out)
    return out


def topopt_oc_update(rho, sens, vol_frac, move_limit):
    """oc_update (topopt:284-331)."""
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    sens = np.ascontiguousarray(sens, dtype=np.float64)
    out = np.zeros(len(rho))
    lib().orc_topopt_oc_update(len(rho), rho, sens, float(vol_frac), float(move_limit), out)
    return out


def cantilever_load(nelx, nely, load=1.0, node=None):
    """cantilever_load (topopt:398-415): left edge clamped, -y point load at the
    bottom-right node (or at `node`) of Grid::new(nelx + 1, nely + 1, h)."""
    nx, ny = nelx + 1, nely + 1
    f = np.zeros(2 * nx * ny)
    bcs = []
    for j in range(ny):
        n = j * nx
        bcs += [(2 * n, 0.0), (2 * n + 1, 0.0)]
    f[2 * (nx - 1 if node is None else node) + 1] = -load
    return f, bcs


def topopt(nelx, nely, vol_frac, radius, max_iter, f, bcs, h=1.0, e0=1.0, nu=0.3, penal=3.0, move_limit=0.2,
           emin=None, density_filter=False, banded=None):
    """topopt_simp (topopt:342-385) -> (compliance history (max_iter + 1), final densities).

    density_filter=True: the density filter / OC loop of the published 88-line
    SIMP code (not in the reference).  banded: solve by banded Cholesky instead
    of the reference's dense LU (default: banded above 1000 dofs)."""
    if emin is None:
        emin = TOPO_E_MIN_FACTOR * e0
    ndof = 2 * (nelx + 1) * (nely + 1)
    if banded is None:
        banded = ndof > 1000
    f = np.ascontiguousarray(f, dtype=np.float64)
    assert len(f) == ndof
    dof, val = _bcs(bcs)
    comp = np.zeros(max_iter + 1)
    rho = np.zeros(nelx * nely)
    if lib().orc_topopt(nelx, nely, h, e0, nu, vol_frac, penal, radius, move_limit, emin, max_iter,
                        int(density_filter), int(banded), f, dof, val, len(dof), comp, rho):
        raise OracleError(_err())
    return comp, rho
