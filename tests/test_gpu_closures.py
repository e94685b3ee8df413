"""Caller-evaluated sources and fluxes -- the reference's closures across the C ABI.

solve_poisson (crates/tpt-fem-thermal/src/lib.rs:206-240) takes the source f(x)
and the optional Neumann flux g(x, n) and Robin coefficient h(x, n) as
closures; solve_elasticity (crates/tpt-fem-elasticity/src/lib.rs:355-381) the
body force b(x).  The library reports the points where the reference would
call them, takes the values there, and must then match the oracle -- which
calls the same Python functions from the reference's own loops -- bit for bit
for loads and matrices, and to 1e-12 of the oracle's dense LU for solutions.
The C-function entry points (tptfem_solve_poisson_fn / _elasticity_fn) must
give the same bits as the per-point route.
"""
import ctypes as C
import math

import numpy as np
import pytest

import tpt_fem as F
from tpt_fem import _native as N
from meshes import box, jitter, quad_grid, tri_grid
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def src(x, y, z=0.0):
    return 1.0 + math.sin(3.0 * x) * y - 0.5 * z * z


def body3(x, y, z=0.0):
    return [0.1 * y, -1.0 + x * z, math.cos(x + y)]


def body2(x, y, z=0.0):
    return [0.1 * y, -1.0 + x * x]


def flux(x, n):
    # depends on the point and on the outward normal
    return 2.0 * x[0] - x[1] + 0.25 * n[0] + (n[1] if len(n) > 1 else 0.0)


def robin_h(x, n):
    return 0.5 + x[0] * x[1] + (0.3 if n[0] > 0.5 else 0.0)


MESHES = {
    "tet4": (O.CELL_TET, F.CELL_TET4, lambda: (lambda ce: (jitter(ce[0], 0.05, 5), ce[1]))(box([4, 3, 3]))),
    "quad4": (O.CELL_QUAD, F.CELL_QUAD4, lambda: quad_grid(5, 3, 2.0, 1.0)),
    "tri3": (O.CELL_TRI, F.CELL_TRI3, lambda: tri_grid(4, 4)),
}


def meshes(ctx, name):
    ocell, fcell, make = MESHES[name]
    c, e = make()
    return O.Mesh(ocell, c, e), F.Mesh.from_arrays(fcell, c, e, ctx=ctx), c


@pytest.mark.parametrize("name", list(MESHES))
def test_source_load_at_quadrature_points_is_bit_exact(ctx, name):
    om, m, _ = meshes(ctx, name)
    for order in ((1, 2, 3) if name == "quad4" else (2,)):
        assert np.array_equal(F.load_poisson_source(m, src, order), O.load_poisson_source(om, src, order))
    pts = F.quadrature_points(m, 2)
    assert pts.shape[0] == m.n_elems and pts.shape[2] == m.cdim


@pytest.mark.parametrize("name", list(MESHES))
def test_body_force_closure_load_is_bit_exact(ctx, name):
    om, m, _ = meshes(ctx, name)
    b = body3 if name == "tet4" else body2
    assert np.array_equal(F.load_body(m, b, 2), O.load_body(om, b, 2))


@pytest.mark.parametrize("name", list(MESHES))
def test_general_neumann_flux_is_bit_exact(ctx, name):
    om, m, _ = meshes(ctx, name)
    for dpn, mask in ((1, 0xFFFFFFFF), (3 if name == "tet4" else 2, 0xFFFFFFFF), (2, 0b10)):
        start = np.random.default_rng(dpn).standard_normal(m.n_nodes * dpn)
        got = F.apply_neumann(m, dpn, flux, start.copy(), comp_mask=mask)
        ref = O.apply_neumann(om, dpn, flux, start.copy(), comp_mask=mask)
        assert np.array_equal(got, ref)
    x, nrm = F.boundary_points(m)
    assert np.allclose(np.linalg.norm(nrm, axis=1), 1.0, atol=1e-15)


@pytest.mark.parametrize("name", list(MESHES))
def test_robin_closure_matrix_is_bit_exact(ctx, name):
    om, m, c = meshes(ctx, name)
    k = np.random.default_rng(7).uniform(0.5, 2.0, size=om.n_elems)
    K = F.assemble_poisson(m, k, 2, robin=robin_h)
    ref = O.apply_robin(O.assemble_poisson(om, k, 2), om, 1, robin_h).to_csr()
    rp, ci, va = K.to_csr()
    assert np.array_equal(rp, ref.row_ptrs) and np.array_equal(ci, ref.col_ind) and np.array_equal(va, ref.values)


@pytest.mark.parametrize("name", list(MESHES))
def test_solve_poisson_with_every_closure_matches_dense_lu(ctx, name):
    om, m, c = meshes(ctx, name)
    left = [(int(i), 0.1 * float(c[i, 1])) for i in O.nodes_on_plane(c, 0, 0.0, 1e-9)]
    sol = F.solve_poisson(m, 1.5, 2, src, left, neumann=flux, robin=robin_h, tol=1e-14)
    coo = O.apply_robin(O.assemble_poisson(om, 1.5, 2), om, 1, robin_h)
    rhs = O.apply_neumann(om, 1, flux, O.load_poisson_source(om, src, 2))
    u_ref = O.solve_with_dirichlet(coo, rhs, left)
    u = sol.to_numpy()
    assert np.max(np.abs(u - u_ref)) <= 1e-12 * np.max(np.abs(u_ref))


def _c_solve_poisson(ctx, m, k, order, source, bcs, neumann=None, robin=None):
    calls = {"n": 0}

    def s_cb(x, dim, _u):
        calls["n"] += 1
        return source(*[x[i] for i in range(dim)])

    def f_cb(fn):
        def cb(x, n, dim, _u):
            return fn([x[i] for i in range(dim)], [n[i] for i in range(dim)])
        return N.FLUX_FN(cb)

    sf = N.SOURCE_FN(s_cb)
    nf = f_cb(neumann) if neumann else N.FLUX_FN()
    rf = f_cb(robin) if robin else N.FLUX_FN()
    dof = np.array([d for d, _ in bcs], np.int64)
    val = np.array([v for _, v in bcs], np.float64)
    u = np.zeros(m.n_nodes)
    o = F._opts(tol=1e-14)
    st = N.SolveStats()
    ctx.check(ctx.lib.tptfem_solve_poisson_fn(ctx.h, m.h, k, order, sf, None, N.ptr(dof), N.ptr(val), len(dof),
                                              nf, None, rf, None, C.byref(o), N.ptr(u), C.byref(st)))
    return u, calls["n"]


@pytest.mark.parametrize("name", ["tet4", "quad4"])
def test_c_function_entry_points_match_the_point_route(ctx, name):
    om, m, c = meshes(ctx, name)
    left = [(int(i), 0.0) for i in O.nodes_on_plane(c, 0, 0.0, 1e-9)]
    py = F.solve_poisson(m, 1.5, 2, src, left, neumann=flux, robin=robin_h, tol=1e-14).to_numpy()
    u, calls = _c_solve_poisson(ctx, m, 1.5, 2, src, left, neumann=flux, robin=robin_h)
    assert np.array_equal(u, py)
    assert calls == F.quadrature_points(m, 2).shape[0] * F.quadrature_points(m, 2).shape[1]
    # without the optional closures: the plain constant-free source path
    u2, _ = _c_solve_poisson(ctx, m, 1.5, 2, src, left)
    py2 = F.solve_poisson(m, 1.5, 2, src, left, tol=1e-14).to_numpy()
    assert np.array_equal(u2, py2)


def test_c_body_function_matches_the_point_route(ctx):
    om, m, c = meshes(ctx, "tet4")
    clamp = [(int(i), k, 0.0) for i in O.nodes_on_plane(c, 0, 0.0, 1e-9) for k in range(3)]
    py = F.solve_elasticity(m, "3d", 2.0, 0.3, 2, clamp, body=body3, tol=1e-14).to_numpy().reshape(-1)

    def b_cb(x, dim, out, _u):
        v = body3(*[x[i] for i in range(dim)])
        for a in range(3):
            out[a] = v[a]

    bf = N.BODY_FN(b_cb)
    dof = np.array([3 * n + k for n, k, _ in clamp], np.int64)
    val = np.zeros(len(dof))
    u = np.zeros(3 * m.n_nodes)
    o = F._opts(tol=1e-14)
    st = N.SolveStats()
    ctx.check(ctx.lib.tptfem_solve_elasticity_fn(ctx.h, m.h, F.MODEL_CONTINUUM_3D, 2.0, 0.3, 2, bf, None, N.ptr(dof),
                                                 N.ptr(val), len(dof), C.byref(o), N.ptr(u), C.byref(st)))
    assert np.array_equal(u, py)
    coo = O.assemble_elasticity(om, O.MODEL_3D, 2.0, 0.3, 2)
    u_ref = O.solve_with_dirichlet(coo, O.load_body(om, body3, 2), [(3 * n + k, 0.0) for n, k, _ in clamp])
    assert np.max(np.abs(u - u_ref)) <= 1e-12 * np.max(np.abs(u_ref))


def test_non_finite_closure_values_are_rejected(ctx):
    _, m, c = meshes(ctx, "tri3")
    with pytest.raises(F.TptFemError):
        F.load_poisson_source(m, lambda x, y, z=0.0: float("nan"), 2)
    with pytest.raises(F.TptFemError):
        F.apply_neumann(m, 1, lambda x, n: float("inf"), np.zeros(m.n_nodes))
