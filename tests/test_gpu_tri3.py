"""Tri3 (P1 triangle) meshes on the device path: Poisson and plane
elasticity matrices, loads and tractions bit-exact against the oracle's
restatement of the reference (thermal:29-196, elasticity:197-348,
assembly:46-59 and 563-667, quadrature:223-234), plus the reference's own
Tri3 known-answer tests (thermal:344 poisson_2d_linear_is_exact,
elasticity:742 plane_stress_patch_test) through the public API."""
import numpy as np
import pytest

import tpt_fem as F
from meshes import jitter, tri_grid
from oracle import oracle as O
from test_gpu_parity import assert_csr_equal

pytestmark = pytest.mark.gpu

CROSS_COORDS = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0], [0.5, 0.5]])
CROSS_CONN = np.array([[0, 1, 4], [1, 3, 4], [3, 2, 4], [2, 0, 4]])


def test_tri3_mesh_round_trip(ctx):
    c, e = tri_grid(4, 3)
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    m._coords = m._conn = None
    assert m.n_elems == 24 and m.dim == 2
    assert np.array_equal(m.conn_array, e) and np.array_equal(m.coords_array, c)


@pytest.mark.parametrize("seed", [0, 1])
def test_poisson_tri3_per_element_k(ctx, seed):
    c, e = tri_grid(7, 5, 2.0, 1.0)
    c = jitter(c, 0.05, seed)
    k = np.exp(np.random.default_rng(seed + 20).normal(size=len(e)))
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    K = F.assemble_poisson(m, k, 2)
    assert_csr_equal(K, O.assemble_poisson(O.Mesh(O.CELL_TRI, c, e), k, 2))


@pytest.mark.parametrize("model,omodel", [("plane-stress", O.MODEL_PLANE_STRESS),
                                          ("plane-strain", O.MODEL_PLANE_STRAIN)])
def test_elasticity_tri3(ctx, model, omodel):
    c, e = tri_grid(6, 4, 3.0, 1.0)
    c = jitter(c, 0.06, 5)
    E = np.linspace(1.0, 3.0, len(e))
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, model, E, 0.3, 2)
    assert_csr_equal(K, O.assemble_elasticity(O.Mesh(O.CELL_TRI, c, e), omodel, E, 0.3, 2))


def test_tri3_rejects_the_3d_model(ctx):
    c, e = tri_grid(2, 2)
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    with pytest.raises(F.TptFemError) as ex:
        F.assemble_elasticity(m, "3d", 1.0, 0.3, 2)
    assert ex.value.name == "MODEL_DIM_MISMATCH"


def test_tri3_loads_bit_exact(ctx):
    c, e = tri_grid(5, 4)
    c = jitter(c, 0.05, 8)
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    om = O.Mesh(O.CELL_TRI, c, e)
    assert np.array_equal(F.load_poisson_source(m, 1.3, 2), O.load_poisson_source(om, 1.3, 2))
    b = [0.25, -9.81]
    assert np.array_equal(F.load_body(m, b, 2), O.load_body(om, b, 2))


@pytest.mark.parametrize("axis,sign", [(0, 1.0), (1, -1.0)])
def test_tri3_traction_bit_exact(ctx, axis, sign):
    c, e = tri_grid(5, 3, 2.0, 1.0)
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    t = np.array([0.4, -1e-3])
    rhs0 = np.random.default_rng(4).normal(size=2 * len(c))
    got = F.apply_traction(m, 2, axis, sign, t, rhs0.copy())
    om = O.Mesh(O.CELL_TRI, c, e)
    want = rhs0.copy()
    for comp in range(2):
        O.apply_traction(om, 2, axis, sign, t[comp], 1 << comp, want)
    assert np.array_equal(got, want)


def test_tri3_traction_total_is_edge_length_times_t(ctx):
    c, e = tri_grid(8, 4, 2.0, 1.0)
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    rhs = F.apply_traction(m, 2, 0, 1.0, [0.0, -2e-3], np.zeros(2 * len(c)))
    assert abs(rhs[1::2].sum() - (-2e-3 * 1.0)) < 1e-15 and not rhs[0::2].any()


def test_poisson_2d_linear_is_exact(ctx):  # thermal:344
    m = F.Mesh.from_arrays(F.CELL_TRI3, CROSS_COORDS, CROSS_CONN, ctx=ctx)
    res = F.solve_poisson(m, 1.0, 2, 0.0, [(0, 0.0), (1, 1.0), (2, 1.0), (3, 2.0)], tol=1e-14)
    u = np.array(res.values)
    assert abs(u[4] - 1.0) < 1e-10 and abs(u[0]) < 1e-12 and abs(u[3] - 2.0) < 1e-12


def test_plane_stress_patch_test(ctx):  # elasticity:742
    m = F.Mesh.from_arrays(F.CELL_TRI3, CROSS_COORDS, CROSS_CONN, ctx=ctx)
    bcs = []
    for node, x, y in [(0, 0.0, 0.0), (1, 0.1, 0.0), (2, 0.0, 0.2), (3, 0.1, 0.2)]:
        bcs += [(node, 0, x), (node, 1, y)]
    u = F.solve_elasticity(m, "plane-stress", 1.0, 0.3, 2, bcs, tol=1e-14).to_numpy()
    assert abs(u[4, 0] - 0.05) < 1e-9 and abs(u[4, 1] - 0.1) < 1e-9


def test_tri3_linear_fields_on_a_distorted_mesh(ctx):
    c, e = tri_grid(6, 5)
    c = jitter(c, 0.05, 14)
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    bnd = [i for i in range(len(c)) if min(c[i][0], c[i][1]) < 1e-12 or max(c[i][0], c[i][1]) > 1 - 1e-12]
    res = F.solve_poisson(m, 1.0, 2, 0.0, [(i, c[i][0] + c[i][1]) for i in bnd], tol=1e-14)
    assert np.max(np.abs(np.array(res.values) - (c[:, 0] + c[:, 1]))) < 1e-12
    bcs = [(i, 0, 0.1 * c[i][0]) for i in bnd] + [(i, 1, 0.2 * c[i][1]) for i in bnd]
    u = F.solve_elasticity(m, "plane-strain", 1.0, 0.3, 2, bcs, tol=1e-14).to_numpy()
    assert np.max(np.abs(u[:, 0] - 0.1 * c[:, 0])) < 1e-12
    assert np.max(np.abs(u[:, 1] - 0.2 * c[:, 1])) < 1e-12


def test_tri3_solution_matches_oracle_dense_solve(ctx):
    c, e = tri_grid(6, 4, 2.0, 1.0)
    c = jitter(c, 0.04, 2)
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    om = O.Mesh(O.CELL_TRI, c, e)
    left = [int(i) for i in O.nodes_on_plane(c, 0, 0.0, 1e-9)]
    bcs = [(2 * n + k, 0.0) for n in left for k in range(2)]
    E = np.linspace(0.5, 2.0, len(e))
    K = F.assemble_elasticity(m, "plane-stress", E, 0.3, 2)
    rhs = F.apply_traction(m, 2, 0, 1.0, [0.0, -1e-3], np.zeros(K.nrows))
    u, st = F.solve_with_dirichlet(K, rhs, bcs, tol=1e-13)
    coo = O.assemble_elasticity(om, O.MODEL_PLANE_STRESS, E, 0.3, 2)
    u_ref = O.solve_with_dirichlet(coo, rhs, bcs)
    assert np.max(np.abs(u - u_ref)) <= 1e-10 * np.max(np.abs(u_ref))
