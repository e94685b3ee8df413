"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Pattern and values are compared BIT-EXACTLY (integer/index work and the
reference's FP64 operation order reproduced without FMA); solutions against
the oracle's dense LU to 1e-12 relative.
"""
import numpy as np
import pytest

import tpt_fem as F
from meshes import box, jitter, quad_grid, unit_cube_bcs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def oracle_csr(coo):
    c = coo.to_csr()
    return c.nrows, c.ncols, c.row_ptrs, c.col_ind, c.values


def assert_csr_equal(mat, coo):
    nr, nc, rp, ci, va = oracle_csr(coo)
    grp, gci, gva = mat.to_csr()
    assert (mat.nrows, mat.ncols, mat.nnz) == (nr, nc, len(va))
    assert np.array_equal(grp, rp)
    assert np.array_equal(gci, ci)
    assert np.array_equal(gva, va), f"max |diff| {np.max(np.abs(gva - va))}"


# ---- meshes --------------------------------------------------------------------

@pytest.mark.parametrize("n", [[1, 1, 1], [4, 4, 4], [3, 5, 2], [8, 8, 8]])
def test_device_box_mesh_bit_exact(ctx, n):
    m = F.Mesh.box_mesh([0, 0, 0], [1, 1, 1], n, ctx=ctx)
    c, e = box(n)
    assert np.array_equal(m.coords_array, c)
    assert np.array_equal(m.conn_array, e)


def test_device_box_mesh_offset_box(ctx):
    m = F.Mesh.box_mesh([0, 0, 0], [4, 1, 1], [20, 5, 5], ctx=ctx)
    c, e = box([20, 5, 5], mx=(4.0, 1.0, 1.0))
    assert np.array_equal(m.coords_array, c) and np.array_equal(m.conn_array, e)


# ---- Poisson assembly ---------------------------------------------------------------

def test_poisson_box8_pattern_and_values(ctx):
    c, e = box([8, 8, 8])
    m = F.Mesh.box_mesh([0, 0, 0], [1, 1, 1], [8, 8, 8], ctx=ctx)
    K = F.assemble_poisson(m, 1.0, 2)
    assert K.nnz == 4617
    assert_csr_equal(K, O.assemble_poisson(O.Mesh(O.CELL_TET, c, e), 1.0, 2))


@pytest.mark.parametrize("seed", [0, 1])
def test_poisson_jittered_tets_per_element_k(ctx, seed):
    c, e = box([5, 4, 6])
    c = jitter(c, 0.04, seed)
    k = np.exp(np.random.default_rng(seed + 10).normal(size=len(e)))
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_poisson(m, k, 2)
    assert_csr_equal(K, O.assemble_poisson(O.Mesh(O.CELL_TET, c, e), k, 2))


@pytest.mark.parametrize("order", [1, 2, 3])
def test_poisson_quad4(ctx, order):
    c, e = quad_grid(7, 5, 2.0, 1.0)
    c = jitter(c, 0.05, 3)
    k = np.linspace(0.5, 2.0, len(e))
    m = F.Mesh.from_arrays(F.CELL_QUAD4, c, e, ctx=ctx)
    K = F.assemble_poisson(m, k, order)
    assert_csr_equal(K, O.assemble_poisson(O.Mesh(O.CELL_QUAD, c, e), k, order))


# ---- elasticity assembly --------------------------------------------------------------

def test_elasticity_tets_box(ctx):
    c, e = box([4, 3, 3])
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", 1.0, 0.3, 2)
    assert_csr_equal(K, O.assemble_elasticity(O.Mesh(O.CELL_TET, c, e), O.MODEL_3D, 1.0, 0.3, 2))
    assert np.diff(K.to_csr()[0]).max() <= 37


def test_elasticity_jittered_tets_per_element_E(ctx):
    c, e = box([4, 4, 3])
    c = jitter(c, 0.05, 7)
    E = 1e-3 + (1 - 1e-3) * np.random.default_rng(8).uniform(size=len(e)) ** 3
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", E, 0.3, 2)
    assert_csr_equal(K, O.assemble_elasticity(O.Mesh(O.CELL_TET, c, e), O.MODEL_3D, E, 0.3, 2))


@pytest.mark.parametrize("model,omodel", [("plane-stress", O.MODEL_PLANE_STRESS),
                                          ("plane-strain", O.MODEL_PLANE_STRAIN)])
def test_elasticity_quad4(ctx, model, omodel):
    c, e = quad_grid(6, 4, 3.0, 1.0)
    c = jitter(c, 0.06, 4)
    E = np.linspace(1.0, 3.0, len(e))
    m = F.Mesh.from_arrays(F.CELL_QUAD4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, model, E, 0.3, 2)
    assert_csr_equal(K, O.assemble_elasticity(O.Mesh(O.CELL_QUAD, c, e), omodel, E, 0.3, 2))


def test_reassemble_equals_fresh_assembly(ctx):
    c, e = box([4, 4, 4])
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    rng = np.random.default_rng(5)
    K = F.assemble_elasticity(m, "3d", rng.uniform(0.1, 1, len(e)), 0.3, 2)
    E2 = rng.uniform(0.1, 1, len(e))
    K.reassemble(E2)
    assert_csr_equal(K, O.assemble_elasticity(O.Mesh(O.CELL_TET, c, e), O.MODEL_3D, E2, 0.3, 2))


def test_reassemble_rebuilds_pattern_when_zeros_appear(ctx):
    # k = 0 on some elements removes their contributions; the pattern shrinks
    # exactly as the reference's zero-skip would.
    c, e = box([4, 4, 4])
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_poisson(m, np.ones(len(e)), 2)
    k2 = np.ones(len(e))
    k2[::3] = 0.0
    K.reassemble(k2)
    assert_csr_equal(K, O.assemble_poisson(O.Mesh(O.CELL_TET, c, e), k2, 2))


def test_matvec_bit_exact(ctx):
    c, e = box([5, 5, 5])
    c = jitter(c, 0.03, 2)
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", 1.0, 0.25, 2)
    x = np.random.default_rng(1).normal(size=K.ncols + 3)
    coo = O.assemble_elasticity(O.Mesh(O.CELL_TET, c, e), O.MODEL_3D, 1.0, 0.25, 2)
    assert np.array_equal(K.matvec(x), coo.to_csr().matvec(x))


# ---- loads ---------------------------------------------------------------------------

def test_poisson_source_load_bit_exact(ctx):
    c, e = box([5, 4, 3])
    c = jitter(c, 0.04, 9)
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    assert np.array_equal(F.load_poisson_source(m, 1.7, 2),
                          O.load_poisson_source(O.Mesh(O.CELL_TET, c, e), 1.7, 2))
    cq, eq = quad_grid(5, 3)
    cq = jitter(cq, 0.05, 1)
    mq = F.Mesh.from_arrays(F.CELL_QUAD4, cq, eq, ctx=ctx)
    assert np.array_equal(F.load_poisson_source(mq, -0.3, 3),
                          O.load_poisson_source(O.Mesh(O.CELL_QUAD, cq, eq), -0.3, 3))


def test_body_load_bit_exact(ctx):
    c, e = box([3, 4, 5])
    c = jitter(c, 0.04, 11)
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    b = [0.1, -0.2, 9.81]
    assert np.array_equal(F.load_body(m, b, 2), O.load_body(O.Mesh(O.CELL_TET, c, e), b, 2))


@pytest.mark.parametrize("axis,sign", [(0, 1.0), (2, -1.0)])
def test_traction_bit_exact(ctx, axis, sign):
    # Vector traction t on the faces whose outward normal is sign*e_axis,
    # expressed with the reference's scalar apply_neumann one component at a time.
    c, e = box([4, 3, 3], mx=(4.0, 1.0, 1.0))
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    t = np.array([0.3, 0.0, -1e-3])
    rng = np.random.default_rng(3)
    rhs0 = rng.normal(size=3 * len(c))
    got = F.apply_traction(m, 3, axis, sign, t, rhs0.copy())
    om = O.Mesh(O.CELL_TET, c, e)
    want = rhs0.copy()
    for comp in range(3):
        O.apply_traction(om, 3, axis, sign, t[comp], 1 << comp, want)
    assert np.array_equal(got, want)


def test_traction_total_equals_face_area_times_t(ctx):
    m = F.Mesh.box_mesh([0, 0, 0], [4, 1, 1], [8, 3, 3], ctx=ctx)
    rhs = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(3 * m.n_nodes))
    assert abs(rhs[2::3].sum() - (-1e-3 * 1.0)) < 1e-15


# ---- Dirichlet reduction and solve ------------------------------------------------------

def test_reduce_system_bit_exact(ctx):
    c, e = box([5, 4, 4])
    c = jitter(c, 0.03, 4)
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", 2.0, 0.3, 2)
    rhs = np.random.default_rng(2).normal(size=K.nrows)
    # clamp x=0 (dofs listed twice with different values: first wins for lifting,
    # last wins in the returned solution)
    x0 = [int(i) for i in O.nodes_on_plane(c, 0, 0.0, 1e-9)]
    bcs = [(3 * n + k, 0.01 * k) for n in x0 for k in range(3)] + [(3 * x0[0], 5.0)]
    S = F.reduce_system(K, rhs, bcs)
    rp, ci, va, fred, free = S.download()
    coo = O.assemble_elasticity(O.Mesh(O.CELL_TET, c, e), O.MODEL_3D, 2.0, 0.3, 2)
    kred, ofred, ofree = O.reduce_system(coo, rhs, bcs)
    kc = kred.to_csr()
    assert np.array_equal(free, ofree)
    assert np.array_equal(fred, ofred)
    assert np.array_equal(rp, kc.row_ptrs) and np.array_equal(ci, kc.col_ind) and np.array_equal(va, kc.values)


@pytest.mark.parametrize("solver", [F.SOLVER_JACOBI_PCG, F.SOLVER_MP_PCG, F.SOLVER_FSAI_MP_PCG])
def test_poisson_box8_solution_vs_dense_lu(ctx, solver):
    c, e = box([8, 8, 8])
    m = F.Mesh.box_mesh([0, 0, 0], [1, 1, 1], [8, 8, 8], ctx=ctx)
    bcs = unit_cube_bcs(c)
    res = F.solve_poisson(m, 1.0, 2, 1.0, bcs, solver=solver, tol=1e-14)
    om = O.Mesh(O.CELL_TET, c, e)
    u_ref = O.solve_with_dirichlet(O.assemble_poisson(om, 1.0, 2), O.load_poisson_source(om, 1.0, 2), bcs)
    u = np.array(res.values)
    assert np.max(np.abs(u - u_ref)) <= 1e-12 * np.max(np.abs(u_ref))
    assert res.stats["rel_residual"] <= 1e-14
    assert abs(u[364] - 0.05491766911624052) < 1e-12


def test_elasticity_solution_vs_dense_lu(ctx):
    c, e = box([4, 3, 3], mx=(2.0, 1.0, 1.0))
    c = jitter(c, 0.03, 6)
    E = np.random.default_rng(4).uniform(0.01, 1.0, len(e))
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", E, 0.3, 2)
    rhs = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    x0 = [int(i) for i in O.nodes_on_plane(c, 0, 0.0, 1e-9)]
    bcs = [(3 * n + k, 0.0) for n in x0 for k in range(3)]
    coo = O.assemble_elasticity(O.Mesh(O.CELL_TET, c, e), O.MODEL_3D, E, 0.3, 2)
    u_ref = O.solve_with_dirichlet(coo, rhs, bcs)
    for solver in (F.SOLVER_JACOBI_PCG, F.SOLVER_MP_PCG, F.SOLVER_FSAI_MP_PCG):
        u, st = F.solve_with_dirichlet(K, rhs, bcs, solver=solver, tol=1e-13)
        assert st["rel_residual"] <= 1e-13 and st["solver_used"] == solver and not st["fell_back"]
        assert np.max(np.abs(u - u_ref)) <= 1e-10 * np.max(np.abs(u_ref))


def _fsai_vs_oracle(S, dpn):
    lrp, lci, lva, s2 = S.fsai()
    rp, ci, va, fred, free = S.download()
    csr = O.Csr(S.n_free, S.n_free, rp, ci, va)
    prp, pci = O.node_block_lower_pattern(csr, free, dpn)
    assert np.array_equal(lrp, prp) and np.array_equal(lci, pci)
    G = O.fsai(csr, (prp, pci))
    diag = G.values[G.row_ptrs[1:] - 1]  # the diagonal closes each row
    assert np.allclose(s2, diag ** 2, rtol=2e-7, atol=0)
    off = np.concatenate([G.values[G.row_ptrs[i]:G.row_ptrs[i + 1] - 1] / diag[i] for i in range(S.n_free)])
    want = off.astype(np.float16).astype(np.float64)
    assert np.all(np.abs(lva - want) <= 1e-3 * np.abs(want) + 1e-7)


def test_fsai_factor_elasticity_matches_oracle(ctx):
    c, e = box([4, 3, 3], mx=(2.0, 1.0, 1.0))
    c = jitter(c, 0.03, 21)
    E = np.random.default_rng(22).uniform(0.01, 1.0, len(e))
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", E, 0.3, 2)
    x0 = [int(i) for i in O.nodes_on_plane(c, 0, 0.0, 1e-9)]
    # clamp x=0 and one component of one extra node: partial nodes must work
    bcs = [(3 * n + k, 0.0) for n in x0 for k in range(3)] + [(3 * (len(c) - 1) + 1, 0.0)]
    S = F.reduce_system(K, np.ones(K.nrows), bcs)
    _fsai_vs_oracle(S, 3)


def test_fsai_factor_poisson_is_tril_pattern(ctx):
    c, e = box([5, 5, 4])
    c = jitter(c, 0.03, 23)
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_poisson(m, np.exp(np.random.default_rng(24).normal(size=len(e))), 2)
    S = F.reduce_system(K, np.ones(K.nrows), unit_cube_bcs(c))
    _fsai_vs_oracle(S, 1)


@pytest.mark.parametrize("solver", [F.SOLVER_JACOBI_PCG, F.SOLVER_FSAI_MP_PCG])
def test_node_block_layout_matches_scalar_csr(ctx, solver):
    # The node-block operator/factor (used when every free node has all dofs
    # free) must give the same solution as the scalar-CSR path.
    c, e = box([6, 3, 3], mx=(2.0, 1.0, 1.0))
    c = jitter(c, 0.03, 41)
    E = np.random.default_rng(42).uniform(0.05, 1.0, len(e))
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", E, 0.3, 2)
    rhs = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    x0 = [int(i) for i in O.nodes_on_plane(c, 0, 0.0, 1e-9)]
    bcs = [(3 * n + k, 0.0) for n in x0 for k in range(3)]
    S1 = F.reduce_system(K, rhs, bcs)
    S2 = F.reduce_system(K, rhs, bcs)
    st1 = S1.solve(solver=solver, tol=1e-12)  # node-block, symmetric half storage
    st2 = S2.solve(solver=solver, tol=1e-12, csr_only=True)
    u1, u2 = S1.solution(), S2.solution()
    assert st1["rel_residual"] <= 1e-12 and st2["rel_residual"] <= 1e-12
    assert abs(st1["iterations"] - st2["iterations"]) <= max(3, st2["iterations"] // 20)
    assert np.max(np.abs(u1 - u2)) <= 1e-9 * np.max(np.abs(u2))
    st3 = S1.solve(solver=solver, tol=1e-12, full_operator=True)  # node-block, full storage
    u3 = S1.solution()
    assert st3["rel_residual"] <= 1e-12
    assert abs(st3["iterations"] - st2["iterations"]) <= max(3, st2["iterations"] // 20)
    assert np.max(np.abs(u3 - u2)) <= 1e-9 * np.max(np.abs(u2))
    prof = S1.profile_spmv(2)
    assert prof["nb_ms"] > 0 and prof["nbs_ms"] > 0  # both node-block layouts were built
    assert prof["nbs_bytes"] < 0.75 * prof["nb_bytes"]


def test_quad_linear_patch_reproduced(ctx):
    # u = x + y is harmonic: P1/Q1 reproduce it exactly on a distorted mesh.
    c, e = quad_grid(6, 5)
    c = jitter(c, 0.05, 12)
    m = F.Mesh.from_arrays(F.CELL_QUAD4, c, e, ctx=ctx)
    bnd = [i for i in range(len(c)) if min(c[i][0], c[i][1]) < 1e-12 or max(c[i][0], c[i][1]) > 1 - 1e-12]
    res = F.solve_poisson(m, 1.0, 2, 0.0, [(i, c[i][0] + c[i][1]) for i in bnd], tol=1e-14)
    assert np.max(np.abs(np.array(res.values) - (c[:, 0] + c[:, 1]))) < 1e-12


def test_plane_stress_quad_patch(ctx):
    c, e = quad_grid(4, 4)
    c = jitter(c, 0.05, 13)
    m = F.Mesh.from_arrays(F.CELL_QUAD4, c, e, ctx=ctx)
    bnd = [i for i in range(len(c)) if min(c[i][0], c[i][1]) < 1e-12 or max(c[i][0], c[i][1]) > 1 - 1e-12]
    bcs = [(i, 0, 0.1 * c[i][0]) for i in bnd] + [(i, 1, 0.2 * c[i][1]) for i in bnd]
    res = F.solve_elasticity(m, "plane-stress", 1.0, 0.3, 2, bcs, tol=1e-14)
    u = res.to_numpy()
    assert np.max(np.abs(u[:, 0] - 0.1 * c[:, 0])) < 1e-12
    assert np.max(np.abs(u[:, 1] - 0.2 * c[:, 1])) < 1e-12


def test_solver_is_deterministic(ctx):
    m = F.Mesh.box_mesh([0, 0, 0], [1, 1, 1], [10, 10, 10], ctx=ctx)
    c = m.coords_array
    K = F.assemble_poisson(m, 1.0, 2)
    rhs = F.load_poisson_source(m, 1.0, 2)
    bcs = unit_cube_bcs(c)
    u1, s1 = F.solve_with_dirichlet(K, rhs, bcs)
    u2, s2 = F.solve_with_dirichlet(K, rhs, bcs)
    assert np.array_equal(u1, u2) and s1["iterations"] == s2["iterations"]


# ---- errors mapped to status codes, never a device fault --------------------------------

def test_bad_inputs_map_to_status_codes(ctx):
    c, e = box([2, 2, 2])
    bad = e.copy()
    bad[0, 0] = len(c)
    with pytest.raises(F.TptFemError) as ei:
        F.Mesh.from_arrays(F.CELL_TET4, c, bad, ctx=ctx)
    assert ei.value.name == "INVALID_ARG"
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    with pytest.raises(F.TptFemError) as ei:
        F.assemble_elasticity(m, "plane-stress", 1.0, 0.3, 2)
    assert ei.value.name == "MODEL_DIM_MISMATCH"
    with pytest.raises(F.TptFemError) as ei:
        F.assemble_poisson(m, np.nan, 2)
    assert ei.value.name == "INVALID_ARG"
    flat = c.copy()
    flat[:, 2] = 0.0  # every tet degenerate
    mf = F.Mesh.from_arrays(F.CELL_TET4, flat, e, ctx=ctx)
    with pytest.raises(F.TptFemError) as ei:
        F.assemble_poisson(mf, 1.0, 2)
    assert ei.value.name == "NUMERIC"


def test_not_spd_and_not_converged_are_reported(ctx):
    m = F.Mesh.box_mesh([0, 0, 0], [1, 1, 1], [6, 6, 6], ctx=ctx)
    c = m.coords_array
    bcs = unit_cube_bcs(c)
    K = F.assemble_poisson(m, -1.0, 2)
    rhs = F.load_poisson_source(m, 1.0, 2)
    with pytest.raises(F.TptFemError) as ei:
        F.solve_with_dirichlet(K, rhs, bcs)
    assert ei.value.name in ("NUMERIC", "BREAKDOWN")
    K = F.assemble_poisson(m, 1.0, 2)
    with pytest.raises(F.TptFemError) as ei:
        F.solve_with_dirichlet(K, rhs, bcs, max_iter=3)
    assert ei.value.name == "NOT_CONVERGED"
    # the context stays usable after every error
    u, st = F.solve_with_dirichlet(K, rhs, bcs)
    assert st["rel_residual"] <= 1e-10


@pytest.mark.parametrize("dim", [3, 1])
def test_factor_pattern_from_group_adjacency_matches_row_union(ctx, dim):
    # With the node-block operator built (every free node has all dofs free), the
    # factor pattern comes from its group adjacency; without it, from a sorted
    # union per row.  Both must give the same rows, columns and values.
    c, e = box([6, 4, 3], mx=(2.0, 1.0, 1.0))
    c = jitter(c, 0.03, 61)
    coef = np.random.default_rng(62).uniform(0.05, 1.0, len(e))
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    if dim == 3:
        K = F.assemble_elasticity(m, "3d", coef, 0.3, 2)
        bcs = [(3 * n + k, 0.0) for n in O.nodes_on_plane(c, 0, 0.0, 1e-9) for k in range(3)]
    else:
        K = F.assemble_poisson(m, coef, 2)
        bcs = unit_cube_bcs(c)
    rows = F.reduce_system(K, np.ones(K.nrows), bcs)
    rp1, ci1, va1, s1 = rows.fsai()
    groups = F.reduce_system(K, np.ones(K.nrows), bcs)
    groups.solve(solver=F.SOLVER_JACOBI_PCG, tol=1e-8)  # builds the node-block operator first
    rp2, ci2, va2, s2 = groups.fsai()
    assert np.array_equal(rp1, rp2) and np.array_equal(ci1, ci2)
    assert np.array_equal(va1, va2) and np.array_equal(s1, s2)


def test_profiled_numeric_assembly_rewrites_identical_values(ctx):
    c, e = box([5, 4, 3], mx=(2.0, 1.0, 1.0))
    c = jitter(c, 0.03, 71)
    E = np.random.default_rng(72).uniform(0.05, 1.0, len(e))
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", E, 0.3, 2)
    before = K.to_csr()
    ms = K.profile_assembly(3)
    after = K.to_csr()
    assert ms > 0.0
    for a, b in zip(before, after):
        assert np.array_equal(a, b)
