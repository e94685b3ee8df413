"""The CPU oracle pinned against the reference's own tests and golden files.

Each test restates a reference unit test (file:line cited) on the oracle, or
checks the oracle against a committed golden fixture, so the oracle the GPU
path is later compared with is itself anchored on the reference.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as O


def unit_cube_bcs(coords):
    bcs = []
    for axis in range(3):
        for coord in (0.0, 1.0):
            for nid in O.nodes_on_plane(coords, axis, coord, 1e-9):
                bcs.append((int(nid), 0.0))
    return bcs


# ---- golden fixtures -----------------------------------------------------------

def test_box_mesh_matches_committed_vtk_golden():
    # mesh_gen_box_structured.vtk, written by crates/tpt-fem/examples/mesh_gen_box.rs:15-21
    g = np.load(os.path.join(GOLDEN, "box4_structured.npz"))
    c, e = O.box_mesh([0, 0, 0], [1, 1, 1], [4, 4, 4])
    assert np.array_equal(g["points"], c)
    assert np.array_equal(g["conn"], e)


def test_thermal_vtk_mesh_matches_and_its_field_is_stale():
    # thermal_solve.vtk: connectivity of box_mesh([6,6,6]) matches; its temperature
    # field predates the current Map (it was written with a transposed inverse),
    # so it is NOT a value golden -- the current-code centre value differs.
    g = np.load(os.path.join(GOLDEN, "box6_thermal_mesh.npz"))
    c, e = O.box_mesh([0, 0, 0], [1, 1, 1], [6, 6, 6])
    assert np.array_equal(g["points"], c)
    assert np.array_equal(g["conn"], e)
    m = O.Mesh(O.CELL_TET, c, e)
    coo = O.assemble_poisson(m, 1.0, 2)
    f = O.load_poisson_source(m, 1.0, 2)
    u = O.solve_with_dirichlet(coo, f, unit_cube_bcs(c))
    assert abs(u[171] - 0.05396558174335943) < 1e-12
    assert abs(g["stale_temperature"][171] - u[171]) > 1e-3


# ---- crates/tpt-fem-sparse/src/lib.rs tests --------------------------------------

def test_coo_sums_duplicates_and_sorts():  # sparse:378
    c = O.Coo()
    for r, col, v in [(1, 1, 1.0), (0, 1, 1.0), (0, 0, 1.0), (0, 0, 1.0), (1, 0, 1.0)]:
        c.push(r, col, v)
    csr = c.to_csr()
    assert (csr.nrows, csr.ncols) == (2, 2)
    assert list(csr.row_ptrs) == [0, 2, 4]
    assert list(csr.col_ind) == [0, 1, 0, 1]
    assert list(csr.values) == [2.0, 1.0, 1.0, 1.0]


def _coo(entries):
    c = O.Coo()
    for e in entries:
        c.push(*e)
    return c


def test_solve_2x2():  # sparse:394
    x = O.solve(_coo([(0, 0, 2.0), (0, 1, 1.0), (1, 0, 1.0), (1, 1, 3.0)]), [3.0, 5.0])
    assert abs(x[0] - 0.8) < 1e-10 and abs(x[1] - 1.4) < 1e-10


def test_solve_3x3_diagonally_dominant():  # sparse:407
    c = _coo([(0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0), (1, 1, 4.0), (1, 2, -1.0), (2, 1, -1.0), (2, 2, 4.0)])
    for v in O.solve(c, [3.0, 2.0, 3.0]):
        assert abs(v - 1.0) < 1e-9


def test_solve_with_duplicates():  # sparse:444
    c = _coo([(0, 0, 1.0), (0, 0, 1.0), (0, 1, 0.5), (0, 1, 0.5), (1, 0, 0.5), (1, 0, 0.5), (1, 1, 1.5),
              (1, 1, 1.5)])
    x = O.solve(c, [3.0, 5.0])
    assert abs(x[0] - 0.8) < 1e-10 and abs(x[1] - 1.4) < 1e-10


def test_csr_matvec_sequential_row_sums():  # sparse:195-205 semantics
    c = _coo([(0, 0, 2.0), (0, 2, 1.0), (1, 1, 3.0)])
    y = c.to_csr().matvec(np.array([1.0, 2.0, 3.0, 4.0]))
    assert list(y) == [5.0, 6.0, 0.0, 0.0]  # y has max(nrows, len(x)) entries


# ---- crates/tpt-fem-assembly/src/lib.rs tests --------------------------------------

def square_tri_mesh():
    coords = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]])
    conn = np.array([[0, 1, 3], [0, 3, 2]])
    return O.Mesh(O.CELL_TRI, coords, conn)


def test_assemble_sizes_and_symmetry():  # assembly:775
    m = square_tri_mesh()
    mats = np.stack([np.eye(3), np.eye(3)])
    csr = O.assemble_given(m, 1, mats).to_csr()
    assert (csr.nrows, csr.ncols, csr.nnz) == (4, 4, 4)


def test_dirichlet_reduces_to_known_solution():  # assembly:795
    m = O.Mesh(O.CELL_LINE, np.array([[0.0], [0.5], [1.0]]), np.array([[0, 1], [1, 2]]))
    k = np.array([[2.0, -2.0], [-2.0, 2.0]])
    coo = O.assemble_given(m, 1, np.stack([k, k]))
    u = O.solve_with_dirichlet(coo, [0.0, 0.0, 0.0], [(0, 0.0), (2, 1.0)])
    assert abs(u[0]) < 1e-12 and abs(u[1] - 0.5) < 1e-12 and abs(u[2] - 1.0) < 1e-12


def test_neumann_conserves_total_load():  # assembly:814
    m = O.Mesh(O.CELL_TRI, np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), np.array([[0, 1, 2]]))
    rhs = O.apply_neumann(m, 1, lambda x, n: 1.0, np.zeros(3))
    assert abs(rhs.sum() - (2.0 + 2.0 ** 0.5)) < 1e-9


def test_boundary_faces_of_square():  # assembly:851
    assert O.boundary_face_count(square_tri_mesh()) == 4


# ---- element / quadrature / mesh-gen tests ----------------------------------------

def test_jacobian_3d_sheared_tet():  # element:887
    X = np.array([[1.0, 1.0, 1.0], [3.0, 1.0, 1.0], [1.0, 4.0, 1.0], [1.0, 1.0, 5.0]])
    jac, det, inv = O.map_at(O.CELL_TET, X, [0.2, 0.2, 0.2])
    assert abs(det - 24.0) < 1e-12
    assert np.allclose(jac, np.diag([2.0, 3.0, 4.0]), atol=1e-12)
    assert np.allclose(jac @ inv, np.eye(3), atol=1e-12)


def test_tet_degree2_rule_monomial_exactness():  # quadrature:532
    from math import factorial
    pts, w = O.cell_quad(O.CELL_TET, 2)
    assert abs(w.sum() - 1.0 / 6.0) < 1e-9
    for i in range(3):
        for j in range(3 - i):
            for k in range(3 - i - j):
                exact = factorial(i) * factorial(j) * factorial(k) / factorial(i + j + k + 3)
                approx = np.sum(w * pts[:, 0] ** i * pts[:, 1] ** j * pts[:, 2] ** k)
                assert abs(approx - exact) < 1e-9


def test_box_mesh_counts_and_orientation():  # mesh-gen:830
    c, e = O.box_mesh([0, 0, 0], [1, 1, 1], [2, 2, 2])
    assert len(c) == 27 and len(e) == 48
    for t in e:
        a, b, cc, d = c[t]
        assert np.dot(b - a, np.cross(cc - a, d - a)) > 0


# ---- thermal / elasticity tests -----------------------------------------------------

def test_poisson_2d_linear_is_exact():  # thermal:344
    coords = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0], [0.5, 0.5]])
    conn = np.array([[0, 1, 4], [1, 3, 4], [3, 2, 4], [2, 0, 4]])
    m = O.Mesh(O.CELL_TRI, coords, conn)
    coo = O.assemble_poisson(m, 1.0, 2)
    rhs = O.load_poisson_source(m, 0.0, 2)
    u = O.solve_with_dirichlet(coo, rhs, [(0, 0.0), (1, 1.0), (2, 1.0), (3, 2.0)])
    assert abs(u[4] - 1.0) < 1e-10 and abs(u[0]) < 1e-12 and abs(u[3] - 2.0) < 1e-12


def test_plane_stress_patch_test():  # elasticity:742
    coords = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0], [0.5, 0.5]])
    conn = np.array([[0, 1, 4], [1, 3, 4], [3, 2, 4], [2, 0, 4]])
    m = O.Mesh(O.CELL_TRI, coords, conn)
    coo = O.assemble_elasticity(m, O.MODEL_PLANE_STRESS, 1.0, 0.3, 2)
    bcs = []
    for node, x, y in [(0, 0.0, 0.0), (1, 0.1, 0.0), (2, 0.0, 0.2), (3, 0.1, 0.2)]:
        bcs += [(2 * node, x), (2 * node + 1, y)]
    u = O.solve_with_dirichlet(coo, np.zeros(10), bcs)
    assert abs(u[8] - 0.05) < 1e-9 and abs(u[9] - 0.1) < 1e-9


def test_poisson_box8_sanity_values():
    # Poisson on box_mesh [8,8,8], k=1, f=1, u=0 on all faces (the plain-method case).
    c, e = O.box_mesh([0, 0, 0], [1, 1, 1], [8, 8, 8])
    m = O.Mesh(O.CELL_TET, c, e)
    coo = O.assemble_poisson(m, 1.0, 2)
    csr = coo.to_csr()
    assert (csr.nrows, csr.nnz, int(np.diff(csr.row_ptrs).max())) == (729, 4617, 7)
    f = O.load_poisson_source(m, 1.0, 2)
    kred, fred, free = O.reduce_system(coo, f, unit_cube_bcs(c))
    assert len(free) == 343 and kred.to_csr().nnz == 2107
    u = O.solve_with_dirichlet(coo, f, unit_cube_bcs(c))
    assert abs(u[364] - 0.05491766911624052) < 1e-12


def test_elasticity_tet_keeps_74_of_144_entries_on_kuhn_tets():
    c, e = O.box_mesh([0, 0, 0], [1, 1, 1], [2, 2, 2])
    m = O.Mesh(O.CELL_TET, c, e)
    for eid in range(m.n_elems):
        k = O.elasticity_element_matrix(m, eid, O.MODEL_3D, 1.0, 0.3, 2)
        assert int(np.count_nonzero(k)) == 74


def test_tet4_elasticity_linear_patch_on_box_mesh():
    # A linear displacement field is reproduced exactly (new test: the
    # reference pins no 3-D Tet4 elasticity values).
    c, e = O.box_mesh([0, 0, 0], [1, 1, 1], [3, 3, 3])
    m = O.Mesh(O.CELL_TET, c, e)
    coo = O.assemble_elasticity(m, O.MODEL_3D, 1.0, 0.3, 2)
    A = np.array([[0.01, 0.02, -0.01], [0.0, 0.03, 0.01], [0.02, -0.01, 0.0]])
    uex = (c @ A.T).reshape(-1)
    bnd = set()
    for axis in range(3):
        for coord in (0.0, 1.0):
            bnd |= set(int(i) for i in O.nodes_on_plane(c, axis, coord, 1e-9))
    bcs = [(3 * n + k, uex[3 * n + k]) for n in sorted(bnd) for k in range(3)]
    u = O.solve_with_dirichlet(coo, np.zeros(3 * len(c)), bcs)
    assert np.max(np.abs(u - uex)) < 1e-12


def test_pcg_jacobi_matches_dense_lu_on_poisson_box8():
    c, e = O.box_mesh([0, 0, 0], [1, 1, 1], [8, 8, 8])
    m = O.Mesh(O.CELL_TET, c, e)
    coo = O.assemble_poisson(m, 1.0, 2)
    f = O.load_poisson_source(m, 1.0, 2)
    kred, fred, free = O.reduce_system(coo, f, unit_cube_bcs(c))
    x_lu = O.solve(kred, fred)
    csr = kred.to_csr()
    x, it, rel = O.pcg_jacobi(csr, fred, tol=1e-13)
    assert it > 0 and rel < 1e-13
    assert np.max(np.abs(x - x_lu)) < 1e-12 * np.max(np.abs(x_lu))
    # the int32-index form is the same arithmetic, bit for bit
    x32, it32, rel32 = O.pcg_jacobi_i32(csr.nrows, csr.row_ptrs, csr.col_ind, csr.values, fred, tol=1e-13,
                                        nthreads=1)
    x1, it1, rel1 = O.pcg_jacobi(csr, fred, tol=1e-13, nthreads=1)
    assert (it32, rel32) == (it1, rel1) and np.array_equal(x32, x1)


def test_robin_conserves_total_measure():  # assembly:835
    m = O.Mesh(O.CELL_TRI, np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), np.array([[0, 1, 2]]))
    coo = O.apply_robin(O.Coo(), m, 1, lambda x, n: 1.0)
    assert abs(coo.to_csr().values.sum() - (2.0 + 2.0 ** 0.5)) < 1e-9
    sel = O.apply_robin_selected(O.Coo(), m, 1, -1, 1.0, 1.0)
    assert np.array_equal(sel.to_csr().values, coo.to_csr().values)
