"""Robin boundary terms (apply_robin, crates/tpt-fem-assembly/src/lib.rs:674-753)
assembled on the device after the element terms, as solve_poisson pushes them
(crates/tpt-fem-thermal/src/lib.rs:235-237): patterns and values bit-exact
against the oracle's restatement on Tri3, Quad4 and Tet4 meshes, including
the entries the Robin pushes add where the element matrices have zeros."""
import numpy as np
import pytest

import tpt_fem as F
from meshes import box, jitter, quad_grid, tri_grid
from oracle import oracle as O
from test_gpu_parity import assert_csr_equal

pytestmark = pytest.mark.gpu


def oracle_robin(cell, c, e, k, axis, sign, h):
    om = O.Mesh(cell, c, e)
    coo = O.assemble_poisson(om, k, 2)
    return O.apply_robin_selected(coo, om, 1, axis, sign, h), om


@pytest.mark.parametrize("axis,sign", [(-1, 1.0), (0, 1.0), (1, -1.0)])
def test_robin_tri3(ctx, axis, sign):
    c, e = tri_grid(6, 4, 2.0, 1.0)
    c = jitter(c, 0.05, 3)
    k = np.linspace(0.5, 2.0, len(e))
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    K = F.assemble_poisson(m, k, 2, robin=(axis, sign, 2.5))
    coo, _ = oracle_robin(O.CELL_TRI, c, e, k, axis, sign, 2.5)
    assert_csr_equal(K, coo)


def test_robin_quad4(ctx):
    c, e = quad_grid(5, 4, 2.0, 1.0)
    c = jitter(c, 0.05, 6)
    m = F.Mesh.from_arrays(F.CELL_QUAD4, c, e, ctx=ctx)
    K = F.assemble_poisson(m, 1.0, 3, robin=(0, 1.0, 0.75))
    om = O.Mesh(O.CELL_QUAD, c, e)
    coo = O.apply_robin_selected(O.assemble_poisson(om, 1.0, 3), om, 1, 0, 1.0, 0.75)
    assert_csr_equal(K, coo)


def test_robin_tet4_adds_entries_where_elements_have_zeros(ctx):
    c, e = box([4, 3, 3])
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K0 = F.assemble_poisson(m, 1.0, 2)
    K = F.assemble_poisson(m, 1.0, 2, robin=(2, -1.0, 1.5))
    coo, _ = oracle_robin(O.CELL_TET, c, e, 1.0, 2, -1.0, 1.5)
    assert_csr_equal(K, coo)
    assert K.nnz > K0.nnz  # face pairs that the Kuhn tets' stiffness leaves uncoupled


def test_robin_survives_reassembly(ctx):
    c, e = tri_grid(5, 5)
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    K = F.assemble_poisson(m, np.ones(len(e)), 2, robin=(-1, 1.0, 3.0))
    k2 = np.random.default_rng(1).uniform(0.2, 2.0, len(e))
    K.reassemble(k2)
    coo, _ = oracle_robin(O.CELL_TRI, c, e, k2, -1, 1.0, 3.0)
    assert_csr_equal(K, coo)


def test_robin_solution_matches_oracle_dense_solve(ctx):
    # heat source, cooled by a Robin (convection) term on the right edge, held at
    # u = 0 on the left edge
    c, e = tri_grid(8, 4, 2.0, 1.0)
    c = jitter(c, 0.04, 9)
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    K = F.assemble_poisson(m, 1.0, 2, robin=(0, 1.0, 4.0))
    rhs = F.load_poisson_source(m, 1.0, 2)
    bcs = [(int(i), 0.0) for i in O.nodes_on_plane(c, 0, 0.0, 1e-9)]
    u, st = F.solve_with_dirichlet(K, rhs, bcs, tol=1e-13)
    coo, om = oracle_robin(O.CELL_TRI, c, e, 1.0, 0, 1.0, 4.0)
    u_ref = O.solve_with_dirichlet(coo, O.load_poisson_source(om, 1.0, 2), bcs)
    assert np.max(np.abs(u - u_ref)) <= 1e-10 * np.max(np.abs(u_ref))
