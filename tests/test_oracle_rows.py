"""The row-restricted oracle used by the configuration-size parity tests,
checked on the CPU against the oracle's whole-matrix path.

csr_rows restates Coo::to_csr(assemble(...)) (crates/tpt-fem-sparse/src/lib.rs:122-175
over crates/tpt-fem-assembly/src/lib.rs:428-480) one row at a time; reduced_rows
restates reduce_system (assembly:504-535) for those rows; load_poisson_rows the
load loop of solve_poisson (crates/tpt-fem-thermal/src/lib.rs:224-230).  Each must
give, bit for bit, the rows of the full COO + stable sort + duplicate sum path.
"""
import numpy as np

from meshes import box, jitter, quad_grid, tri_grid
from oracle import oracle as O


def full_rows(csr, rows):
    ptr = [0]
    cols, vals = [], []
    for r in rows:
        a, b = csr.row_ptrs[r], csr.row_ptrs[r + 1]
        cols += list(csr.col_ind[a:b])
        vals += list(csr.values[a:b])
        ptr.append(len(cols))
    return np.array(ptr), np.array(cols, np.int64), np.array(vals)


def same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b)) and all(x.dtype == y.dtype for x, y in zip(a, b))


def test_elasticity_rows_match_full_to_csr_on_jittered_tets():
    c, e = box([5, 4, 3], mx=(2.0, 1.0, 1.0))
    c = jitter(c, 0.05, 11)
    E = np.random.default_rng(12).uniform(0.1, 2.0, size=len(e))
    m = O.Mesh(O.CELL_TET, c, e)
    full = O.assemble_elasticity(m, O.MODEL_3D, E, 0.3, 2).to_csr()
    rows = np.arange(3 * len(c))
    assert same(O.csr_rows(m, "elasticity", E, rows), full_rows(full, rows))
    pick = np.random.default_rng(13).choice(len(rows), 40)
    assert same(O.csr_rows(m, "elasticity", E, pick), full_rows(full, pick))


def test_elasticity_rows_on_the_structured_cantilever_with_per_element_E():
    from tpt_fem import workloads as W
    n = [8, 3, 3]
    c, e = box(n, mx=(4.0, 1.0, 1.0))
    E = W.cantilever_young(n)
    m = O.Mesh(O.CELL_TET, c, e)
    full = O.assemble_elasticity(m, O.MODEL_3D, E, 0.3, 2).to_csr()
    rows = np.arange(3 * len(c))
    assert same(O.csr_rows(m, "elasticity", E, rows), full_rows(full, rows))


def test_poisson_rows_match_full_to_csr():
    c, e = box([4, 5, 3])
    k = np.exp(np.random.default_rng(14).standard_normal(len(e)))
    for coords in (c, jitter(c, 0.04, 15)):
        m = O.Mesh(O.CELL_TET, coords, e)
        full = O.assemble_poisson(m, k, 2).to_csr()
        rows = np.arange(len(coords))
        assert same(O.csr_rows(m, "poisson", k, rows), full_rows(full, rows))
        assert same(O.csr_rows(m, "poisson", 1.5, rows[::3]), full_rows(O.assemble_poisson(m, 1.5, 2).to_csr(),
                                                                         rows[::3]))


def test_2d_cells_match_full_to_csr():
    for (c, e), cell in ((quad_grid(5, 3), O.CELL_QUAD), (tri_grid(4, 4), O.CELL_TRI)):
        m = O.Mesh(cell, c, e)
        for order in (1, 2, 3):
            full = O.assemble_poisson(m, 2.0, order).to_csr()
            rows = np.arange(len(c))
            assert same(O.csr_rows(m, "poisson", 2.0, rows, quad_order=order), full_rows(full, rows))
        full = O.assemble_elasticity(m, O.MODEL_PLANE_STRESS, 1.0, 0.3, 2).to_csr()
        rows = np.arange(2 * len(c))
        got = O.csr_rows(m, "elasticity", 1.0, rows, model=O.MODEL_PLANE_STRESS)
        assert same(got, full_rows(full, rows))


def test_reduced_rows_match_reduce_system_with_duplicate_bcs():
    c, e = box([4, 3, 3])
    c = jitter(c, 0.03, 16)
    m = O.Mesh(O.CELL_TET, c, e)
    coo = O.assemble_elasticity(m, O.MODEL_3D, 1.0, 0.3, 2)
    rhs = np.random.default_rng(17).standard_normal(3 * len(c))
    x0 = O.nodes_on_plane(c, 0, 0.0, 1e-9)
    bcs = [(3 * int(n) + k, 0.01 * (k + 1)) for n in x0 for k in range(3)]
    bcs += [(bcs[2][0], 5.0), (bcs[0][0], -1.0)]  # duplicates: lifting uses the first value
    kred, fred, free = O.reduce_system(coo, rhs, bcs)
    kr = kred.to_csr()
    fidx = -np.ones(len(rhs), np.int64)
    fidx[free] = np.arange(len(free))
    ptr, cols, vals = O.csr_rows(m, "elasticity", 1.0, free)
    rp, rc, rv, rf = O.reduced_rows(ptr, cols, vals, rhs[free], bcs, fidx)
    assert np.array_equal(rf, fred)
    assert same((rp, rc, rv), (kr.row_ptrs, kr.col_ind, kr.values))


def test_poisson_load_rows_match_the_load_loop():
    c, e = box([3, 4, 5])
    c = jitter(c, 0.05, 18)
    m = O.Mesh(O.CELL_TET, c, e)
    rhs = O.load_poisson_source(m, 1.25, 2)
    nodes = np.array([0, 5, 17, len(c) - 1, 5], np.int64)
    assert np.array_equal(O.load_poisson_rows(m, 1.25, nodes), rhs[nodes])
