"""The row-partitioned FP64 Jacobi-PCG of the library (tptfem_dist_*) on one
GPU: several ranks in lock step, exchanging ghost values by device copies,
give the serial solution; the Python driver over the library's ranks equals
the library's own lock-step loop."""
import ctypes as C

import numpy as np
import pytest

import tpt_fem as F
from meshes import box, jitter
from tpt_fem import _native as N
from tpt_fem import distributed as D
from tpt_fem import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture
def system(ctx):
    n = [12, 4, 4]
    c, e = box(n, mx=(4.0, 1.0, 1.0))
    c = jitter(c, 0.02, 3)
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", W.cantilever_young(n, seed=4), 0.3, 2)
    rhs = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    dof, val = W.clamp_x0_bcs(c)
    return F.reduce_system(K, rhs, list(zip(dof, val)))


def solve_local(ctx, S, nranks):
    x = np.zeros(S.n_free)
    it, rel = C.c_int64(), C.c_double()
    ctx.check(ctx.lib.tptfem_dist_solve_local(ctx.h, S.h, nranks, 1e-10, 0, N.ptr(x), C.byref(it), C.byref(rel)))
    return x, it.value, rel.value


@pytest.mark.parametrize("nranks", [1, 2, 3, 4])
def test_lockstep_ranks_give_the_serial_solution(ctx, system, nranks):
    S = system
    st = S.solve(solver=F.SOLVER_JACOBI_PCG, tol=1e-10)
    rp, ci, va, fred, _ = S.download()
    import scipy.sparse as sp
    A = sp.csr_matrix((va, ci, rp), shape=(S.n_free, S.n_free))
    x, it, rel = solve_local(ctx, S, nranks)
    assert rel <= 1e-10
    assert np.linalg.norm(A @ x - fred) <= 2e-10 * np.linalg.norm(fred)
    assert abs(it - st["iterations"]) <= max(5, st["iterations"] // 50)


def test_python_driver_over_library_ranks_equals_library_loop(ctx, system):
    S = system
    starts = D.partition_rows(S.n_free, 3, 3)
    ranks = [D.LibRank(S, k, 3, starts) for k in range(3)]
    for r in ranks:
        for q in range(3):
            assert r.recv_counts[q] == ranks[q].send_counts[r.rank]
    it, rel = D.solve(ranks, D.LocalComm(), tol=1e-10)
    x = np.concatenate([r.solution() for r in ranks])
    x2, it2, rel2 = solve_local(ctx, S, 3)
    assert it == it2 and abs(rel - rel2) <= 1e-15 and np.array_equal(x, x2)
