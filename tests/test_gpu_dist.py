"""The row-partitioned FP64 PCG of the library (tptfem_dist_*) on one GPU:
several ranks in lock step, exchanging ghost values by device copies, give the
serial solution; the Python driver over the library's ranks equals the
library's own lock-step loop.  With the partitioned two-level preconditioner
(block FSAI, classic or learned, plus the aggregation coarse space, whose
partial matrices and restrictions the driver sums over the ranks) the solve
takes a fraction of Jacobi's iterations, about as many as the one-GPU
two-level solver at one rank and a few more as the partition cuts the
factor's couplings."""
import os

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


def cantilever(ctx, n, seed=4):
    c, e = box(n, mx=(4.0, 1.0, 1.0))
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", W.cantilever_young(n, seed=seed), 0.3, 2)
    rhs = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    dof, val = W.clamp_x0_bcs(c)
    return F.reduce_system(K, rhs, list(zip(dof, val)))


def host_csr(S):
    import scipy.sparse as sp
    rp, ci, va, fred, _ = S.download()
    return sp.csr_matrix((va, ci, rp), shape=(S.n_free, S.n_free)), fred


def driver_solve(S, nranks, kind=None, aggs=0):
    starts = D.partition_rows(S.n_free, 3, nranks)
    ranks = [D.LibRank(S, k, nranks, starts) for k in range(nranks)]
    if kind:
        assert len({r.set_precond(kind, aggs) for r in ranks}) == 1
    it, rel = D.solve(ranks, D.LocalComm(), tol=1e-10)
    return np.concatenate([r.solution() for r in ranks]), it, rel, ranks[0].coarse_size


@pytest.fixture(scope="module")
def cant(ctx):
    S = cantilever(ctx, [40, 10, 10])
    A, fred = host_csr(S)
    jac = S.solve(solver=F.SOLVER_JACOBI_PCG, tol=1e-10)["iterations"]
    return S, A, fred, jac


@pytest.mark.parametrize("nranks", [1, 2, 4])
def test_partitioned_two_level_classic_fsai(ctx, cant, nranks):
    S, A, fred, jac = cant
    x, it, rel, nc = driver_solve(S, nranks, "fsai", 0)
    assert nc > 0 and rel <= 1e-10
    assert np.linalg.norm(A @ x - fred) <= 1e-9 * np.linalg.norm(fred)
    one = S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=1e-10, fresh_setup=True, coarse=True)["iterations"]
    assert it <= jac / 4, (it, jac)
    if nranks == 1:  # the same factor and coarse space as the one-GPU solver
        assert abs(it - one) <= max(5, one // 10), (it, one)
    else:
        assert it <= 1.6 * one, (it, one)


def test_partitioned_coarse_space_pays_and_block_fsai_alone_converges(ctx, cant):
    S, A, fred, jac = cant
    x, it_fsai, rel, nc = driver_solve(S, 3, "fsai", None)
    assert nc == 0 and rel <= 1e-10 and np.linalg.norm(A @ x - fred) <= 1e-9 * np.linalg.norm(fred)
    _, it_two, _, nc2 = driver_solve(S, 3, "fsai", 0)
    assert nc2 > 0 and it_two < 0.6 * it_fsai < jac, (it_two, it_fsai, jac)


def test_partitioned_learned_block_factor(ctx):
    from tpt_fem import lfsai as LF
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    model = LF.LearnedFsai.load(ctx, os.path.join(root, "tpt-fem_b200", "weights", "lfsai_elasticity.bin"))
    S = cantilever(ctx, [40, 10, 10], seed=97)
    model.attach(S)
    A, fred = host_csr(S)
    one = S.solve(solver=F.SOLVER_LEARNED_FSAI_PCG, tol=1e-10, fresh_setup=True, coarse=True)
    assert not one["fell_back"]
    for nranks in (1, 4):
        x, it, rel, nc = driver_solve(S, nranks, "learned", 0)
        assert nc > 0 and rel <= 1e-10
        assert np.linalg.norm(A @ x - fred) <= 1e-9 * np.linalg.norm(fred)
        bound = max(5, one["iterations"] // 10) + one["iterations"] if nranks == 1 else 1.6 * one["iterations"]
        assert it <= bound, (nranks, it, one["iterations"])


def test_partitioned_preconditioner_call_order_is_checked(ctx, cant):
    S = cant[0]
    starts = D.partition_rows(S.n_free, 3, 2)
    r = D.LibRank(S, 0, 2, starts)
    with pytest.raises(F.TptFemError, match="no block preconditioner"):
        r.precondition()
    with pytest.raises(F.TptFemError, match="kind"):
        ctx.check(ctx.lib.tptfem_dist_set_precond(ctx.h, r.h, S.h, 7, -1, None))
    assert r.set_precond("fsai", 0) > 0
    r.start()
    with pytest.raises(F.TptFemError, match="not factored"):
        r.precondition()
    with pytest.raises(F.TptFemError, match="already set"):
        r.set_precond("fsai", 0)
    # a solve that rebuilds the system's coarse space with another aggregate
    # count leaves the rank's coarse data stale: refused, not read
    S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=1e-8, fresh_setup=True, coarse=True, coarse_aggregates=3)
    with pytest.raises(F.TptFemError, match="rebuilt"):
        r.start()


def test_library_two_level_loop_equals_python_driver(ctx, cant):
    S, A, fred, jac = cant
    x, it, rel, nc = driver_solve(S, 3, "fsai", 0)
    x2 = np.zeros(S.n_free)
    it2, rel2 = C.c_int64(), C.c_double()
    ctx.check(ctx.lib.tptfem_dist_solve_local_precond(ctx.h, S.h, 3, 1, 0, 1e-10, 0, N.ptr(x2), C.byref(it2),
                                                      C.byref(rel2)))
    assert nc > 0 and it2.value == it and abs(rel2.value - rel) <= 1e-15 and np.array_equal(x2, x)
    assert rel2.value <= 1e-10 and np.linalg.norm(A @ x2 - fred) <= 2e-10 * np.linalg.norm(fred)
