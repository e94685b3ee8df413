"""Two-level (FSAI + aggregation coarse space) solves on the GPU: the coarse
matrix against the CPU oracle's P^T A P, convergence to the FP64 tolerance,
agreement with the plain method, and the iterations it saves."""
import numpy as np
import pytest

import tpt_fem as F
from tpt_fem import lfsai as LF
from tpt_fem import workloads as W
from meshes import box, jitter
from oracle import coarse_oracle as CO
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def cantilever(ctx, n, seed=3, jit=0.0):
    mn, mx = [0.0, 0.0, 0.0], [4.0, 1.0, 1.0]
    c, e = box(n, mn=mn, mx=mx)
    if jit:
        c = jitter(c, jit, seed)
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", W.cantilever_young(n, seed=seed), 0.3, 2)
    rhs = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    dof, val = W.clamp_x0_bcs(c)
    return F.reduce_system(K, rhs, list(zip(dof, val))), c


@pytest.mark.parametrize("jit,n,aggs,tol", [(0.0, [12, 4, 4], 12, 1e-12), (0.02, [12, 4, 4], 12, 1e-12),
                                             (0.0, [40, 8, 8], 160, 1e-10)])
def test_coarse_matrix_matches_oracle(ctx, jit, n, aggs, tol):
    # the last case's coarse matrix spans several 64 x 64 tiles of the dense inverse
    S, c = cantilever(ctx, n, jit=jit)
    st = S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=tol, coarse=True, coarse_aggregates=aggs)
    assert st["coarse_size"] > 0 and st["rel_residual"] <= tol
    info = S.coarse(with_inverse=True)
    rp, ci, va, fred, free = S.download()
    Ac, P, na, nm = CO.coarse_matrix(rp, ci, va, c, free, 3, info["bins"])
    assert (info["na"], info["nm"]) == (na, nm) and st["coarse_size"] == na * nm
    ev_dev = np.sort(1.0 / np.linalg.eigvalsh(0.5 * (info["ainv"] + info["ainv"].T)))
    ev_orc = np.sort(np.linalg.eigvalsh(Ac))
    assert np.allclose(ev_dev, ev_orc, rtol=2e-4, atol=1e-6 * ev_orc.max())


def test_two_level_solution_and_iterations(ctx):
    S, c = cantilever(ctx, [32, 8, 8])
    one = S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=1e-10)
    u1 = S.solution()
    two = S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=1e-10, coarse=True, coarse_aggregates=64, fresh_setup=True)
    u2 = S.solution()
    # direct solve of the same reduced system (scipy sparse LU) as the reference solution
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    rp, ci, va, fred, free = S.download()
    A = sp.csc_matrix(sp.csr_matrix((va, ci, rp), shape=(len(fred), len(fred))))
    x = spl.spsolve(A, fred)
    assert two["coarse_size"] > 0 and two["rel_residual"] <= 1e-10
    assert two["iterations"] < 0.5 * one["iterations"]
    scale = np.max(np.abs(x))
    assert np.max(np.abs(u2[free] - x)) <= 1e-6 * scale and np.max(np.abs(u1[free] - x)) <= 1e-6 * scale
    # deterministic: the same solve twice gives the same bits
    again = S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=1e-10, coarse=True, coarse_aggregates=64, fresh_setup=True)
    assert again["iterations"] == two["iterations"] and np.array_equal(S.solution(), u2)
    # a different aggregate count rebuilds the coarse space on the same system
    other = S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=1e-10, coarse=True, coarse_aggregates=16, fresh_setup=True)
    assert not other["fell_back"] and 0 < other["coarse_size"] < two["coarse_size"]
    assert other["rel_residual"] <= 1e-10 and other["iterations"] < one["iterations"]
    back = S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=1e-10, coarse=True, coarse_aggregates=64, fresh_setup=True)
    assert back["iterations"] == two["iterations"] and np.array_equal(S.solution(), u2)


def test_learned_two_level(ctx):
    S, c = cantilever(ctx, [32, 8, 8], seed=5)
    model = LF.LearnedFsai(ctx, seed=1)
    model.attach(S)
    one = S.solve(solver=F.SOLVER_LEARNED_FSAI_PCG, tol=1e-10, fresh_setup=True)
    two = S.solve(solver=F.SOLVER_LEARNED_FSAI_PCG, tol=1e-10, fresh_setup=True, coarse=True, coarse_aggregates=64)
    assert not two["fell_back"] and two["coarse_size"] > 0 and two["rel_residual"] <= 1e-10
    assert two["iterations"] < 0.5 * one["iterations"]


def test_poisson_coarse_space(ctx):
    c, e = box([16, 16, 16])
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    k = np.exp(np.random.default_rng(2).normal(0.0, 1.0, len(e)))
    K = F.assemble_poisson(m, k, 2)
    rhs = F.load_poisson_source(m, 1.0, 2)
    on_b = np.nonzero(np.any((c < 1e-9) | (c > 1 - 1e-9), axis=1))[0]
    S = F.reduce_system(K, rhs, [(int(i), 0.0) for i in on_b])
    one = S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=1e-10)
    two = S.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=1e-10, coarse=True, coarse_aggregates=27, fresh_setup=True)
    assert two["coarse_size"] > 0 and two["rel_residual"] <= 1e-10
    assert two["iterations"] < one["iterations"]
    info = S.coarse(with_inverse=True)
    rp, ci, va, fred, free = S.download()
    Ac, P, na, nm = CO.coarse_matrix(rp, ci, va, c, free, 1, info["bins"])
    ev_dev = np.sort(1.0 / np.linalg.eigvalsh(0.5 * (info["ainv"] + info["ainv"].T)))
    assert np.allclose(ev_dev, np.sort(np.linalg.eigvalsh(Ac)), rtol=2e-4)


def test_coarse_not_applicable_runs_without_it(ctx):
    # a roller support fixes one component only: partial node groups, no node-block layout
    S, c = cantilever(ctx, [8, 3, 3])
    c2, e = box([8, 3, 3], mn=[0.0, 0.0, 0.0], mx=[4.0, 1.0, 1.0])
    m = F.Mesh.from_arrays(F.CELL_TET4, c2, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", 1.0, 0.3, 2)
    rhs = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    x0 = [int(i) for i in O.nodes_on_plane(c2, 0, 0.0, 1e-9)]
    bcs = [(3 * n, 0.0) for n in x0] + [(3 * x0[0] + 1, 0.0), (3 * x0[0] + 2, 0.0), (3 * x0[1] + 2, 0.0),
                                        (3 * x0[-1] + 1, 0.0), (3 * x0[-1] + 2, 0.0)]
    S2 = F.reduce_system(K, rhs, bcs)
    st = S2.solve(solver=F.SOLVER_FSAI_MP_PCG, tol=1e-10, coarse=True)
    assert st["coarse_size"] == 0 and st["rel_residual"] <= 1e-10


def test_refresh_matches_a_freshly_reduced_system(ctx):
    # new coefficients on the same mesh: refreshed values equal a new reduction bit for bit,
    # and every method solves the refreshed system as it solves the new one
    mn, mx, n = [0.0, 0.0, 0.0], [4.0, 1.0, 1.0], [16, 4, 4]
    c, e = box(n, mn=mn, mx=mx)
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    dof, val = W.clamp_x0_bcs(c)
    bcs = list(zip(dof, val))
    K1 = F.assemble_elasticity(m, "3d", W.cantilever_young(n, seed=1), 0.3, 2)
    rhs1 = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K1.nrows))
    S = F.reduce_system(K1, rhs1, bcs)
    model = LF.LearnedFsai(ctx, seed=2)
    model.attach(S)
    kinds = [dict(solver=F.SOLVER_JACOBI_PCG, csr_only=True), dict(solver=F.SOLVER_FSAI_MP_PCG, coarse=True),
             dict(solver=F.SOLVER_LEARNED_FSAI_PCG, coarse=True), dict(solver=F.SOLVER_JACOBI_PCG)]
    for kw in kinds:
        S.solve(tol=1e-10, **kw)
    K2 = F.assemble_elasticity(m, "3d", W.cantilever_young(n, seed=2), 0.3, 2)
    rhs2 = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -2e-3], np.zeros(K2.nrows))
    S.refresh(K2, rhs2)
    T = F.reduce_system(K2, rhs2, bcs)
    model.attach(T)
    for a, b in zip(S.download(), T.download()):
        assert np.array_equal(a, b)
    for kw in kinds:
        sa = S.solve(tol=1e-10, **kw)
        ua = S.solution()
        sb = T.solve(tol=1e-10, **kw)
        ub = T.solution()
        assert sa["rel_residual"] <= 1e-10 and not sa["fell_back"]
        assert sa["iterations"] == sb["iterations"] and np.array_equal(ua, ub)
    # a matrix with another pattern is rejected
    K3 = F.assemble_elasticity(F.Mesh.from_arrays(F.CELL_TET4, *box([8, 2, 2]), ctx=ctx), "3d", 1.0, 0.3, 2)
    with pytest.raises(F.TptFemError):
        S.refresh(K3, np.zeros(K3.nrows))


def test_overlapped_coarse_setup_repeats_bit_for_bit(ctx):
    # Fresh set-ups after the first form the coarse matrix and its inverse on a
    # second stream while the network computes the factor: every repeat must
    # give the same iterations and the same solution bits as the first solve,
    # whose set-up ran on one stream.
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    model = LF.LearnedFsai.load(ctx, os.path.join(root, "tpt-fem_b200", "weights", "lfsai_elasticity.bin"))
    S, _ = cantilever(ctx, [48, 12, 12], seed=11)
    model.attach(S)
    runs = []
    for _ in range(3):
        st = S.solve(solver=F.SOLVER_LEARNED_FSAI_PCG, tol=1e-10, fresh_setup=True, coarse=True)
        assert st["coarse_size"] > 0 and st["rel_residual"] <= 1e-10 and not st["fell_back"]
        runs.append((st["iterations"], S.solution()))
    for it, u in runs[1:]:
        assert it == runs[0][0] and np.array_equal(u, runs[0][1])


def test_alternating_coarse_on_and_off_repeats_bit_for_bit(ctx):
    # Solves that switch the coarse space on and off share one engine, which
    # keeps the captured graph of the other setting: each setting must give
    # the same iterations and solution bits every time it comes back.
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    model = LF.LearnedFsai.load(ctx, os.path.join(root, "tpt-fem_b200", "weights", "lfsai_elasticity.bin"))
    S, _ = cantilever(ctx, [40, 10, 10], seed=13)
    model.attach(S)
    seen = {}
    for coarse in (True, False, True, False, True):
        st = S.solve(solver=F.SOLVER_LEARNED_FSAI_PCG, tol=1e-10, fresh_setup=True, coarse=coarse)
        assert st["rel_residual"] <= 1e-10 and not st["fell_back"] and (st["coarse_size"] > 0) == coarse
        got = (st["iterations"], S.solution())
        if coarse in seen:
            assert got[0] == seen[coarse][0] and np.array_equal(got[1], seen[coarse][1])
        else:
            seen[coarse] = got
    assert seen[True][0] < seen[False][0]
