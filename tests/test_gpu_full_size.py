"""The benchmark workloads at their full sizes, through properties that do
not depend on size: exact pattern sizes (the nnz counts the reference's
to_csr gives for these meshes), symmetry and the rigid-body null space of
the assembled operators, load totals, and solutions to the stated tolerance
whose residual is re-checked on the host from the downloaded matrix."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import tpt_fem as F
from tpt_fem import lfsai as LF
from tpt_fem import workloads as W

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WEIGHTS = os.path.join(ROOT, "tpt-fem_b200", "weights")


def csr(K):
    rp, ci, va = K.to_csr()
    return sp.csr_matrix((va, ci, rp), shape=(K.nrows, K.nrows))


def reduced_csr(S):
    rp, ci, va, fred, _ = S.download()
    return sp.csr_matrix((va, ci, rp), shape=(S.n_free, S.n_free)), fred


def check_operator(A, dpn, rng):
    x, y = rng.standard_normal(A.shape[0]), rng.standard_normal(A.shape[0])
    scale = np.abs(A).sum(axis=1).max() * np.linalg.norm(x) * np.linalg.norm(y)
    assert abs(x @ (A @ y) - y @ (A @ x)) <= 1e-13 * scale
    for c in range(dpn):  # translations span the null space of the unconstrained operator
        t = np.zeros(A.shape[0])
        t[c::dpn] = 1.0
        assert np.linalg.norm(A @ t) <= 1e-12 * np.abs(A).sum(axis=1).max() * np.sqrt(A.shape[0])


def test_elasticity_unit_cube_64(ctx):
    m = F.Mesh.box_mesh([0, 0, 0], [1, 1, 1], [64, 64, 64], ctx=ctx)
    K = F.assemble_elasticity(m, "3d", 1.0, 0.3, 2)
    assert (K.nrows, K.nnz) == (823875, 29801277)
    check_operator(csr(K), 3, np.random.default_rng(1))
    rhs = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    assert abs(rhs[2::3].sum() + 1e-3) < 1e-15 and not rhs[0::3].any()
    dof, val = W.clamp_x0_bcs(m.coords_array)
    assert len(dof) == 12675
    S = F.reduce_system(K, rhs, list(zip(dof, val)))
    assert S.n_free == 811200
    model = LF.LearnedFsai.load(ctx, os.path.join(WEIGHTS, "lfsai_elasticity.bin"))
    model.attach(S)
    st = S.solve(solver=F.SOLVER_LEARNED_FSAI_PCG, tol=1e-10, coarse=True)
    assert not st["fell_back"] and st["rel_residual"] <= 1e-10
    A, fred = reduced_csr(S)
    u = S.solution()
    free = np.setdiff1d(np.arange(K.nrows), dof)
    assert np.linalg.norm(fred - A @ u[free]) <= 2e-10 * np.linalg.norm(fred)


def test_poisson_grf_128(ctx):
    prob = W.GrfPoisson(ctx, 128)
    K = prob.matrix(5000)
    assert K.nnz == 14926977
    check_operator(csr(K), 1, np.random.default_rng(2))
    assert abs(prob.rhs.sum() - 1.0) < 1e-9  # unit source over the unit cube
    S = F.reduce_system(K, prob.rhs, prob.bcs)
    model = LF.LearnedFsai.load(ctx, os.path.join(WEIGHTS, "lfsai_poisson.bin"))
    model.attach(S)
    st = S.solve(solver=F.SOLVER_LEARNED_FSAI_PCG, tol=1e-8, coarse=True)
    assert not st["fell_back"] and st["rel_residual"] <= 1e-8
    A, fred = reduced_csr(S)
    u = S.solution()
    free = np.setdiff1d(np.arange(K.nrows), [d for d, _ in prob.bcs])
    assert np.linalg.norm(fred - A @ u[free]) <= 2e-8 * np.linalg.norm(fred)


def test_cantilever_280x70x70(ctx):
    mn, mx, n = W.CANTILEVERS["cantilever_280x70x70"]
    m = F.Mesh.box_mesh(mn, mx, n, ctx=ctx)
    assert (m.n_nodes, m.n_elems) == (1416521, 8232000)
    K = F.assemble_elasticity(m, "3d", W.cantilever_young(n), 0.3, 2)
    assert (K.nrows, K.nnz) == (4249563, 154811997)
    rhs = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    assert abs(rhs[2::3].sum() + 1e-3) < 1e-15
    dof, val = W.clamp_x0_bcs(m.coords_array)
    S = F.reduce_system(K, rhs, list(zip(dof, val)))
    assert (S.n_free, S.nnz) == (4234440, 154260946)
    model = LF.LearnedFsai.load(ctx, os.path.join(WEIGHTS, "lfsai_elasticity.bin"))
    model.attach(S)
    st = S.solve(solver=F.SOLVER_LEARNED_FSAI_PCG, tol=1e-10, coarse=True)
    assert not st["fell_back"] and st["rel_residual"] <= 1e-10 and st["iterations"] < 400
    A, fred = reduced_csr(S)
    u = S.solution()
    free = np.setdiff1d(np.arange(K.nrows), dof)
    # naive FP64 summation of the recheck reads up to ~1.4e-10 at this conditioning
    assert np.linalg.norm(fred - A @ u[free]) <= 3e-10 * np.linalg.norm(fred)
