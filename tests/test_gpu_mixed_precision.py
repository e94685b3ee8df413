"""The FP32-inner / FP64-refinement PCG (SOLVER_MP_PCG: FP32 operator values,
vectors and SpMV inside; FP64 true residual, solution accumulation and
refinement outside) against the FP64 oracle, and where it breaks down.

On the well-conditioned unit cube it reaches the FP64 residual target and its
solution agrees with the oracle's FP64 solve.  On the elongated elasticity
cantilevers the FP32 operator cannot resolve the near-rigid-body modes: the
refinement needs far more inner iterations at 40x10x10 and never reaches
1e-10 at 100x25x25, even with a homogeneous modulus, while FP64 Jacobi-PCG
converges.  That is why the headline solver keeps the operator and the
Krylov recurrences in FP64 and puts reduced precision in the preconditioner
(FP16 factor, FP32 coarse inverse).
"""
import numpy as np
import pytest

import tpt_fem as F
from tpt_fem import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def elasticity_system(ctx, mn, mx, n, young):
    mesh = F.Mesh.box_mesh(mn, mx, n, ctx=ctx)
    K = F.assemble_elasticity(mesh, "3d", young, 0.3, 2)
    rhs = F.apply_traction(mesh, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    dof, val = W.clamp_x0_bcs(mesh.coords_array)
    return mesh, K, rhs, dof, F.reduce_system(K, rhs, list(zip(dof, val)))


def test_mp_pcg_on_the_cube_matches_the_fp64_oracle(ctx):
    mesh, K, rhs, dof, S = elasticity_system(ctx, [0, 0, 0], [1, 1, 1], [12, 12, 12], 1.0)
    st = S.solve(solver=F.SOLVER_MP_PCG, tol=1e-10, fresh_setup=True)
    assert st["rel_residual"] <= 1e-10 and st["outer_steps"] >= 2
    rp, ci, va, fred, free = S.download()
    csr = O.Csr(S.n_free, S.n_free, rp, ci, va)
    x_ref, it, rel = O.pcg_jacobi(csr, fred, tol=1e-13)
    assert it > 0 and rel <= 1e-13
    u = S.solution()[free]
    assert np.max(np.abs(u - x_ref)) <= 1e-8 * np.max(np.abs(x_ref))


def test_fp32_operator_falls_behind_then_fails_on_the_cantilever(ctx):
    # 40x10x10 (heterogeneous modulus): converges, with far more iterations
    n = [40, 10, 10]
    *_, S = elasticity_system(ctx, [0, 0, 0], [4, 1, 1], n, W.cantilever_young(n))
    jac = S.solve(solver=F.SOLVER_JACOBI_PCG, tol=1e-10, fresh_setup=True, csr_only=True)
    mp = S.solve(solver=F.SOLVER_MP_PCG, tol=1e-10, fresh_setup=True, max_iter=4 * jac["iterations"])
    assert mp["rel_residual"] <= 1e-10 and mp["iterations"] >= 2 * jac["iterations"]
    # 100x25x25 with E = 1: FP64 converges, the FP32 operator cannot reach 1e-10
    *_, S = elasticity_system(ctx, [0, 0, 0], [4, 1, 1], [100, 25, 25], 1.0)
    jac = S.solve(solver=F.SOLVER_JACOBI_PCG, tol=1e-10, fresh_setup=True, csr_only=True)
    assert jac["rel_residual"] <= 1e-10
    with pytest.raises(F.TptFemError, match="NOT_CONVERGED"):
        S.solve(solver=F.SOLVER_MP_PCG, tol=1e-10, fresh_setup=True, max_iter=4 * jac["iterations"])
