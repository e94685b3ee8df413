"""Batched topology optimisation on the GPU against the oracle restatement of
the reference's topopt_simp (crates/tpt-fem-topopt/src/lib.rs:342-385), its own
tests (topopt:421-495), and batch independence."""
import numpy as np
import pytest

import tpt_fem as F
from tpt_fem import topopt as T
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12  # displacement solve tolerance used for parity


def params(nelx, nely, vf, radius, iters, **kw):
    return T.TopOptParams(grid=T.Grid(nelx + 1, nely + 1, 1.0), vol_frac=vf, filter_radius=radius, max_iter=iters, **kw)


def test_element_stiffness_is_bit_exact():
    for nu, h in ((0.3, 1.0), (0.25, 0.5)):
        assert np.array_equal(T.element_stiffness_unit(nu, h), O.topopt_ke0(nu, h))


def check_against_oracle(res, P, f, bcs, rtol_c=1e-8, atol_rho=1e-7):
    emin = T.E_MIN_FACTOR * P.e0 if P.emin is None else P.emin
    oc, orho = O.topopt(P.grid.nelx, P.grid.nely, P.vol_frac, P.filter_radius, P.max_iter, f, bcs, h=P.grid.h,
                        e0=P.e0, nu=P.nu, penal=P.penal, move_limit=P.move_limit, emin=emin,
                        density_filter=P.density_filter)
    assert np.max(np.abs(res.compliance - oc) / np.abs(oc)) <= rtol_c
    assert np.max(np.abs(res.densities - orho)) <= atol_rho


def test_reference_cantilever_test(ctx):
    # topopt:421-452 through the GPU path, and against the oracle
    P = params(19, 9, 0.5, 2.0, 40)
    f, bcs = T.cantilever_load(P.grid)
    res = T.topopt_simp(P, f, bcs, ctx=ctx, rel_tol=TOL)
    assert len(res.densities) == P.grid.n_elem() and len(res.compliance) == 41
    assert res.compliance[-1] < res.compliance[0]
    assert abs(res.densities.sum() - 0.5 * P.grid.n_elem()) < 1e-6
    assert np.all(np.diff(res.compliance) <= 1e-9)
    check_against_oracle(res, P, f, bcs)


def test_reference_full_volume_and_denser_tests(ctx):
    # topopt:454-476 and topopt:478-495
    P1 = params(15, 7, 1.0, 2.0, 10)
    P2 = params(23, 11, 0.4, 2.0, 30)
    f1, b1 = T.cantilever_load(P1.grid)
    f2, b2 = T.cantilever_load(P2.grid)
    (r1, r2), _ = T.topopt_batch(ctx, [(P1, f1, b1), (P2, f2, b2)], rel_tol=TOL)
    assert abs(r1.densities.sum() - P1.grid.n_elem()) < 1e-6 and np.all(np.abs(r1.densities - 1.0) < 1e-6)
    assert r2.compliance[-1] < r2.compliance[0]
    check_against_oracle(r1, P1, f1, b1)
    check_against_oracle(r2, P2, f2, b2)


def test_density_filter_mode_matches_oracle(ctx):
    # the batched workload's settings: Emin 1e-9, density filter R 1.5, mid-right load
    P = params(60, 20, 0.4, 1.5, 100, emin=1e-9, density_filter=True)
    f, bcs = T.cantilever_load(P.grid, node=P.grid.nx * (P.grid.nely // 2) + P.grid.nelx)
    res = T.topopt_simp(P, f, bcs, ctx=ctx, rel_tol=TOL)
    assert res.compliance[-1] < 0.5 * res.compliance[0]
    check_against_oracle(res, P, f, bcs, rtol_c=1e-6, atol_rho=1e-5)


def test_batch_equals_single_runs_and_uneven_sizes(ctx):
    rng = np.random.default_rng(3)
    probs = []
    for k, (nx, ny) in enumerate([(12, 4), (30, 10), (18, 6), (24, 8), (12, 4)]):
        P = params(nx, ny, float(rng.uniform(0.3, 0.5)), 1.5, 15 + 5 * k, density_filter=bool(k % 2))
        f, bcs = T.cantilever_load(P.grid, node=P.grid.nx * (ny // 2) + nx)
        probs.append((P, f, bcs))
    batch, st = T.topopt_batch(ctx, probs, rel_tol=TOL, block_threads=256)
    assert st["block_threads"] == 256 and st["not_converged"] == 0
    for (P, f, bcs), r in zip(probs, batch):
        single, _ = T.topopt_batch(ctx, [(P, f, bcs)], rel_tol=TOL, block_threads=256)
        assert np.array_equal(single[0].compliance, r.compliance)
        assert np.array_equal(single[0].densities, r.densities)
        check_against_oracle(r, P, f, bcs, rtol_c=1e-7, atol_rho=1e-6)


def test_block_sizes_agree_and_autotuner_reports(ctx):
    P = params(40, 12, 0.45, 1.5, 20)
    f, bcs = T.cantilever_load(P.grid)
    outs = [T.topopt_batch(ctx, [(P, f, bcs)], rel_tol=TOL, block_threads=nt)[0][0] for nt in (256, 512, 1024)]
    for o in outs[1:]:
        assert np.max(np.abs(o.compliance - outs[0].compliance) / outs[0].compliance) < 1e-9
    res, st = T.topopt_batch(ctx, [(P, f, bcs)], rel_tol=TOL)
    assert st["block_threads"] in (256, 512, 1024)
    _, st2 = T.topopt_batch(ctx, [(P, f, bcs)], rel_tol=TOL)
    assert st2["tune_ms"] == 0.0 and st2["block_threads"] == st["block_threads"]


def test_nonzero_dirichlet_values_and_duplicates(ctx):
    # lifting uses the first (dof, value) pair, the solution the last (assembly:525, 555-557)
    P = params(8, 4, 0.5, 1.5, 5)
    f, bcs = T.cantilever_load(P.grid)
    bcs = [(d, 0.01 * (i % 3)) for i, (d, _) in enumerate(bcs)] + [(bcs[1][0], 0.02)]
    res = T.topopt_simp(P, f, bcs, ctx=ctx, rel_tol=TOL)
    check_against_oracle(res, P, f, bcs)


def test_zero_iterations_and_invalid_input(ctx):
    P = params(10, 5, 0.5, 1.5, 0)
    f, bcs = T.cantilever_load(P.grid)
    res = T.topopt_simp(P, f, bcs, ctx=ctx, rel_tol=TOL)
    oc, orho = O.topopt(10, 5, 0.5, 1.5, 0, f, bcs)
    assert len(res.compliance) == 1 and abs(res.compliance[0] - oc[0]) <= 1e-9 * oc[0]
    assert np.all(res.densities == 0.5)
    bad = params(10, 5, 1.5, 1.5, 3)
    with pytest.raises(F.TptFemError):
        T.topopt_simp(bad, f, bcs, ctx=ctx)
    with pytest.raises(F.TptFemError):
        T.topopt_simp(P, f, [(10 ** 6, 0.0)], ctx=ctx)


def test_two_level_and_plain_jacobi_agree(ctx):
    # the per-instance coarse space changes the iterations, not the optimisation
    probs = []
    for nx, ny in [(60, 20), (36, 12)]:
        P = params(nx, ny, 0.4, 1.5, 30, emin=1e-9, density_filter=True)
        f, bcs = T.cantilever_load(P.grid, node=P.grid.nx * (ny // 2) + nx)
        probs.append((P, f, bcs))
    two, st2 = T.topopt_batch(ctx, probs, rel_tol=TOL, pcg_only=True)
    one, st1 = T.topopt_batch(ctx, probs, rel_tol=TOL, plain_jacobi=True, pcg_only=True)
    assert st1["direct_instances"] == 0 and st2["direct_instances"] == 0
    assert st2["pcg_iterations"] < 0.75 * st1["pcg_iterations"]
    for a, b in zip(two, one):
        assert np.max(np.abs(a.compliance - b.compliance) / b.compliance) < 1e-8
        assert np.max(np.abs(a.densities - b.densities)) < 1e-7


def test_banded_cholesky_and_pcg_agree(ctx):
    # the default direct solve (banded Cholesky + refinement) against two-level PCG,
    # both to a 1e-12 residual, on grids banded along y (wide) and along x (tall)
    probs = []
    for nx, ny, dens in [(60, 20, True), (9, 31, False), (33, 12, True), (1, 5, False)]:
        P = params(nx, ny, 0.4, 1.5, 12, emin=1e-9 if dens else None, density_filter=dens)
        f, bcs = T.cantilever_load(P.grid, node=P.grid.nx * (ny // 2) + nx)
        probs.append((P, f, bcs))
    d, std = T.topopt_batch(ctx, probs, rel_tol=TOL)
    p, stp = T.topopt_batch(ctx, probs, rel_tol=TOL, pcg_only=True)
    assert std["direct_instances"] == len(probs) and std["not_converged"] == 0
    assert std["pcg_iterations"] == 0 and stp["pcg_iterations"] > 0
    for a, b in zip(d, p):
        assert np.max(np.abs(a.compliance - b.compliance) / b.compliance) < 1e-9
        assert np.max(np.abs(a.densities - b.densities)) < 1e-7


def test_wide_grids_fall_back_to_pcg_in_the_same_batch(ctx):
    # 112 x 112 elements: half-bandwidth 2 * 113 + 3 = 229 > 224, solved by PCG
    probs = []
    for nx, ny in [(112, 112), (24, 8)]:
        P = params(nx, ny, 0.5, 1.5, 2)
        f, bcs = T.cantilever_load(P.grid)
        probs.append((P, f, bcs))
    res, st = T.topopt_batch(ctx, probs, rel_tol=1e-10)
    assert st["direct_instances"] == 1 and st["not_converged"] == 0 and st["pcg_iterations"] > 0
    single, _ = T.topopt_batch(ctx, [probs[1]], rel_tol=1e-10)
    assert np.max(np.abs(single[0].compliance - res[1].compliance) / res[1].compliance) < 1e-12
    check_against_oracle(res[1], *probs[1])


def test_largest_batch_grid_direct_matches_pcg(ctx):
    # the batched workload's largest grid (240 x 80 elements, 39,042 dofs, half-bandwidth 165):
    # banded Cholesky without refinement against two-level PCG, both to 1e-11
    P = params(240, 80, 0.4, 1.5, 3, emin=1e-9, density_filter=True)
    f, bcs = T.cantilever_load(P.grid, node=P.grid.nx * (P.grid.nely // 2) + P.grid.nelx)
    d, std = T.topopt_batch(ctx, [(P, f, bcs)], rel_tol=1e-11)
    p, stp = T.topopt_batch(ctx, [(P, f, bcs)], rel_tol=1e-11, pcg_only=True)
    assert std["direct_instances"] == 1 and std["refinement_steps"] == 0 and std["not_converged"] == 0
    assert stp["direct_instances"] == 0 and stp["not_converged"] == 0
    assert np.max(np.abs(d[0].compliance - p[0].compliance) / p[0].compliance) < 1e-9
    assert np.max(np.abs(d[0].densities - p[0].densities)) < 1e-7
