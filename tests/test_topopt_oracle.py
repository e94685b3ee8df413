"""Topology-optimisation oracle (CPU) against the reference's own topopt tests
(crates/tpt-fem-topopt/src/lib.rs:421-495) and its internal consistency: the
banded Cholesky solve against the reference's dense-LU path, the windowed
sensitivity filter against the all-pairs definition, and the OC volume
constraint."""
import numpy as np
import pytest

from oracle import oracle as O


def test_ke0_is_symmetric_with_rigid_body_null_space():
    k = O.topopt_ke0(0.3, 1.0)
    assert np.allclose(k, k.T, rtol=0, atol=1e-15)
    # translations x, y and the rotation of the unit square (nodes 00, 10, 11, 01)
    xy = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]])
    for mode in (np.tile([1.0, 0.0], 4), np.tile([0.0, 1.0], 4), np.stack([-xy[:, 1], xy[:, 0]], 1).ravel()):
        assert np.max(np.abs(k @ mode)) < 1e-14
    assert np.all(np.linalg.eigvalsh(k)[3:] > 1e-3)


def test_cantilever_lowers_compliance_and_keeps_volume():
    # topopt:421-452 -- Grid::new(20, 10, 1.0) is 19 x 9 elements
    f, bcs = O.cantilever_load(19, 9)
    comp, rho = O.topopt(19, 9, 0.5, 2.0, 40, f, bcs, banded=False)
    assert len(rho) == 19 * 9 and len(comp) == 41
    assert comp[-1] < comp[0]
    assert abs(rho.sum() - 0.5 * 19 * 9) < 1e-6
    assert np.all(np.diff(comp) <= 1e-9)


def test_full_volume_stays_solid():
    # topopt:454-476
    f, bcs = O.cantilever_load(15, 7)
    comp, rho = O.topopt(15, 7, 1.0, 2.0, 10, f, bcs, banded=False)
    assert abs(rho.sum() - 15 * 7) < 1e-6
    assert np.all(np.abs(rho - 1.0) < 1e-6)


def test_denser_initial_compliance_exceeds_optimized():
    # topopt:478-495
    f, bcs = O.cantilever_load(23, 11)
    comp, _ = O.topopt(23, 11, 0.4, 2.0, 30, f, bcs, banded=False)
    assert comp[-1] < comp[0]


def test_banded_solve_matches_dense_lu_path():
    f, bcs = O.cantilever_load(19, 9)
    c1, r1 = O.topopt(19, 9, 0.5, 2.0, 40, f, bcs, banded=False)
    c2, r2 = O.topopt(19, 9, 0.5, 2.0, 40, f, bcs, banded=True)
    assert np.max(np.abs(c2 - c1) / c1) < 1e-11
    assert np.max(np.abs(r2 - r1)) < 1e-10


@pytest.mark.parametrize("radius", [1.5, 2.0, 2.7])
def test_windowed_filter_equals_all_pairs(radius):
    nelx, nely = 9, 5
    raw = np.random.default_rng(1).standard_normal(nelx * nely)
    c = np.array([[(e % nelx) + 0.5, (e // nelx) + 0.5] for e in range(nelx * nely)])
    ref = np.zeros_like(raw)
    for e in range(len(raw)):  # filter_sensitivity (topopt:259-279), every f in order
        num = den = 0.0
        for f in range(len(raw)):
            d2 = (c[e, 0] - c[f, 0]) ** 2 + (c[e, 1] - c[f, 1]) ** 2
            if d2 <= radius * radius:
                w = radius - np.sqrt(d2)
                num += w * raw[f]
                den += w
        ref[e] = num / den if den > 0 else raw[e]
    assert np.array_equal(O.topopt_filter_sensitivity(nelx, nely, 1.0, raw, radius), ref)


def test_oc_update_meets_volume_and_move_limit():
    rng = np.random.default_rng(2)
    rho = rng.uniform(0.1, 0.9, 200)
    sens = -rng.uniform(0.0, 5.0, 200)
    out = O.topopt_oc_update(rho, sens, 0.5, 0.2)
    assert abs(out.sum() - 100.0) < 1e-6
    assert np.all(out <= rho + 0.2 + 1e-15) and np.all(out >= rho - 0.2 - 1e-15)
    assert np.all(out >= 1e-3) and np.all(out <= 1.0)


def test_density_filter_mode_keeps_physical_volume():
    nelx, nely = 30, 10
    f, bcs = O.cantilever_load(nelx, nely, node=(nelx + 1) * (nely // 2) + nelx)
    comp, rho = O.topopt(nelx, nely, 0.4, 1.5, 20, f, bcs, emin=1e-9, density_filter=True)
    assert comp[-1] < comp[0]
    assert abs(rho.mean() - 0.4) < 1e-3 * 0.4 * 2
