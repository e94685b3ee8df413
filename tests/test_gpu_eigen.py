"""Lanczos and power iteration on device matrices (crates/tpt-fem-eigen/src/
lib.rs:62-262) against the numpy restatement in oracle/eigen_oracle.py and
against dense eigen-decompositions."""
import numpy as np
import pytest
import scipy.sparse as sp

import tpt_fem as F
from meshes import box, jitter, tri_grid
from oracle import eigen_oracle as G

pytestmark = pytest.mark.gpu


def dense(K):
    rp, ci, va = K.to_csr()
    return sp.csr_matrix((va, ci, rp), shape=(K.nrows, K.nrows))


@pytest.fixture
def tri_poisson(ctx):
    c, e = tri_grid(6, 4, 1.5, 1.0)
    c = jitter(c, 0.05, 21)
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    return F.assemble_poisson(m, np.linspace(0.5, 2.0, len(e)), 2)


def test_full_basis_gives_the_spectrum(tri_poisson):
    K = tri_poisson
    A = dense(K).toarray()
    ref = np.linalg.eigvalsh(A)
    small = K.lanczos_eigs(4, "smallest", K.nrows)
    large = K.lanczos_eigs(4, "largest", K.nrows)
    assert np.allclose([v for v, _ in small], ref[:4], atol=1e-9 * ref[-1])
    assert np.allclose([v for v, _ in large], ref[::-1][:4], atol=1e-9 * ref[-1])
    for v, x in small + large:
        assert abs(np.linalg.norm(x) - 1.0) < 1e-12
        assert np.linalg.norm(A @ x - v * x) < 1e-7 * ref[-1]


@pytest.mark.parametrize("dim", [12, 25])
def test_ritz_values_match_oracle(tri_poisson, dim):
    K = tri_poisson
    got = K.lanczos_eigs(3, "largest", dim)
    want = G.lanczos_eigs(dense(K), 3, True, dim)
    assert len(got) == len(want) == 3
    for (gv, gx), (wv, wx) in zip(got, want):
        assert abs(gv - wv) <= 1e-10 * abs(wv)
        assert min(np.linalg.norm(gx - wx), np.linalg.norm(gx + wx)) < 1e-7


def test_elasticity_largest_modes(ctx):
    c, e = box([3, 3, 2])
    m = F.Mesh.from_arrays(F.CELL_TET4, jitter(c, 0.04, 5), e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", 1.0, 0.3, 2)
    got = K.lanczos_eigs(2, "largest", 40, vectors=False)
    want = G.lanczos_eigs(dense(K), 2, True, 40)
    for (gv, _), (wv, _) in zip(got, want):
        assert abs(gv - wv) <= 1e-10 * abs(wv)


def test_power_iteration_matches_oracle(tri_poisson):
    K = tri_poisson
    lam, x, it = K.power_iteration(500, 1e-10)
    wl, wx = G.power_iteration(dense(K), 500, 1e-10)
    assert abs(lam - wl) <= 1e-12 * abs(wl) and np.linalg.norm(x - wx) < 1e-8
    assert abs(lam - np.linalg.eigvalsh(dense(K).toarray())[-1]) < 1e-6 * lam
