"""The eigen oracle against the reference's own tests
(crates/tpt-fem-eigen/src/lib.rs:561-623), restated."""
import numpy as np

from oracle import eigen_oracle as G


def test_power_iteration_dominant():  # eigen:562
    a = np.array([[2.0, 1.0], [1.0, 2.0]])
    lam, v = G.power_iteration(a, 200, 1e-12)
    assert abs(lam - 3.0) < 1e-8
    assert np.linalg.norm(a @ v - lam * v) < 1e-6


def test_lanczos_1d_laplacian():  # eigen:596
    n = 10
    a = 2.0 * np.eye(n) - np.eye(n, k=1) - np.eye(n, k=-1)
    small = G.lanczos_eigs(a, 1, False, n)
    assert abs(small[0][0] - (2.0 - 2.0 * np.cos(np.pi / (n + 1)))) < 1e-6
    large = G.lanczos_eigs(a, 1, True, n)
    assert abs(large[0][0] - (2.0 - 2.0 * np.cos(np.pi * n / (n + 1)))) < 1e-6


def test_ritz_pairs_are_eigenpairs_for_a_full_basis():
    rng = np.random.default_rng(0)
    b = rng.normal(size=(12, 12))
    a = b @ b.T + 12 * np.eye(12)
    for val, vec in G.lanczos_eigs(a, 3, True, 12):
        assert np.linalg.norm(a @ vec - val * vec) < 1e-8 * abs(val)
