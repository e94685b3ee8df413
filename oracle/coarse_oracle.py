"""CPU oracle of the aggregation coarse space (TEST INFRASTRUCTURE ONLY).

The reference has no iterative solver; this numpy restatement of the device's
coarse space (tpt-fem_b200/csrc/coarse.cu) is the checker for it: free mesh
nodes binned into the given number of boxes per axis over the bounding box of
the free nodes, one aggregate per non-empty box (in box order), the rigid-body
modes of each aggregate about its centroid orthonormalised, P the block
diagonal of those modes and A_c = P^T A P.  The mode basis inside an aggregate
is any orthonormal basis of the same span, so tests compare basis-invariant
quantities (eigenvalues of A_c, the operator P A_c^-1 P^T).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def raw_modes(y, dpn):
    """dpn x nm matrix of raw rigid modes at relative position y."""
    if dpn == 1:
        return np.ones((1, 1))
    if dpn == 2:
        return np.array([[1.0, 0.0, -y[1]], [0.0, 1.0, y[0]]])
    return np.array([[1.0, 0.0, 0.0, 0.0, y[2], -y[1]],
                     [0.0, 1.0, 0.0, -y[2], 0.0, y[0]],
                     [0.0, 0.0, 1.0, y[1], -y[0], 0.0]])


def aggregates(coords, free, dpn, bins):
    """Aggregate of every free node group (binning rule of coarse.cu)."""
    free = np.asarray(free)
    nodes = free[::dpn] // dpn
    pos = np.zeros((len(nodes), 3))
    pos[:, :coords.shape[1]] = coords[nodes]
    lo, hi = pos.min(axis=0), pos.max(axis=0)
    L = hi - lo
    k = np.zeros((len(nodes), 3), dtype=np.int64)
    for d in range(3):
        if L[d] > 0:
            k[:, d] = np.minimum(bins[d] - 1, np.floor((pos[:, d] - lo[d]) / L[d] * bins[d]).astype(np.int64))
    k = np.maximum(k, 0)
    bid = (k[:, 2] * bins[1] + k[:, 1]) * bins[0] + k[:, 0]
    ub, agg = np.unique(bid, return_inverse=True)
    return agg, pos


def prolongation(coords, free, dpn, bins):
    """P (n_free x nc, orthonormal columns per aggregate)."""
    agg, pos = aggregates(coords, free, dpn, bins)
    na = agg.max() + 1
    rows, cols, vals = [], [], []
    nm = {1: 1, 2: 3, 3: 6}[dpn]
    for I in range(na):
        g = np.nonzero(agg == I)[0]
        y = pos[g] - pos[g].mean(axis=0)
        R = np.vstack([raw_modes(yy, dpn) for yy in y])  # (len(g) dpn) x nm
        U, sv, _ = np.linalg.svd(R, full_matrices=False)
        keep = sv > 1e-6 * sv.max()
        Q = U[:, keep]
        r = (g[:, None] * dpn + np.arange(dpn)[None, :]).ravel()
        for j in range(Q.shape[1]):
            rows.append(r)
            cols.append(np.full(len(r), I * nm + j))
            vals.append(Q[:, j])
    n = len(free)
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(n, na * nm)), na, nm


def coarse_matrix(rp, ci, va, coords, free, dpn, bins):
    n = len(rp) - 1
    A = sp.csr_matrix((va, ci, rp), shape=(n, n))
    P, na, nm = prolongation(coords, free, dpn, bins)
    Ac = (P.T @ A @ P).toarray()
    dropped = np.diag(Ac) == 0
    Ac[dropped, dropped] = 1.0
    return Ac, P, na, nm
