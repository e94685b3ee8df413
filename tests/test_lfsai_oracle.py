"""The learned-FSAI oracle (CPU): its analytic gradient against central finite
differences, its starting factor, and the Kaporin objective against the classic
FSAI oracle (the objective's minimiser on a fixed pattern)."""
import numpy as np

from meshes import box
from oracle import lfsai_oracle as L
from oracle import oracle as O


def tiny_system(seed=0):
    c, e = box([3, 2, 2], mx=(1.5, 1.0, 1.0))
    E = np.random.default_rng(seed).uniform(0.1, 1.0, len(e))
    coo = O.assemble_elasticity(O.Mesh(O.CELL_TET, c, e), O.MODEL_3D, E, 0.3, 2)
    x0 = [int(i) for i in O.nodes_on_plane(c, 0, 0.0, 1e-9)]
    kred, fred, free = O.reduce_system(coo, np.zeros(3 * len(c)), [(3 * n + k, 0.0) for n in x0 for k in range(3)])
    k = kred.to_csr()
    # exactly symmetric copy: the network's backward uses A^ for A^T
    import scipy.sparse as sp
    A = sp.csr_matrix((k.values, k.col_ind, k.row_ptrs), shape=(k.nrows, k.nrows))
    A = sp.csr_matrix(0.5 * (A + A.T))
    A.sort_indices()
    csr = O.Csr(A.shape[0], A.shape[0], A.indptr.astype(np.int64), A.indices.astype(np.int64), A.data)
    lrp, lci = O.node_block_lower_pattern(csr, free, 3)
    return csr, free, lrp, lci


def random_params(seed):
    rng = np.random.default_rng(seed)
    p = 0.3 * rng.standard_normal(L.OFF["total"])
    a, _ = L.OFF["w0"]
    p[a] = -1.0
    return p


def test_oracle_gradient_matches_finite_differences():
    csr, free, lrp, lci = tiny_system()
    g = L.Graph(csr.row_ptrs, csr.col_ind, csr.values, free, 3, lrp, lci)
    p = random_params(7)
    loss, grad = L.loss_grad(p, g)
    rng = np.random.default_rng(11)
    idx = rng.choice(len(p), size=60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (L.loss_grad(p + e, g)[0] - L.loss_grad(p - e, g)[0]) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-5 * np.max(np.abs(grad)), (i, fd, grad[i])


def test_initial_parameters_give_first_order_factor():
    csr, free, lrp, lci = tiny_system(1)
    g = L.Graph(csr.row_ptrs, csr.col_ind, csr.values, free, 3, lrp, lci)
    p = np.zeros(L.OFF["total"])
    p[L.OFF["w0"][0]] = -1.0
    f = L.forward(p, g)
    assert np.allclose(f["lhat"], -g.al)
    # diag(G^ A^ G^T) = 1 by construction
    d = (f["G"] @ g.ahat @ f["G"].T).diagonal()
    assert np.allclose(d, 1.0, rtol=1e-12)


def fsai_offdiag(g):
    csr = O.Csr(g.n, g.n, g.ahat.indptr.astype(np.int64), g.ahat.indices.astype(np.int64), g.ahat.data)
    G = O.fsai(csr, (g.lrp, g.lci))
    diag = G.values[G.row_ptrs[1:] - 1]
    off = np.concatenate([G.values[G.row_ptrs[i]:G.row_ptrs[i + 1] - 1] for i in range(g.n)])
    return off / diag[g.lrow], diag


def test_classic_fsai_minimises_the_kaporin_objective():
    csr, free, lrp, lci = tiny_system(2)
    g = L.Graph(csr.row_ptrs, csr.col_ind, csr.values, free, 3, lrp, lci)
    off, diag = fsai_offdiag(g)
    q, w, loss = L.kaporin(g, off)
    # stationarity: the gradient 2 w / (n q) vanishes at the FSAI values
    assert np.max(np.abs(w)) <= 1e-10
    # and the FSAI scaling is the objective's sig = q^-1/2
    assert np.allclose(1.0 / np.sqrt(q), diag, rtol=1e-10)
    rng = np.random.default_rng(5)
    for _ in range(5):
        assert L.kaporin(g, off + 0.05 * rng.standard_normal(off.size))[2] > loss
    assert L.forward(random_params(3), g)["loss"] > loss
