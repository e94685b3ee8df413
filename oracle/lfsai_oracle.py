"""CPU oracle of the learned-FSAI network (TEST INFRASTRUCTURE ONLY).

The reference has no learned preconditioner; this numpy restatement (FP64) of
the device network in tpt-fem_b200/csrc/lfsai.cu is the checker for the
device's forward and backward kernels.  Its own analytic gradient is checked
against central finite differences in tests/test_lfsai_oracle.py.

Network (A^ = D^-1/2 A D^-1/2):
  h0_i  = [1, sum|a^_ij|, sum a^_ij, sum a^_ij^2, onehot(dof component), deg/40]
  h_l+1 = tanh(Ws h_l + Wa (|A^_off| h_l) + Wb (A^_off h_l) + b)
  z_ij  = tanh(U h_i + V h_j + ue a^_ij + ce),  L^_ij = we . z_ij + w0 a^_ij
  g_i   = e_i + L^_i,  q_i = g_i A^ g_i^T,  sig_i = q_i^-1/2
  G^    = diag(sig) (I + L^)          (unit diagonal of G^ A^ G^T)
Objective (Kaporin's condition number of G^ A^ G^T, up to the constant
log det A^ / n):  loss = (1/n) sum_i log q_i.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

D0, H, LAYERS = 8, 16, 2


def offsets():
    o, p = {}, 0
    for l in range(LAYERS):
        din = D0 if l == 0 else H
        for name, size in (("ws", H * din), ("wa", H * din), ("wb", H * din), ("b", H)):
            o[f"{name}{l}"] = (p, size)
            p += size
    for name, size in (("U", H * H), ("V", H * H), ("ue", H), ("ce", H), ("we", H), ("w0", 1)):
        o[name] = (p, size)
        p += size
    o["total"] = p
    return o


OFF = offsets()


def view(params, name, shape=None):
    a, s = OFF[name]
    v = params[a:a + s]
    return v.reshape(shape) if shape else v


class Graph:
    """Matrix-derived inputs of the network for one reduced system."""

    def __init__(self, rp, ci, va, free, dpn, lrp, lci):
        n = len(rp) - 1
        self.n = n
        A = sp.csr_matrix((va, ci, rp), shape=(n, n))
        d = A.diagonal()
        self.dis = 1.0 / np.sqrt(d)
        ah = sp.diags(self.dis) @ A @ sp.diags(self.dis)
        self.ahat = sp.csr_matrix(ah)
        # keep explicit structure of A's off-diagonal entries (zeros included)
        rows = np.repeat(np.arange(n), np.diff(rp))
        m = rows != ci
        vals = va[m] * self.dis[rows[m]] * self.dis[ci[m]]
        self.off = sp.csr_matrix((vals, (rows[m], ci[m])), shape=(n, n))
        self.absoff = sp.csr_matrix((np.abs(vals), (rows[m], ci[m])), shape=(n, n))
        x = np.zeros((n, D0))
        x[:, 0] = 1.0
        x[:, 1] = np.asarray(self.absoff.sum(axis=1)).ravel()
        x[:, 2] = np.asarray(self.off.sum(axis=1)).ravel()
        x[:, 3] = np.asarray(self.off.multiply(self.off).sum(axis=1)).ravel()
        if dpn > 1:
            comp = np.asarray(free) % dpn
            for c in range(3):
                x[:, 4 + c] = comp == c
        x[:, 7] = np.bincount(rows[m], minlength=n) / 40.0
        self.x0 = x
        self.lrp, self.lci = np.asarray(lrp), np.asarray(lci)
        self.lrow = np.repeat(np.arange(n), np.diff(self.lrp))
        full = self.ahat.tocsr()
        self.al = np.asarray(full[self.lrow, self.lci]).ravel() if len(self.lci) else np.zeros(0)


def kaporin(g, lhat):
    """q_i, W = (I + L^) A^ (rows of the pattern) and the loss (1/n) sum log q_i."""
    Gt = sp.csr_matrix(sp.identity(g.n) + sp.csr_matrix((lhat, (g.lrow, g.lci)), shape=(g.n, g.n)))
    W = sp.csr_matrix(Gt @ g.ahat)
    q = np.asarray(W.multiply(Gt).sum(axis=1)).ravel()
    w_lower = np.asarray(W[g.lrow, g.lci]).ravel() if len(g.lci) else np.zeros(0)
    return q, w_lower, float(np.mean(np.log(q)))


def forward(params, g):
    p = params.astype(np.float64)
    acts = []
    x = g.x0
    for l in range(LAYERS):
        din = D0 if l == 0 else H
        ws, wa, wb = (view(p, f"{k}{l}", (H, din)) for k in ("ws", "wa", "wb"))
        b = view(p, f"b{l}")
        ya, yb = g.absoff @ x, g.off @ x
        h = np.tanh(x @ ws.T + ya @ wa.T + yb @ wb.T + b)
        acts.append((x, ya, yb, h))
        x = h
    U, V = view(p, "U", (H, H)), view(p, "V", (H, H))
    P, Q = x @ U.T, x @ V.T
    ue, ce, we, w0 = view(p, "ue"), view(p, "ce"), view(p, "we"), view(p, "w0")[0]
    a = P[g.lrow] + Q[g.lci] + np.outer(g.al, ue) + ce
    z = np.tanh(a)
    lhat = w0 * g.al + z @ we
    q, w_lower, loss = kaporin(g, lhat)
    sig = 1.0 / np.sqrt(q)
    Lh = sp.csr_matrix((lhat, (g.lrow, g.lci)), shape=(g.n, g.n))
    G = sp.diags(sig) @ (sp.identity(g.n) + Lh)
    return dict(G=sp.csr_matrix(G), lhat=lhat, sig=sig, q=q, w_lower=w_lower, loss=loss, P=P, Q=Q, z=z,
                acts=acts, h=x)


def loss_grad(params, g):
    """Kaporin loss (1/n) sum_i log q_i and its gradient with respect to the parameters (FP64)."""
    f = forward(params, g)
    n = g.n
    # d loss / d L^_ij = 2 W_ij / (n q_i)
    dl = 2.0 * f["w_lower"] / (n * f["q"][g.lrow])
    p = params.astype(np.float64)
    grad = np.zeros_like(p)

    def put(name, val):
        a, s = OFF[name]
        grad[a:a + s] += np.asarray(val).ravel()

    z, we, al = f["z"], view(p, "we"), g.al
    put("we", z.T @ dl)
    put("w0", [np.sum(dl * al)])
    da = dl[:, None] * we[None, :] * (1.0 - z * z)
    put("ue", da.T @ al)
    put("ce", da.sum(axis=0))
    dP = np.zeros((n, H))
    dQ = np.zeros((n, H))
    np.add.at(dP, g.lrow, da)
    np.add.at(dQ, g.lci, da)
    h = f["h"]
    put("U", dP.T @ h)
    put("V", dQ.T @ h)
    dH = dP @ view(p, "U", (H, H)) + dQ @ view(p, "V", (H, H))
    for l in reversed(range(LAYERS)):
        din = D0 if l == 0 else H
        x, ya, yb, hl = f["acts"][l]
        dpre = dH * (1.0 - hl * hl)
        put(f"ws{l}", dpre.T @ x)
        put(f"wa{l}", dpre.T @ ya)
        put(f"wb{l}", dpre.T @ yb)
        put(f"b{l}", dpre.sum(axis=0))
        if l > 0:
            ws, wa, wb = (view(p, f"{k}{l}", (H, din)) for k in ("ws", "wa", "wb"))
            dH = dpre @ ws + g.absoff @ (dpre @ wa) + g.off @ (dpre @ wb)
    return f["loss"], grad
