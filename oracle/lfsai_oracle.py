"""CPU oracle of the learned-FSAI network (TEST INFRASTRUCTURE ONLY).

The reference has no learned preconditioner; this numpy restatement (FP64) of
the device network in tpt-fem_b200/csrc/lfsai.cu is the checker for the
device's forward and backward kernels.  Its own analytic gradient is checked
against central finite differences in tests/test_lfsai_oracle.py.
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
    for name, size in (("U", H * H), ("V", H * H), ("ue", H), ("ce", H), ("we", H), ("w0", 1), ("q", H),
                       ("q0", 1)):
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
        off = self.ahat - sp.diags(self.ahat.diagonal())
        off.eliminate_zeros()
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


def forward(params, g, keep=False):
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
    rho = x @ view(p, "q") + view(p, "q0")[0]
    sig = np.exp(0.5 * rho)
    ue, ce, we, w0 = view(p, "ue"), view(p, "ce"), view(p, "we"), view(p, "w0")[0]
    a = P[g.lrow] + Q[g.lci] + np.outer(g.al, ue) + ce
    z = np.tanh(a)
    lhat = w0 * g.al + z @ we
    Lh = sp.csr_matrix((lhat, (g.lrow, g.lci)), shape=(g.n, g.n))
    G = sp.diags(sig) @ (sp.identity(g.n) + Lh)
    out = dict(G=sp.csr_matrix(G), lhat=lhat, sig=sig, P=P, Q=Q, z=z, acts=acts, h=x)
    return out


def loss_grad(params, g, Z):
    """Loss = mean over entries of (G^ A^ G^T Z - Z)^2 and its gradient (FP64)."""
    f = forward(params, g)
    G, A = f["G"], g.ahat
    n, m = Z.shape
    U1 = G.T @ Z
    V1 = A @ U1
    W1 = G @ V1
    E = W1 - Z
    loss = float(np.sum(E * E) / (n * m))
    GW = 2.0 * E / (n * m)
    GV = G.T @ GW
    GU = A @ GV
    sig, lhat = f["sig"], f["lhat"]
    dGdiag = np.sum(GW * V1, axis=1) + np.sum(Z * GU, axis=1)
    dGoff = np.sum(GW[g.lrow] * V1[g.lci], axis=1) + np.sum(Z[g.lrow] * GU[g.lci], axis=1)
    dl = sig[g.lrow] * dGoff
    dsig = dGdiag + np.bincount(g.lrow, weights=lhat * dGoff, minlength=n)
    drho = 0.5 * sig * dsig
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
    put("q", h.T @ drho)
    put("q0", [drho.sum()])
    dH = dP @ view(p, "U", (H, H)) + dQ @ view(p, "V", (H, H)) + np.outer(drho, view(p, "q"))
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
    return loss, grad
