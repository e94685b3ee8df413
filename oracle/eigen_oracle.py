"""Test-only restatement of crates/tpt-fem-eigen/src/lib.rs in numpy:
lanczos (lib.rs:134-164, one modified Gram-Schmidt pass), the cyclic Jacobi
method (lib.rs:166-214), lanczos_eigs (lib.rs:223-262) and power_iteration
(lib.rs:62-88).  It checks the device library's tptfem_lanczos_eigs and
tptfem_power_iteration; it is never part of the product.  `A` is a
scipy.sparse matrix or a dense array."""
import numpy as np


def _mv(A, x):
    return A @ x


def lanczos(A, m):
    n = A.shape[0]
    v0 = np.zeros(n)
    v0[0] = 1.0
    basis, alpha, beta = [v0], [], []
    for j in range(m):
        w = _mv(A, basis[j])
        a = float(w @ basis[j])
        for k in range(j + 1):
            p = float(w @ basis[k])
            w = w - p * basis[k]
        alpha.append(a)
        if j + 1 == m:
            break
        b = float(np.sqrt(w @ w))
        if b < 1e-12:
            break
        beta.append(b)
        basis.append(w / b)
    return basis, alpha, beta


def jacobi(a, max_sweeps=200):
    a = [list(r) for r in a]
    n = len(a)
    v = [[1.0 if i == j else 0.0 for j in range(n)] for i in range(n)]
    for _ in range(max_sweeps):
        changed = False
        for p in range(n):
            for q in range(p + 1, n):
                if abs(a[p][q]) > 1e-12:
                    changed = True
                    theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q])
                    t = 1.0 / (theta + np.sqrt(1.0 + theta * theta)) if theta >= 0.0 else \
                        1.0 / (theta - np.sqrt(1.0 + theta * theta))
                    c = 1.0 / np.sqrt(1.0 + t * t)
                    s = t * c
                    for i in range(n):
                        aip, aiq = a[i][p], a[i][q]
                        a[i][p] = c * aip - s * aiq
                        a[i][q] = s * aip + c * aiq
                    for i in range(n):
                        api, aqi = a[p][i], a[q][i]
                        a[p][i] = c * api - s * aqi
                        a[q][i] = s * api + c * aqi
                    for i in range(n):
                        vip, viq = v[i][p], v[i][q]
                        v[i][p] = c * vip - s * viq
                        v[i][q] = s * vip + c * viq
        if not changed:
            break
    return [a[i][i] for i in range(n)], v


def lanczos_eigs(A, num, largest, dim):
    basis, alpha, beta = lanczos(A, dim)
    m = len(basis)
    t = [[0.0] * m for _ in range(m)]
    for i in range(m):
        t[i][i] = alpha[i]
    for i in range(m - 1):
        t[i][i + 1] = t[i + 1][i] = beta[i]
    eig, q = jacobi(t, 200)
    idx = sorted(range(m), key=lambda i: eig[i])
    order = list(reversed(idx))[:num] if largest else idx[:num]
    out = []
    for i in order:
        vec = np.zeros(len(basis[0]))
        for r, vr in enumerate(basis):
            vec += q[r][i] * vr
        out.append((eig[i], vec / np.sqrt(vec @ vec)))
    return out


def power_iteration(A, max_iter, tol):
    n = A.shape[0]
    x = np.arange(1, n + 1, dtype=np.float64)
    x /= np.sqrt(x @ x)
    lam = 0.0
    for _ in range(max_iter):
        y = _mv(A, x)
        x = y / np.sqrt(y @ y)
        new = float(x @ _mv(A, x)) / float(x @ x)
        if abs(new - lam) < tol * max(abs(new), 1.0):
            lam = new
            break
        lam = new
    return lam, x
