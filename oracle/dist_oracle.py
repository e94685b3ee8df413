"""Test-only numpy restatement of one rank of the library's row-partitioned
PCG (tpt-fem_b200/csrc/dist.cu): the same row ranges, ghost ordering (sorted by
global column), send lists (ascending owned rows each peer reads), vector
updates and call sequence, on host arrays.  It lets the multi-process driver
(tpt_fem.distributed.solve over torch.distributed) be tested with gloo on CPU.

The block preconditioner is restated in kind, not in the library's numbers:
classic FSAI of the owned diagonal block (pattern: the block's strictly lower
entries of each row) and a coarse space of contiguous row aggregates with the
constant mode, each rank forming its part P_k^T A_k P of A_c and P_k^T r_k of
the restriction for the driver to sum."""
import numpy as np


class NumpyRank:
    def __init__(self, A, b, rank, size, starts):
        A = A.tocsr()
        self.rank, self.size = rank, size
        r0, r1 = int(starts[rank]), int(starts[rank + 1])
        self.r0, self.r1, self.n_owned = r0, r1, r1 - r0
        rows = A[r0:r1]
        cols = rows.indices
        ghost = np.unique(cols[(cols < r0) | (cols >= r1)])
        self.n_ghost = len(ghost)
        owner = np.searchsorted(starts, ghost, side="right") - 1
        self.recv_counts = np.bincount(owner, minlength=size).astype(np.int64)
        local = np.where((cols >= r0) & (cols < r1), cols - r0, self.n_owned + np.searchsorted(ghost, cols))
        import scipy.sparse as sp
        self.A = sp.csr_matrix((rows.data, local, rows.indptr), shape=(self.n_owned, self.n_owned + self.n_ghost))
        self.dinv = 1.0 / rows.diagonal(k=r0)
        self.b = np.asarray(b[r0:r1], dtype=np.float64)
        send = []
        self.send_counts = np.zeros(size, np.int64)
        for q in range(size):
            if q == rank:
                continue
            qc = A[int(starts[q]):int(starts[q + 1])].indices
            need = np.unique(qc[(qc >= r0) & (qc < r1)]) - r0
            send.append(need)
            self.send_counts[q] = len(need)
        self.send_idx = np.concatenate(send) if send else np.zeros(0, np.int64)
        self.send_buf = np.zeros(len(self.send_idx))
        self.p = np.zeros(self.n_owned + self.n_ghost)
        self._A = A

    pc = False
    coarse_size = 0
    coarse_ready = False

    def set_precond(self, kind="fsai", coarse_aggregates=0):
        if kind != "fsai":
            raise ValueError("the numpy rank has the classic block FSAI only")
        r0, r1, n = self.r0, self.r1, self.n_owned
        B = self._A[r0:r1, r0:r1].toarray()
        self.sig2 = np.zeros(n)
        L = np.zeros((n, n))
        for i in range(n):  # A[P,P] y = e_last, P = lower pattern of row i, then i
            P = np.append(np.nonzero(B[i, :i])[0], i)
            y = np.linalg.solve(B[np.ix_(P, P)], np.eye(len(P))[-1])
            self.sig2[i] = y[-1]
            L[i, P[:-1]] = y[:-1] / y[-1]
        self.L = L
        self.pc, self.coarse_ready = True, False
        self.coarse_size = 0
        if coarse_aggregates is not None:
            nt = self._A.shape[0]
            na = coarse_aggregates if coarse_aggregates > 0 else max(2, nt // 16)
            agg = np.arange(nt) * na // nt
            P = np.zeros((nt, na))
            P[np.arange(nt), agg] = 1.0 / np.sqrt(np.bincount(agg, minlength=na))[agg]
            self.Pk = P[r0:r1]
            self.ac = np.ascontiguousarray(self.Pk.T @ (self._A[r0:r1] @ P))
            self.yc = np.zeros(na)
            self.coarse_size = na
        return self.coarse_size

    def coarse_matrix(self):
        import torch
        return torch.from_numpy(self.ac.reshape(-1))

    def coarse_vector(self):
        import torch
        return torch.from_numpy(self.yc)

    def coarse_factor(self):
        self.ainv = np.linalg.inv(self.ac)
        self.coarse_ready = True

    def precondition(self):
        t = self.sig2 * (self.r + self.L @ self.r)
        z = t + self.L.T @ t
        if self.coarse_size:
            z = z + self.Pk @ (self.ainv @ self.yc)
        self.z = z
        return np.array([self.r @ z])

    def _after_update(self):
        if self.coarse_size:
            self.yc[:] = self.Pk.T @ self.r
        return np.array([self.r @ self.r, 0.0])

    def _segments(self, buf, counts):
        import torch
        out, off = {}, 0
        for q, c in enumerate(counts):
            if c:
                out[q] = torch.from_numpy(buf[off:off + c])
            off += int(c)
        return out

    def send_segments(self):
        return self._segments(self.send_buf, self.send_counts)

    def recv_segments(self):
        return self._segments(self.p[self.n_owned:], self.recv_counts)

    def start(self):
        self.x = np.zeros(self.n_owned)
        self.r = self.b.copy()
        if self.pc:
            self.p[:] = 0.0
            return self._after_update()
        self.z = self.dinv * self.r
        self.p[:self.n_owned] = self.z
        return np.array([self.r @ self.r, self.r @ self.z])

    def pack(self):
        self.send_buf[:] = self.p[self.send_idx]

    def spmv_dot(self):
        self.q = self.A @ self.p
        return np.array([self.p[:self.n_owned] @ self.q])

    def update(self, alpha):
        self.x += alpha * self.p[:self.n_owned]
        self.r -= alpha * self.q
        if self.pc:
            return self._after_update()
        self.z = self.dinv * self.r
        return np.array([self.r @ self.r, self.r @ self.z])

    def direction(self, beta):
        self.p[:self.n_owned] = self.z + beta * self.p[:self.n_owned]

    def residual_begin(self):
        self.pbak = self.p[:self.n_owned].copy()
        self.p[:self.n_owned] = self.x

    def residual_end(self):
        self.r = self.b - self.A @ self.p
        self.p[:self.n_owned] = self.pbak
        if self.pc:
            return self._after_update()
        self.z = self.dinv * self.r
        return np.array([self.r @ self.r, self.r @ self.z])

    def solution(self):
        return self.x.copy()
