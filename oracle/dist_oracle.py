"""Test-only numpy restatement of one rank of the library's row-partitioned
Jacobi-PCG (tpt-fem_b200/csrc/dist.cu): the same row ranges, ghost ordering
(sorted by global column), send lists (ascending owned rows each peer reads)
and vector updates, on host arrays.  It lets the multi-process driver
(tpt_fem.distributed.solve over torch.distributed) be tested with gloo on CPU."""
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
        self.z = self.dinv * self.r
        return np.array([self.r @ self.r, self.r @ self.z])

    def direction(self, beta):
        self.p[:self.n_owned] = self.z + beta * self.p[:self.n_owned]

    def solution(self):
        return self.x.copy()
