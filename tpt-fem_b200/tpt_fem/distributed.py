"""Row-partitioned FP64 PCG over several GPUs (one torch.distributed rank per
GPU).  The library does each rank's device work (tptfem_dist_*: its rows of the
reduced system with ghost columns, q = A p, the vector updates, the
preconditioner and the partial dot products); this module exchanges the ghost
values of p and sums the scalars and the coarse-space vectors.  The reference
solves on one CPU thread; this path has no counterpart there.

    ranks = [LibRank(system, rank, size, partition_rows(...))]     # this process's GPU
    for r in ranks:                                                # optional; Jacobi otherwise
        r.set_precond("learned", coarse_aggregates=0)
    it, rel = solve(ranks, TorchComm(group))                       # NCCL across processes

With a block preconditioner (block FSAI, classic or learned, plus the
aggregation coarse space) `solve` first sums the ranks' partial coarse matrices
and has every rank factor the sum; each iteration then sums the nc coarse
restriction values as well.  `solve` also runs several ranks of one process in
lock step (LocalComm), which is how the partitioned path is tested on a single
GPU.  Partial sums are added over local ranks in order and then across
processes, so all ranks take the same alpha and beta.
"""
import ctypes as C

import numpy as np

from . import _native as N


def partition_rows(n_free, dpn, size):
    """Contiguous, node-aligned row ranges (x-slabs of a box mesh), balanced by rows."""
    if n_free % dpn:
        dpn = 1
    groups = n_free // dpn
    starts = [groups * k // size * dpn for k in range(size + 1)]
    starts[-1] = n_free
    return np.array(starts, dtype=np.int64)


class _DevArray:
    """A device buffer of the library exposed to torch through __cuda_array_interface__."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class LibRank:
    """One rank of the partitioned solve on the library (tptfem_dist_*)."""

    def __init__(self, system, rank, size, row_starts):
        self.ctx, self.rank, self.size = system.ctx, rank, size
        self.system = system  # the preconditioner's coarse space reads it
        lib = self.ctx.lib
        self.starts = np.asarray(row_starts, dtype=np.int64)
        h = C.c_void_p()
        self.ctx.check(lib.tptfem_dist_create(self.ctx.h, system.h, rank, size, N.ptr(self.starts), C.byref(h)))
        self.h = h
        no, ng = C.c_int64(), C.c_int64()
        self.send_counts = np.zeros(size, np.int64)
        self.recv_counts = np.zeros(size, np.int64)
        self.ctx.check(lib.tptfem_dist_counts(h, C.byref(no), C.byref(ng), N.ptr(self.send_counts),
                                              N.ptr(self.recv_counts)))
        self.n_owned, self.n_ghost = no.value, ng.value
        sb, gb = C.c_void_p(), C.c_void_p()
        self.ctx.check(lib.tptfem_dist_buffers(h, C.byref(sb), C.byref(gb)))
        self._send_ptr, self._ghost_ptr = sb.value or 0, gb.value or 0

    def _segments(self, ptr, counts):
        import torch
        out, off = {}, 0
        for q, c in enumerate(counts):
            if c:
                out[q] = torch.as_tensor(_DevArray(ptr + 8 * off, c), device="cuda")
            off += int(c)
        return out

    def send_segments(self):
        return self._segments(self._send_ptr, self.send_counts)

    def recv_segments(self):
        return self._segments(self._ghost_ptr, self.recv_counts)

    pc = False
    coarse_size = 0
    coarse_ready = False

    def set_precond(self, kind="fsai", coarse_aggregates=0):
        """Block FSAI ("fsai": classic values, "learned": the network attached to
        the system) and, unless coarse_aggregates is None, the coarse space (0: the
        default aggregate count).  Returns the coarse size (0: none)."""
        k = {"fsai": 1, "learned": 2}[kind]
        nc = C.c_int64()
        aggs = -1 if coarse_aggregates is None else int(coarse_aggregates)
        self.ctx.check(self.ctx.lib.tptfem_dist_set_precond(self.ctx.h, self.h, self.system.h, k, aggs,
                                                           C.byref(nc)))
        self.pc, self.coarse_size, self.coarse_ready = True, nc.value, False
        am, av = C.c_void_p(), C.c_void_p()
        self.ctx.check(self.ctx.lib.tptfem_dist_coarse_buffers(self.h, C.byref(am), C.byref(av)))
        self._am, self._av = am.value or 0, av.value or 0
        return self.coarse_size

    def _dev(self, ptr, n):
        import torch
        return torch.as_tensor(_DevArray(ptr, n), device="cuda")

    def coarse_matrix(self):
        return self._dev(self._am, self.coarse_size * self.coarse_size)

    def coarse_vector(self):
        return self._dev(self._av, self.coarse_size)

    def coarse_factor(self):
        self.ctx.check(self.ctx.lib.tptfem_dist_coarse_factor(self.ctx.h, self.h))
        self.coarse_ready = True

    def precondition(self):
        v = C.c_double()
        self.ctx.check(self.ctx.lib.tptfem_dist_precondition(self.ctx.h, self.h, C.byref(v)))
        return np.array([v.value])

    def start(self):
        o = np.zeros(2)
        self.ctx.check(self.ctx.lib.tptfem_dist_start(self.ctx.h, self.h, N.ptr(o)))
        return o

    def pack(self):
        self.ctx.check(self.ctx.lib.tptfem_dist_pack(self.ctx.h, self.h))

    def spmv_dot(self):
        v = C.c_double()
        self.ctx.check(self.ctx.lib.tptfem_dist_spmv_dot(self.ctx.h, self.h, C.byref(v)))
        return np.array([v.value])

    def update(self, alpha):
        o = np.zeros(2)
        self.ctx.check(self.ctx.lib.tptfem_dist_update(self.ctx.h, self.h, float(alpha), N.ptr(o)))
        return o

    def direction(self, beta):
        self.ctx.check(self.ctx.lib.tptfem_dist_direction(self.ctx.h, self.h, float(beta)))

    def residual_begin(self):
        self.ctx.check(self.ctx.lib.tptfem_dist_residual_begin(self.ctx.h, self.h))

    def residual_end(self):
        o = np.zeros(2)
        self.ctx.check(self.ctx.lib.tptfem_dist_residual_end(self.ctx.h, self.h, N.ptr(o)))
        return o

    def solution(self):
        x = np.zeros(self.n_owned)
        self.ctx.check(self.ctx.lib.tptfem_dist_solution(self.ctx.h, self.h, N.ptr(x)))
        return x

    def __del__(self):
        if getattr(self, "h", None) is not None:
            self.ctx.lib.tptfem_dist_free(self.h)
            self.h = None


class LocalComm:
    """All ranks in this process: exchanges are copies between their buffers."""

    def allreduce(self, v):
        return v

    def sum_tensors(self, ts):
        """Every tensor becomes the sum of all (added in rank order)."""
        if len(ts) > 1:
            s = ts[0].clone()
            for t in ts[1:]:
                s += t
            for t in ts:
                t.copy_(s)
        if ts and ts[0].is_cuda:
            import torch
            torch.cuda.synchronize()

    def exchange(self, ranks):
        sends = [r.send_segments() for r in ranks]
        for r in ranks:
            for q, dst in r.recv_segments().items():
                dst.copy_(sends[q][r.rank])


class TorchComm:
    """One rank per process over torch.distributed (NCCL for GPUs, gloo for host arrays)."""

    def __init__(self, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.dist, self.torch, self.group = dist, torch, group
        self.device = device

    def allreduce(self, v):
        t = self.torch.tensor(np.asarray(v, dtype=np.float64), device=self.device)
        self.dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def sum_tensors(self, ts):
        (t,) = ts
        self.dist.all_reduce(t, group=self.group)
        if t.is_cuda:
            self.torch.cuda.synchronize()

    def exchange(self, ranks):
        (r,) = ranks
        ops = []
        for q, t in r.send_segments().items():
            ops.append(self.dist.P2POp(self.dist.isend, t, q, group=self.group))
        for q, t in r.recv_segments().items():
            ops.append(self.dist.P2POp(self.dist.irecv, t, q, group=self.group))
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()
        if self.device is not None and str(self.device).startswith("cuda"):
            self.torch.cuda.synchronize()


def prepare(ranks, comm):
    """Sum the ranks' partial coarse matrices and factor the sum on every rank
    (once, after set_precond; solve calls it)."""
    r0 = ranks[0]
    if r0.pc and r0.coarse_size and not r0.coarse_ready:
        comm.sum_tensors([r.coarse_matrix() for r in ranks])
        for r in ranks:
            r.coarse_factor()


DELTA = 1e-6  # reliable updates: the true residual replaces the recursive one after this drop


def solve(ranks, comm, tol=1e-10, max_iter=100000):
    """FP64 PCG over the partitioned system -> (iterations, TRUE relative residual).
    Jacobi, or the ranks' block preconditioner when set_precond was called.
    As in the one-GPU solver, the true residual b - A x replaces the recursive
    one whenever the latter has dropped by DELTA since the last replacement and
    before the solve may stop (the search direction is kept)."""
    def total(vals):
        s = np.zeros_like(vals[0])
        for v in vals:  # local ranks in rank order
            s = s + v
        return comm.allreduce(s)

    pc = bool(getattr(ranks[0], "pc", False))
    nc = int(getattr(ranks[0], "coarse_size", 0)) if pc else 0
    if pc:
        prepare(ranks, comm)

    def precondition():  # z = M r on every rank; the summed r.z
        if nc:
            comm.sum_tensors([r.coarse_vector() for r in ranks])
        return total([r.precondition() for r in ranks])[0]

    rr, rz = total([r.start() for r in ranks])
    if pc:
        rz = precondition()
        for r in ranks:
            r.direction(0.0)
    bb, it = rr, 0
    target = tol * tol * bb
    rr_upd = bb
    while bb > 0:
        # the iteration that reaches the replacement threshold stops after the
        # x, r update; the direction then continues from the true residual
        until = max(0.25 * target, DELTA * DELTA * rr_upd)
        while it < max_iter:
            for r in ranks:
                r.pack()
            comm.exchange(ranks)
            pq = total([r.spmv_dot() for r in ranks])[0]
            if not pq > 0.0:
                raise ArithmeticError("PCG breakdown: p.Ap <= 0")
            alpha = rz / pq
            rr, rz_new = total([r.update(alpha) for r in ranks])
            it += 1
            if rr <= until:
                break
            if pc:
                rz_new = precondition()
            beta = rz_new / rz
            rz = rz_new
            for r in ranks:
                r.direction(beta)
        # reliable update: x's ghosts through the usual exchange, then r = b - A x
        for r in ranks:
            r.residual_begin()
            r.pack()
        comm.exchange(ranks)
        rr, rz_t = total([r.residual_end() for r in ranks])
        if rr <= target or it >= max_iter:
            break
        if pc:
            rz_t = precondition()
        beta = rz_t / rz
        rz, rr_upd = rz_t, rr
        for r in ranks:
            r.direction(beta)
    return it, float(np.sqrt(rr / bb)) if bb > 0 else 0.0
