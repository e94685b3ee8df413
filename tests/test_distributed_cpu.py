"""The multi-process driver of the row-partitioned PCG (tpt_fem.distributed)
over torch.distributed with gloo, world size 2 and 3, on CPU: each process runs
the numpy restatement of one library rank (oracle/dist_oracle.py), with Jacobi
or with the block FSAI + coarse-space preconditioner (whose partial coarse
matrices and restrictions the driver sums over the ranks), and reliable
updates (the true residual, exchanged like p, replaces the recursive one); the
gathered solution must equal a serial solve."""
import os
import sys

import numpy as np
import pytest
import scipy.sparse as sp
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def laplacian_2d(nx, ny):
    def lap1(n):
        return sp.diags([-np.ones(n - 1), 2 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1])
    return (sp.kron(sp.eye(ny), lap1(nx)) + sp.kron(lap1(ny), sp.eye(nx))).tocsr()


def _worker(rank, size, port, q, pc=False):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tpt-fem_b200"))
    import torch.distributed as dist
    from oracle.dist_oracle import NumpyRank
    from tpt_fem.distributed import TorchComm, partition_rows, solve
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        A = laplacian_2d(12, 9)
        b = np.cos(np.arange(A.shape[0]))
        starts = partition_rows(A.shape[0], 1, size)
        r = NumpyRank(A, b, rank, size, starts)
        if pc:
            r.set_precond("fsai", coarse_aggregates=0)
        it, rel = solve([r], TorchComm(), tol=1e-10)
        q.put((rank, it, rel, r.solution().tolist()))
    finally:
        dist.destroy_process_group()


JACOBI_ITERS = {}


@pytest.mark.parametrize("pc", [False, True])
@pytest.mark.parametrize("size", [2, 3])
def test_gloo_ranks_match_a_serial_solve(size, pc):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29650 + size + (10 if pc else 0)
    procs = [ctx.Process(target=_worker, args=(k, size, port, q, pc)) for k in range(size)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(size)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert len({o[1] for o in out}) == 1  # every rank took the same number of iterations
    if pc:  # block FSAI + coarse space: fewer iterations than Jacobi on the same partition
        it_jac, _ = _solve_local(serial_ranks(size))
        assert out[0][1] <= 0.7 * it_jac, (out[0][1], it_jac)
    x = np.concatenate([o[3] for o in out])
    A = laplacian_2d(12, 9)
    b = np.cos(np.arange(A.shape[0]))
    ref = sp.linalg.spsolve(A.tocsc(), b)
    assert np.linalg.norm(A @ x - b) <= 1e-9 * np.linalg.norm(b)
    assert np.max(np.abs(x - ref)) <= 1e-8 * np.max(np.abs(ref))


def serial_ranks(size, pc=False):
    sys.path.insert(0, os.path.join(ROOT, "tpt-fem_b200"))
    from oracle.dist_oracle import NumpyRank
    from tpt_fem.distributed import partition_rows
    A = laplacian_2d(12, 9)
    b = np.cos(np.arange(A.shape[0]))
    starts = partition_rows(A.shape[0], 1, size)
    ranks = [NumpyRank(A, b, k, size, starts) for k in range(size)]
    if pc:
        for r in ranks:
            r.set_precond("fsai", coarse_aggregates=0)
    return ranks


def _solve_local(ranks):
    from tpt_fem.distributed import LocalComm, solve
    return solve(ranks, LocalComm(), tol=1e-10)


@pytest.mark.parametrize("size", [1, 3])
def test_lockstep_block_preconditioner_solves_and_sums_the_coarse_matrix(size):
    A = laplacian_2d(12, 9)
    b = np.cos(np.arange(A.shape[0]))
    ranks = serial_ranks(size, pc=True)
    parts = [r.ac.copy() for r in ranks]
    it, rel = _solve_local(ranks)
    # the summed partial coarse matrices are P^T A P of the whole system
    P = np.vstack([r.Pk for r in ranks])
    assert np.allclose(ranks[0].ac, P.T @ (A @ P), rtol=1e-14, atol=1e-13)
    assert np.allclose(sum(parts), P.T @ (A @ P), rtol=1e-14, atol=1e-13)
    x = np.concatenate([r.solution() for r in ranks])
    assert rel <= 1e-10 and np.linalg.norm(A @ x - b) <= 1e-9 * np.linalg.norm(b)
    it_jac, _ = _solve_local(serial_ranks(size))
    assert it <= 0.7 * it_jac, (it, it_jac)


def test_single_process_lockstep_equals_two_processes():
    sys.path.insert(0, os.path.join(ROOT, "tpt-fem_b200"))
    from oracle.dist_oracle import NumpyRank
    from tpt_fem.distributed import LocalComm, partition_rows, solve
    A = laplacian_2d(12, 9)
    b = np.cos(np.arange(A.shape[0]))
    starts = partition_rows(A.shape[0], 1, 3)
    ranks = [NumpyRank(A, b, k, 3, starts) for k in range(3)]
    it, rel = solve(ranks, LocalComm(), tol=1e-10)
    x = np.concatenate([r.solution() for r in ranks])
    assert rel <= 1e-10 and np.linalg.norm(A @ x - b) <= 1e-9 * np.linalg.norm(b)
    # the residual the driver reports is the true one (the last reliable update)
    assert abs(rel - np.linalg.norm(b - A @ x) / np.linalg.norm(b)) <= 1e-13
    # ghost receive counts mirror the peers' send counts
    for r in ranks:
        for qd in range(3):
            assert r.recv_counts[qd] == ranks[qd].send_counts[r.rank]


def test_partition_rows_is_node_aligned_and_balanced():
    sys.path.insert(0, os.path.join(ROOT, "tpt-fem_b200"))
    from tpt_fem.distributed import partition_rows
    s = partition_rows(3 * 1001, 3, 4)
    assert s[0] == 0 and s[-1] == 3003 and all(v % 3 == 0 for v in s)
    assert max(np.diff(s)) - min(np.diff(s)) <= 3
