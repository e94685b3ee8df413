"""The multi-process driver of the row-partitioned Jacobi-PCG
(tpt_fem.distributed) over torch.distributed with gloo, world size 2 and 3, on
CPU: each process runs the numpy restatement of one library rank
(oracle/dist_oracle.py); the gathered solution must equal a serial solve."""
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


def _worker(rank, size, port, q):
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
        it, rel = solve([r], TorchComm(), tol=1e-10)
        q.put((rank, it, rel, r.solution().tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("size", [2, 3])
def test_gloo_ranks_match_a_serial_solve(size):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29650 + size
    procs = [ctx.Process(target=_worker, args=(k, size, port, q)) for k in range(size)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(size)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert len({o[1] for o in out}) == 1  # every rank took the same number of iterations
    x = np.concatenate([o[3] for o in out])
    A = laplacian_2d(12, 9)
    b = np.cos(np.arange(A.shape[0]))
    ref = sp.linalg.spsolve(A.tocsc(), b)
    assert np.linalg.norm(A @ x - b) <= 1e-9 * np.linalg.norm(b)
    assert np.max(np.abs(x - ref)) <= 1e-8 * np.max(np.abs(ref))


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
