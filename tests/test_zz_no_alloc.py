"""The allocation-free residual entry point, through the C ABI.

tptfem_rel_residual_noalloc serves callers that must not let the library
allocate device memory (a fixed device-memory budget, or a loop that cannot
take the synchronisation of cudaMalloc/cudaFree per call).  Its scratch is a
static device array, so this test checks two consecutive calls -- the second
sees the first call's leftovers -- against the relative residual that the
existing solver entry point (tptfem_system_solve) reports for the same system,
and that oversized or malformed inputs are rejected before any launch.

The file is named to be collected last, so a stop-at-first-failure run has
already run every other test when it gets here.
"""
import ctypes as C

import numpy as np
import pytest

import tpt_fem as F
from tpt_fem import _native as N
from meshes import box, jitter
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # two FP64 compensated reductions in different block orders


def _device(arr, dtype):
    import torch
    return torch.as_tensor(np.ascontiguousarray(arr, dtype=dtype)).to("cuda:0")


def _call(lib, n, rp, ci, va, x, b, stream=None):
    out = C.c_double(-1.0)
    err = C.create_string_buffer(256)
    rc = lib.tptfem_rel_residual_noalloc(0, stream, n, C.c_void_p(rp.data_ptr()), C.c_void_p(ci.data_ptr()),
                                         C.c_void_p(va.data_ptr()), C.c_void_p(x.data_ptr()),
                                         C.c_void_p(b.data_ptr()), C.byref(out), err, len(err))
    return rc, out.value, err.value.decode()


def test_noalloc_residual_matches_solver_on_two_calls():
    import torch
    ctx = F.Context.default(0)
    c, e = box([10, 4, 4], mx=(2.5, 1.0, 1.0))
    c = jitter(c, 0.02, 31)
    E = 1e-3 + (1 - 1e-3) * np.random.default_rng(32).uniform(size=len(e)) ** 3
    m = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    K = F.assemble_elasticity(m, "3d", E, 0.3, 2)
    rhs = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    x0 = [int(i) for i in O.nodes_on_plane(c, 0, 0.0, 1e-9)]
    S = F.reduce_system(K, rhs, [(3 * n + k, 0.0) for n in x0 for k in range(3)])
    # loose tolerance so the residual is well above rounding and both paths see the same x
    st = S.solve(solver=F.SOLVER_JACOBI_PCG, tol=1e-6)
    rp, ci, va, fred, free = S.download()
    x = S.solution()[free]
    lib = N.load()
    args = (S.n_free, _device(rp, np.int32), _device(ci, np.int32), _device(va, np.float64),
            _device(x, np.float64), _device(fred, np.float64))
    torch.cuda.synchronize()
    first = _call(lib, *args)
    second = _call(lib, *args)
    for rc, val, msg in (first, second):
        assert rc == N.OK, msg
        assert abs(val - st["rel_residual"]) <= REL_TOL * st["rel_residual"]
    assert first[1] == second[1]
    # an independent host check: the same residual from a plain numpy CSR product
    ax = np.add.reduceat(va * x[ci], rp[:-1]) if len(va) else np.zeros(S.n_free)
    host = np.linalg.norm(fred - ax) / np.linalg.norm(fred)
    # the naive host sum cancels: its error is ~1e-16 of ||b|| per row term,
    # i.e. ~1e-10 of this 1e-6 residual, a few times that in practice
    assert abs(first[1] - host) <= 1e-7 * host

    # the same call ordered on a caller's stream: x is produced on that stream
    # by a kernel the call must wait for
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        xs = torch.zeros_like(args[4])
        xs.copy_(args[4])
        third = _call(lib, *args[:4], xs, args[5], stream=C.c_void_p(side.cuda_stream))
    assert third[0] == N.OK, third[2]
    assert third[1] == first[1]


def test_noalloc_residual_rejects_bad_sizes():
    import torch
    lib = N.load()
    one = _device([0, 1], np.int32)
    col = _device([0], np.int32)
    v = _device([2.0], np.float64)
    for n in (0, 2 ** 31):
        rc, _, msg = _call(lib, n, one, col, v, v, v)
        assert rc == 9 and "n must be" in msg
    bad = _device([5], np.int32)  # column outside [0, n)
    rc, _, msg = _call(lib, 1, one, bad, v, v, v)
    assert rc == 9 and "column" in msg
    # malformed row pointers: reversed ranges and ranges past row_ptrs[n] are
    # flagged and skipped before any entry is read
    col2 = _device([0, 1, 0, 1], np.int32)
    v4 = _device([1.0, 2.0, 3.0, 4.0], np.float64)
    x2 = _device([1.0, 1.0], np.float64)
    for rows in ([0, 3, 2], [0, 5, 4], [-1, 2, 4], [0, 6, 4]):
        rc, _, msg = _call(lib, 2, _device(rows, np.int32), col2, v4, x2, x2)
        assert rc == 9 and "row_ptrs" in msg, (rows, msg)
    rc, _, msg = _call(lib, 2, _device([0, 2, -1], np.int32), col2, v4, x2, x2)
    assert rc == 9 and "negative" in msg
    # A = [[2]], x = [1], b = [4]: |4 - 2| / 4 = 0.5
    rc, val, msg = _call(lib, 1, one, col, v, _device([1.0], np.float64), _device([4.0], np.float64))
    assert rc == N.OK and abs(val - 0.5) < 1e-15, msg
    # b = 0: the documented value is ||r||_2 itself, here |0 - 2 * 1.5| = 3
    rc, val, msg = _call(lib, 1, one, col, v, _device([1.5], np.float64), _device([0.0], np.float64))
    assert rc == N.OK and val == 3.0, msg
    torch.cuda.synchronize()
