"""Parity with the oracle at the benchmark configurations' full sizes.

The small-mesh tests pin every kernel bit for bit; these repeat the check on
the meshes the benchmarks run, where other code paths are taken: host arrays
moved through the chunked pinned staging with int64 -> int32 narrowing,
padded-row compaction at large row lengths, and the node-block layouts.

  * 280x70x70 elasticity cantilever (4.25M dofs), through the host-array
    route (Mesh.from_arrays, assembly, traction, reduction): >= 10,000 rows of
    the CSR and of the reduced system, bit for bit against the row-restricted
    oracle, sampled at random, at both x ends and at the staging chunk
    boundaries; the whole traction vector and the mesh round trip.
  * 128^3 Poisson with a Gaussian-random-field conductivity: the same row
    check, and the source load at the sampled nodes.
  * 64^3 elasticity cube: the WHOLE CSR, traction vector and reduced system,
    against digests of the oracle's full COO + stable-sort path
    (tests/golden/make_scale_fixtures.py).
  * topopt_simp in the reference's semantics, one instance of each batched
    size (60x20 ... 240x80), 100 OC iterations, against the oracle histories.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import tpt_fem as F
from tpt_fem import topopt as T
from tpt_fem import workloads as W
from conftest import GOLDEN
from oracle import oracle as O

pytestmark = pytest.mark.gpu

STAGE_CHUNK = 8 << 20  # bytes per pipelined staging chunk (csrc/staging.cu)
STAGE_THREADS = 16     # most host threads that fill one chunk


def digest(a, dtype):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


def gather_rows(rp, ci, va, rows):
    """(ptr, cols, vals) of the given rows of a CSR held as numpy arrays."""
    rows = np.asarray(rows, np.int64)
    lo, hi = rp[rows], rp[rows + 1]
    ptr = np.concatenate([[0], np.cumsum(hi - lo)])
    idx = np.concatenate([np.arange(a, b) for a, b in zip(lo, hi)]) if len(rows) else np.zeros(0, np.int64)
    return ptr, ci[idx], va[idx]


def assert_rows_equal(got, ref, rows):
    gp, gc, gv = got
    rp_, rc, rv = ref
    if np.array_equal(gp, rp_) and np.array_equal(gc, rc) and np.array_equal(gv, rv):
        return
    for k, r in enumerate(rows):  # name the first differing row
        a = (gc[gp[k]:gp[k + 1]], gv[gp[k]:gp[k + 1]])
        b = (rc[rp_[k]:rp_[k + 1]], rv[rp_[k]:rp_[k + 1]])
        if not (np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])):
            raise AssertionError(f"row {r}: device {a} != oracle {b}")
    raise AssertionError("row layouts differ")


def staging_boundaries(n_elems, n_nodes):
    """Elements and nodes whose staged data straddles a staging chunk or a host
    thread's slice of one.  The chunk unit may be one element (int32 x 4, 16
    bytes) or one index (4 bytes) of the connectivity, one node (24 bytes) or
    one float64 (8 bytes) of the coordinates; all four are covered."""
    elems, nodes = set(), set()
    for unit_bytes, per_item, count, out in ((16, 1, n_elems, elems), (4, 4, n_elems, elems),
                                             (24, 1, n_nodes, nodes), (8, 3, n_nodes, nodes)):
        units = count * per_item
        cel = max(1, STAGE_CHUNK // unit_bytes)
        for c0 in range(0, units, cel):
            ln = min(units, c0 + cel) - c0
            for t in range(STAGE_THREADS + 1):
                b = c0 + ln * t // STAGE_THREADS
                for u in (b - 1, b):
                    if 0 <= u < units:
                        out.add(u // per_item)
    return elems, nodes


def sample_rows(c, e, dpn, rng, n_random=10000):
    rows = set(rng.choice(len(c) * dpn, n_random, replace=False).tolist())
    x = c[:, 0]
    for end in (x.min(), x.max()):  # both x ends
        nodes = np.nonzero(np.abs(x - end) < 1e-9)[0]
        for nd in rng.choice(nodes, min(300, len(nodes)), replace=False):
            rows.update(int(nd) * dpn + k for k in range(dpn))
    elems, nodes = staging_boundaries(len(e), len(c))
    nodes |= set(int(nd) for el in elems for nd in e[el])
    rows.update(nd * dpn + k for nd in nodes for k in range(dpn))
    return np.array(sorted(rows), np.int64)


def check_reduced(S, ref_rows, rows, rhs, bcs, n):
    rp, ci, va, fred, free = S.download()
    fidx = -np.ones(n, np.int64)
    fidx[free] = np.arange(len(free))
    keep = fidx[rows] >= 0
    ptr, cols, vals = ref_rows
    sel = np.nonzero(keep)[0]
    sub = gather_rows(ptr, cols, vals, sel)
    optr, ocols, ovals, ofred = O.reduced_rows(*sub, rhs[rows[sel]], bcs, fidx)
    red_rows = fidx[rows[sel]]
    assert_rows_equal(gather_rows(rp, ci, va, red_rows), (optr, ocols, ovals), rows[sel])
    assert np.array_equal(fred[red_rows], ofred)
    return len(sel)


def test_cantilever_280x70x70_rows_through_host_arrays(ctx):
    mn, mx, n = W.CANTILEVERS["cantilever_280x70x70"]
    c, e = O.box_mesh(mn, mx, n)
    E = W.cantilever_young(n)
    mesh = F.Mesh.from_arrays(F.CELL_TET4, c, e, ctx=ctx)
    mesh._coords = mesh._conn = None  # read the device copy back
    assert np.array_equal(mesh.coords_array, c) and np.array_equal(mesh.conn_array, e)
    K = F.assemble_elasticity(mesh, "3d", E, 0.3, 2)
    assert (K.nrows, K.nnz) == (4249563, 154811997)
    rhs = F.apply_traction(mesh, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    dof, val = W.clamp_x0_bcs(c)
    bcs = list(zip(dof.tolist(), val.tolist()))
    S = F.reduce_system(K, rhs, bcs)

    om = O.Mesh(O.CELL_TET, c, e)
    orhs = np.zeros(3 * len(c))
    O.apply_traction(om, 3, 0, 1.0, -1e-3, 1 << 2, orhs)
    assert np.array_equal(rhs, orhs)

    rows = sample_rows(c, e, 3, np.random.default_rng(280))
    assert len(rows) >= 10000
    ref = O.csr_rows(om, "elasticity", E, rows)
    rp, ci, va = K.to_csr()
    assert_rows_equal(gather_rows(rp, ci, va, rows), ref, rows)
    del rp, ci, va
    assert check_reduced(S, ref, rows, orhs, bcs, K.nrows) >= 9000


def test_poisson_grf_128_rows(ctx):
    n = 128
    mesh = F.Mesh.box_mesh([0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [n, n, n], ctx=ctx)
    c, e = O.box_mesh([0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [n, n, n])
    assert np.array_equal(mesh.coords_array, c) and np.array_equal(mesh.conn_array, e)
    k = np.exp(W.grf_at_centroids(c, e, 5000, ctx=ctx))
    K = F.assemble_poisson(mesh, k, 2)
    assert K.nnz == 14926977
    rhs = F.load_poisson_source(mesh, 1.0, 2)
    on_b = np.nonzero(np.any((c < 1e-9) | (c > 1 - 1e-9), axis=1))[0]
    bcs = [(int(i), 0.0) for i in on_b]
    S = F.reduce_system(K, rhs, bcs)

    om = O.Mesh(O.CELL_TET, c, e)
    rows = sample_rows(c, e, 1, np.random.default_rng(128))
    ref = O.csr_rows(om, "poisson", k, rows)
    rp, ci, va = K.to_csr()
    assert_rows_equal(gather_rows(rp, ci, va, rows), ref, rows)
    del rp, ci, va
    assert np.array_equal(rhs[rows], O.load_poisson_rows(om, 1.0, rows))
    full_rhs = rhs.copy()
    full_rhs[rows] = O.load_poisson_rows(om, 1.0, rows)
    assert check_reduced(S, ref, rows, full_rhs, bcs, K.nrows) > 5000


def test_cube64_whole_system_against_oracle_digests(ctx):
    with open(os.path.join(GOLDEN, "cube64_elasticity_digests.json")) as f:
        g = json.load(f)
    m = F.Mesh.box_mesh([0, 0, 0], [1, 1, 1], [64, 64, 64], ctx=ctx)
    K = F.assemble_elasticity(m, "3d", 1.0, 0.3, 2)
    rp, ci, va = K.to_csr()
    got = {"nrows": K.nrows, "nnz": K.nnz, "row_ptrs": digest(rp, np.int64), "col_ind": digest(ci, np.int64),
           "values": digest(va, np.float64)}
    assert got == g["matrix"]
    del rp, ci, va
    rhs = F.apply_traction(m, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    assert digest(rhs, np.float64) == g["traction_rhs"]["sha256"]
    dof, val = W.clamp_x0_bcs(m.coords_array)
    S = F.reduce_system(K, rhs, list(zip(dof, val)))
    rp, ci, va, fred, free = S.download()
    got = {"nrows": S.n_free, "nnz": S.nnz, "row_ptrs": digest(rp, np.int64), "col_ind": digest(ci, np.int64),
           "values": digest(va, np.float64), "fred": digest(fred, np.float64), "free": digest(free, np.int64)}
    assert got == g["reduced"]


def test_topopt_each_batched_size_matches_oracle_histories(ctx):
    g = np.load(os.path.join(GOLDEN, "topopt_sizes_parity.npz"))
    probs = []
    for nelx, nely in W.TOPOPT_SIZES:
        P = T.TopOptParams(grid=T.Grid(nelx + 1, nely + 1, 1.0), vol_frac=0.4, filter_radius=1.5, max_iter=100,
                           move_limit=0.2)
        f, bcs = T.cantilever_load(P.grid, node=P.grid.nx * (nely // 2) + nelx)
        probs.append((P, f, bcs))
    res, st = T.topopt_batch(ctx, probs, rel_tol=1e-12)
    assert st["not_converged"] == 0
    for (nelx, nely), r in zip(W.TOPOPT_SIZES, res):
        oc = g[f"compliance_{nelx}x{nely}"]
        orho = g[f"densities_{nelx}x{nely}"]
        assert len(r.compliance) == len(oc) == 101
        assert np.max(np.abs(r.compliance - oc) / np.abs(oc)) <= 1e-8, (nelx, nely)
        assert np.max(np.abs(r.densities - orho)) <= 1e-7, (nelx, nely)
