"""Generate the configuration-size parity fixtures from the CPU oracle.

    python tests/golden/make_scale_fixtures.py [cube64|topopt|all]

cube64_elasticity_digests.json
    The 64^3 unit-cube elasticity case (box_mesh [64,64,64] P1 tets, E = 1,
    nu = 0.3, quadrature order 2; x = 0 clamped; traction (0, 0, -1e-3) on
    x = 1).  The oracle runs the reference's whole path -- assemble
    (crates/tpt-fem-assembly/src/lib.rs:428-480), Coo::to_csr with its stable
    sort and duplicate sum (crates/tpt-fem-sparse/src/lib.rs:122-175),
    apply_neumann_order (assembly:601-667) and reduce_system (assembly:504-535)
    -- and the fixture keeps the sizes and the SHA-256 of every array (int64
    indices, float64 values, little-endian bytes): 116M COO triplets are too
    many to commit, their digests are 1 KB.

topopt_sizes_parity.npz
    topopt_simp (crates/tpt-fem-topopt/src/lib.rs:342-385) in the reference's
    own semantics (Emin = 1e-3 E0, the unweighted sensitivity filter) for one
    instance of each batched-workload size, 60x20 ... 240x80: vol_frac 0.4,
    filter radius 1.5, move limit 0.2, unit -y load at the mid-right node,
    100 OC iterations.  Compliance histories and final densities.

The oracle's banded Cholesky stands in for the reference's dense LU above
1000 dofs (the dense factor of a 240x80 grid would need 12 GB).
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tpt-fem_b200"))

from oracle import oracle as O  # noqa: E402
from tpt_fem import workloads as W  # noqa: E402

TOPOPT_SIZES = [(60, 20), (90, 30), (120, 40), (180, 60), (240, 80)]
TOPOPT_ITERS = 100


def digest(a, dtype):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).astype(np.dtype(dtype).newbyteorder("<"),
                                                                        copy=False).tobytes()).hexdigest()


def csr_digests(rp, ci, va):
    return {"nrows": int(len(rp) - 1), "nnz": int(len(ci)), "row_ptrs": digest(rp, np.int64),
            "col_ind": digest(ci, np.int64), "values": digest(va, np.float64)}


def cube64():
    t0 = time.time()
    c, e = O.box_mesh([0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [64, 64, 64])
    m = O.Mesh(O.CELL_TET, c, e)
    coo = O.assemble_elasticity(m, O.MODEL_3D, 1.0, 0.3, 2)
    csr = coo.to_csr()
    out = {"case": "box_mesh [64,64,64] P1 tets, E = 1, nu = 0.3, order 2",
           "matrix": csr_digests(csr.row_ptrs, csr.col_ind, csr.values)}
    del csr
    rhs = np.zeros(3 * len(c))
    O.apply_traction(m, 3, 0, 1.0, -1e-3, 1 << 2, rhs)
    out["traction_rhs"] = {"n": len(rhs), "sha256": digest(rhs, np.float64)}
    dof, val = W.clamp_x0_bcs(c)
    kred, fred, free = O.reduce_system(coo, rhs, list(zip(dof, val)))
    del coo
    kr = kred.to_csr()
    out["reduced"] = csr_digests(kr.row_ptrs, kr.col_ind, kr.values)
    out["reduced"]["fred"] = digest(fred, np.float64)
    out["reduced"]["free"] = digest(free, np.int64)
    with open(os.path.join(HERE, "cube64_elasticity_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    print(f"cube64 fixture in {time.time() - t0:.0f} s")


def topopt():
    t0 = time.time()
    hist, dens = {}, {}
    for nelx, nely in TOPOPT_SIZES:
        f, bcs = O.cantilever_load(nelx, nely, 1.0, node=(nelx + 1) * (nely // 2) + nelx)
        comp, rho = O.topopt(nelx, nely, 0.4, 1.5, TOPOPT_ITERS, f, bcs)
        hist[f"compliance_{nelx}x{nely}"] = comp
        dens[f"densities_{nelx}x{nely}"] = rho
        print(f"topopt {nelx}x{nely}: {time.time() - t0:.0f} s")
    np.savez_compressed(os.path.join(HERE, "topopt_sizes_parity.npz"), **hist, **dens)


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("cube64", "all"):
        cube64()
    if what in ("topopt", "all"):
        topopt()
