"""Exodus II export of device-resident meshes (write_exodus,
crates/tpt-fem-io-exodus/src/lib.rs:384-563) byte for byte against the
oracle's restatement of the reference writer, and read back by the
restated reader."""
import numpy as np
import pytest

import tpt_fem as F
from meshes import box, jitter, quad_grid, tri_grid
from oracle import exodus_oracle as X

pytestmark = pytest.mark.gpu

NAMES = {F.CELL_TET4: "TET4", F.CELL_QUAD4: "QUAD4", F.CELL_TRI3: "TRI3"}


def check(ctx, tmp_path, cell, c, e):
    m = F.Mesh.from_arrays(cell, c, e, ctx=ctx)
    out = tmp_path / "mesh.exo"
    m.write_exodus(out)
    got = out.read_bytes()
    want = X.mesh_to_exodus_bytes(c.tolist(), [(NAMES[cell], list(map(int, row))) for row in e])
    assert got == want
    coords, cells = X.bytes_to_mesh(got)
    assert [n for _, n in cells] == e.tolist()
    assert np.allclose(np.array(coords)[:, :c.shape[1]], c, rtol=1e-7, atol=1e-7)


def test_exodus_tet_box(ctx, tmp_path):
    c, e = box([3, 2, 2], mx=(2.0, 1.0, 1.0))
    check(ctx, tmp_path, F.CELL_TET4, jitter(c, 0.03, 1), e)


def test_exodus_tri3(ctx, tmp_path):
    c, e = tri_grid(5, 4, 2.0, 1.0)
    check(ctx, tmp_path, F.CELL_TRI3, jitter(c, 0.05, 2), e)


def test_exodus_quad4(ctx, tmp_path):
    c, e = quad_grid(4, 3, 1.5, 1.0)
    check(ctx, tmp_path, F.CELL_QUAD4, jitter(c, 0.05, 3), e)
