"""Legacy VTK export of device-resident meshes and fields (write_vtk /
write_vtk_with_data, crates/tpt-fem-io-vtk/src/lib.rs:117-196), pinned byte
for byte to files the reference wrote: mesh_gen_box_structured.vtk
(box_mesh 4^3, crates/tpt-fem/examples/mesh_gen_box.rs) and thermal_solve.vtk
(box_mesh 6^3 with a temperature field).  tests/golden/vtk_digests.json holds
their lengths and SHA-256; box6_thermal_mesh.npz holds that file's field."""
import hashlib
import json
import os

import numpy as np
import pytest

import tpt_fem as F
from meshes import tri_grid

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def digest(path):
    data = open(path, "rb").read()
    return {"bytes": len(data), "sha256": hashlib.sha256(data).hexdigest()}


def golden(name):
    return json.load(open(os.path.join(GOLDEN, "vtk_digests.json")))[name]


def test_box_mesh_file_matches_reference_bytes(ctx, tmp_path):
    m = F.Mesh.box_mesh([0, 0, 0], [1, 1, 1], [4, 4, 4], ctx=ctx)
    out = tmp_path / "box4.vtk"
    m.write_vtk(out)
    assert digest(out) == golden("mesh_gen_box_structured.vtk")


def test_field_file_matches_reference_bytes(ctx, tmp_path):
    g = np.load(os.path.join(GOLDEN, "box6_thermal_mesh.npz"))
    m = F.Mesh.box_mesh([0, 0, 0], [1, 1, 1], [6, 6, 6], ctx=ctx)
    out = tmp_path / "thermal.vtk"
    m.write_vtk(out, {"temperature": g["stale_temperature"]})
    assert digest(out) == golden("thermal_solve.vtk")


def read_legacy(path):
    data = open(path, "rb").read()

    def section(key):
        i = data.index(key)
        j = data.index(b"\n", i)
        return data[i:j].split(), j + 1

    (_, n, _), p0 = section(b"POINTS")
    pts = np.frombuffer(data, ">f8", 3 * int(n), p0).reshape(-1, 3)
    (_, m, k), c0 = section(b"CELLS")
    cells = np.frombuffer(data, ">i4", int(k), c0)
    (_, _), t0 = section(b"CELL_TYPES")
    types = np.frombuffer(data, ">i4", int(m), t0)
    fields = {}
    i = 0
    while True:
        i = data.find(b"\nSCALARS ", i)
        if i < 0:
            break
        name = data[i + 9:data.index(b" ", i + 9)].decode()
        s0 = data.index(b"LOOKUP_TABLE default\n", i) + len(b"LOOKUP_TABLE default\n")
        fields[name] = np.frombuffer(data, ">f8", int(n), s0)
        i = s0
    return pts, cells, types, fields, data


def test_tri3_mesh_with_two_fields(ctx, tmp_path):
    c, e = tri_grid(5, 3, 2.0, 1.0)
    m = F.Mesh.from_arrays(F.CELL_TRI3, c, e, ctx=ctx)
    u = np.sin(c[:, 0]) * c[:, 1]
    K = F.assemble_poisson(m, 1.0, 2)
    rhs = F.load_poisson_source(m, 1.0, 2)
    bcs = [(i, 0.0) for i in m.nodes_on_plane(0, 0.0, 1e-9)]
    sol, _ = F.solve_with_dirichlet(K, rhs, bcs, tol=1e-12)
    out = tmp_path / "tri.vtk"
    m.write_vtk(out, {"u": sol, "g": u}, title="tri3 result")
    pts, cells, types, fields, data = read_legacy(out)
    assert data.startswith(b"# vtk DataFile Version 4.1\ntri3 result\nBINARY\n")
    assert np.array_equal(pts[:, :2], c) and not pts[:, 2].any()
    assert np.array_equal(cells.reshape(-1, 4)[:, 0], np.full(len(e), 3))
    assert np.array_equal(cells.reshape(-1, 4)[:, 1:], e)
    assert np.array_equal(types, np.full(len(e), 5))
    assert np.array_equal(fields["u"], sol) and np.array_equal(fields["g"], u)
    assert data.endswith(b"\n\nCELL_DATA %d\n\n" % len(e))


def test_bad_field_names_are_rejected(ctx, tmp_path):
    m = F.Mesh.box_mesh([0, 0, 0], [1, 1, 1], [2, 2, 2], ctx=ctx)
    with pytest.raises(F.TptFemError):
        m.write_vtk(tmp_path / "x.vtk", {"two words": np.zeros(m.n_nodes)})
