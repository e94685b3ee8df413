"""Regenerate the committed golden fixtures from the reference checkout.

Run once where the reference tree is checked out, with its root as the one
required argument (``python make_golden.py <tpt-fem checkout>``); the tests
only read the ``.npz`` files this writes.

Fixtures:
  box4_structured.npz   points (125,3) and connectivity (384,4) of
                        ``mesh_gen_box_structured.vtk``, written by
                        crates/tpt-fem/examples/mesh_gen_box.rs:15-21 from
                        box_mesh([0,0,0],[1,1,1],[4,4,4]).
  vtk_digests.json      byte length and SHA-256 of those two files, the
                        golden bytes of the reference's VTK writer
                        (crates/tpt-fem-io-vtk/src/lib.rs:117-196).
  box6_thermal_mesh.npz points and connectivity of ``thermal_solve.vtk``
                        (box_mesh([6,6,6]) per crates/tpt-fem/examples/
                        thermal_solve.rs).  Its temperature field is stale
                        (written by an older transposed-inverse Map) and is
                        stored only under the key ``stale_temperature`` so a
                        test can show why it is not a value golden.
"""
import os
import sys

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))


def parse_legacy_vtk(path):
    """Legacy binary VTK (big-endian) unstructured grid: points, tets, point scalars."""
    data = open(path, "rb").read()

    def header(key):
        i = data.find(key)
        j = data.find(b"\n", i)
        return data[i:j].split(), j + 1

    (_, npts, _), p0 = header(b"POINTS")
    npts = int(npts)
    pts = np.frombuffer(data, dtype=">f8", count=3 * npts, offset=p0).astype(np.float64).reshape(npts, 3)
    (_, ncell, nint), c0 = header(b"CELLS")
    ncell, nint = int(ncell), int(nint)
    raw = np.frombuffer(data, dtype=">i4", count=nint, offset=c0).astype(np.int64)
    cells = raw.reshape(ncell, -1)
    assert np.all(cells[:, 0] == 4), "expected tetrahedra"
    out = {"points": pts, "conn": cells[:, 1:].copy()}
    i = data.find(b"LOOKUP_TABLE default\n")
    if i >= 0:
        s0 = i + len(b"LOOKUP_TABLE default\n")
        out["stale_temperature"] = np.frombuffer(data, dtype=">f8", count=npts, offset=s0).astype(np.float64)
    return out


def write_digests(ref):
    import hashlib
    import json
    out = {}
    for name in ("mesh_gen_box_structured.vtk", "thermal_solve.vtk"):
        data = open(os.path.join(ref, name), "rb").read()
        out[name] = {"bytes": len(data), "sha256": hashlib.sha256(data).hexdigest()}
    with open(os.path.join(OUT, "vtk_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path of the tpt-fem checkout>")
    ref = sys.argv[1]
    g = parse_legacy_vtk(os.path.join(ref, "mesh_gen_box_structured.vtk"))
    np.savez_compressed(os.path.join(OUT, "box4_structured.npz"), points=g["points"], conn=g["conn"])
    t = parse_legacy_vtk(os.path.join(ref, "thermal_solve.vtk"))
    np.savez_compressed(os.path.join(OUT, "box6_thermal_mesh.npz"), points=t["points"], conn=t["conn"],
                        stale_temperature=t["stale_temperature"])
    write_digests(ref)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
