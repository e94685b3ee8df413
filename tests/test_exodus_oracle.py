"""The Exodus oracle against the reference's own io-exodus tests
(crates/tpt-fem-io-exodus/src/lib.rs:735-878), restated."""
import struct

import pytest

from oracle import exodus_oracle as X


def test_round_trips_tri_mesh():  # io-exodus:736
    b = X.mesh_to_exodus_bytes([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]], [("TRI3", [0, 1, 2])])
    assert b[:4] == b"CDF\x01"
    coords, cells = X.bytes_to_mesh(b)
    assert len(coords) == 3 and cells == [("TRI3", [0, 1, 2])]
    assert abs(coords[1][0] - 1.0) < 1e-6


def test_round_trips_multi_block():  # io-exodus:755
    pts = [[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0], [2.0, 0.0]]
    cells = [("TRI3", [0, 1, 2]), ("QUAD4", [1, 3, 2, 0]), ("TRI3", [1, 4, 3])]
    _, back = X.bytes_to_mesh(X.mesh_to_exodus_bytes(pts, cells))
    assert len(back) == 3
    assert sum(c == "TRI3" for c, _ in back) == 2 and sum(c == "QUAD4" for c, _ in back) == 1


@pytest.mark.parametrize("data", [b"NOPE", b"CDF\x01"])  # io-exodus:786, 792
def test_rejects_bad_or_truncated_header(data):
    with pytest.raises(X.ParseError):
        X.bytes_to_mesh(data)


def test_rejects_implausible_dimension_count():  # io-exodus:798
    b = b"CDF\x01" + struct.pack(">III", 0, X.NC_DIMENSION, 0xFFFFFFF0)
    with pytest.raises(X.ParseError):
        X.bytes_to_mesh(b)


def test_rejects_truncated_name():  # io-exodus:808
    b = b"CDF\x01" + struct.pack(">III", 0, X.NC_DIMENSION, 1) + bytes([200]) + b"ab"
    with pytest.raises(X.ParseError):
        X.bytes_to_mesh(b)


@pytest.mark.parametrize("bad", [0, 99])  # io-exodus:819, 841
def test_rejects_connect_node_ids_out_of_range(bad):
    b = bytearray(X.mesh_to_exodus_bytes([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]], [("TRI3", [0, 1, 2])]))
    _, v = X.decode_nc3(bytes(b))
    data = v["connect1"][2]
    i = bytes(b).index(data)
    b[i:i + 4] = struct.pack(">I", bad)
    with pytest.raises(X.ParseError):
        X.bytes_to_mesh(bytes(b))


def test_rejects_coords_wrong_dtype():  # io-exodus:863
    b = bytearray(X.mesh_to_exodus_bytes([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]], [("TRI3", [0, 1, 2])]))
    i = bytes(b).index(X._name("coords"))
    j = i + len(X._name("coords")) + 4 + 8 + 4  # name, ndims, two dim ids, natts
    assert struct.unpack(">I", bytes(b[j:j + 4]))[0] == X.NC_FLOAT
    b[j:j + 4] = struct.pack(">I", X.NC_INT)
    with pytest.raises(X.ParseError):
        X.bytes_to_mesh(bytes(b))


def test_layout_offsets_are_four_byte_aligned():
    b = X.mesh_to_exodus_bytes([[0.0, 0.0, 0.0]] * 5, [("TET4", [0, 1, 2, 3]), ("TET4", [1, 2, 3, 4])])
    _, v = X.decode_nc3(b)
    assert len(b) % 4 == 0
    for name, (_, _, data) in v.items():
        assert b.index(data) % 4 == 0 or not data
