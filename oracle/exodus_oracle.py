"""Test-only restatement of the reference's Exodus II writer and reader
(crates/tpt-fem-io-exodus/src/lib.rs): the minimal NetCDF-3 classic (CDF-1)
codec (lib.rs:84-292) and mesh_to_exodus_bytes / bytes_to_mesh
(lib.rs:384-735).  Pure Python on byte strings; it is the checker for the
device library's tptfem_mesh_write_exodus, never part of the product.
Meshes are (cells, coords) with cells a list of (cell_name, node list)."""
import struct

NC_DIMENSION, NC_VARIABLE, NC_FLOAT, NC_INT, NC_CHAR = 10, 11, 5, 4, 2
LEN_NAME = 33
NODES = {"LINE2": 2, "TRI3": 3, "QUAD4": 4, "TET4": 4, "HEX8": 8}


class ParseError(ValueError):
    pass


def _u32(v):
    return struct.pack(">I", v & 0xFFFFFFFF)


def _name(n):  # enc_name (lib.rs:103-113)
    b = n.encode()
    out = bytes([min(len(b), 255)]) + b
    return out + b"\0" * (-len(out) % 4)


def _vsize(dims, dtype, dim_ids):  # vsize_of (lib.rs:123-136)
    s = 1 if dtype == NC_CHAR else 4
    for d in dim_ids:
        s *= dims[d][1]
    if s > 0xFFFFFFFF:
        raise ParseError("variable size overflows u32")
    return s


def _header(dims, vars_, begins):  # build_header (lib.rs:166-192)
    h = b"CDF\x01" + _u32(0) + _u32(NC_DIMENSION) + _u32(len(dims))
    for n, size in dims:
        h += _name(n) + _u32(size)
    h += _u32(NC_VARIABLE) + _u32(len(vars_))
    for (n, dtype, dim_ids, _), b in zip(vars_, begins):
        h += _name(n) + _u32(len(dim_ids)) + b"".join(_u32(d) for d in dim_ids)
        h += _u32(0) + _u32(dtype) + _u32(_vsize(dims, dtype, dim_ids)) + _u32(b)
    return h + _u32(0)


def encode_nc3(dims, vars_):  # encode_nc3 (lib.rs:141-164)
    header = _header(dims, vars_, [0] * len(vars_))
    cursor = (len(header) + 3) & ~3
    begins = []
    for n, dtype, dim_ids, _ in vars_:
        begins.append(cursor)
        cursor = (cursor + _vsize(dims, dtype, dim_ids) + 3) & ~3
    out = bytearray(_header(dims, vars_, begins))
    out += b"\0" * (-len(out) % 4)
    for _, _, _, data in vars_:
        out += data
        out += b"\0" * (-len(out) % 4)
    return bytes(out)


def _floats(v):  # encode_floats (lib.rs:292-298): single precision
    return b"".join(struct.pack(">f", float(x)) for x in v)


def _ints(v):
    return b"".join(_u32(int(x)) for x in v)


def mesh_to_exodus_bytes(coords, cells):
    """mesh_to_exodus_bytes (lib.rs:392-563)."""
    order, blocks = [], []
    for ei, (cell, _) in enumerate(cells):
        if cell in order:
            blocks[order.index(cell)].append(ei)
        else:
            order.append(cell)
            blocks.append([ei])
    nn, ne, nb = len(coords), len(cells), len(order)
    dims = [("num_nodes", nn), ("num_elem", ne), ("num_elem_blk", nb), ("num_node_sets", 0),
            ("num_side_sets", 0), ("len_name", LEN_NAME), ("four", 4), ("time_step", 1), ("num_dim", 3)]
    base = len(dims)
    for bi, cell in enumerate(order):
        dims += [(f"eb{bi}_n", len(blocks[bi])), (f"eb{bi}_np", NODES[cell])]
    c3 = []
    for p in coords:
        c3 += [p[d] if d < len(p) else 0.0 for d in range(3)]
    ids = list(range(1, nb + 1))
    vars_ = [("time_whole", NC_FLOAT, [7], _floats([0.0])),
             ("coords", NC_FLOAT, [0, 8], _floats(c3)),
             ("elem_blk_id", NC_INT, [2], _ints(ids)),
             ("eb_status", NC_INT, [2], _ints([1] * nb)),
             ("eb_prop1", NC_INT, [2], _ints(ids)),
             ("eb_names", NC_CHAR, [5, 2],
              b"".join(c.encode().ljust(LEN_NAME, b"\0")[:LEN_NAME] for c in order))]
    for bi in range(nb):
        conn = [n + 1 for ei in blocks[bi] for n in cells[ei][1]]
        vars_.append((f"connect{bi + 1}", NC_INT, [base + 2 * bi, base + 2 * bi + 1], _ints(conn)))
    vars_.append(("elem_num_map", NC_INT, [1], _ints(range(1, ne + 1))))
    vars_.append(("node_num_map", NC_INT, [0], _ints(range(1, nn + 1))))
    return encode_nc3(dims, vars_)


def _read_u32(b, pos):
    if pos + 4 > len(b):
        raise ParseError("truncated")
    return struct.unpack(">I", b[pos:pos + 4])[0], pos + 4


def _read_name(b, pos):
    if pos >= len(b):
        raise ParseError("truncated name")
    n = b[pos]
    end = pos + 1 + n
    if end > len(b):
        raise ParseError("truncated name")
    name = b[pos + 1:end].decode()
    return name, end + (-(1 + n) % 4)


def _sane(count, b):  # sane_count (lib.rs:138-146)
    if count > len(b) // 4 + 8:
        raise ParseError(f"implausible count {count}")
    return count


def decode_nc3(b):  # decode_nc3 (lib.rs:195-260)
    if len(b) < 4 or b[:4] != b"CDF\x01":
        raise ParseError("not a CDF-1 file")
    pos = 4
    _, pos = _read_u32(b, pos)
    tag, pos = _read_u32(b, pos)
    if tag != NC_DIMENSION:
        raise ParseError("expected dimension tag")
    nd, pos = _read_u32(b, pos)
    dims = []
    for _ in range(_sane(nd, b)):
        n, pos = _read_name(b, pos)
        size, pos = _read_u32(b, pos)
        dims.append((n, size))
    tag, pos = _read_u32(b, pos)
    if tag != NC_VARIABLE:
        raise ParseError("expected variable tag")
    nv, pos = _read_u32(b, pos)
    vars_ = {}
    for _ in range(_sane(nv, b)):
        n, pos = _read_name(b, pos)
        k, pos = _read_u32(b, pos)
        ids = []
        for _ in range(_sane(k, b)):
            d, pos = _read_u32(b, pos)
            if d >= len(dims):
                raise ParseError("dimension id out of range")
            ids.append(d)
        _, pos = _read_u32(b, pos)
        dtype, pos = _read_u32(b, pos)
        _, pos = _read_u32(b, pos)
        begin, pos = _read_u32(b, pos)
        size = _vsize(dims, dtype, ids)
        if begin + size > len(b):
            raise ParseError("variable data out of range")
        vars_[n] = (dtype, ids, b[begin:begin + size])
    return dims, vars_


def bytes_to_mesh(b):
    """bytes_to_mesh (lib.rs:572-735) -> (coords (n, 3), cells)."""
    dims, v = decode_nc3(b)
    if "coords" not in v:
        raise ParseError("missing coords")
    dtype, _, data = v["coords"]
    if dtype != NC_FLOAT:
        raise ParseError("coords variable must be NC_FLOAT")
    c = struct.unpack(f">{len(data) // 4}f", data)
    if len(c) % 3 or not c:
        raise ParseError("bad coords")
    coords = [list(c[i:i + 3]) for i in range(0, len(c), 3)]
    names = []
    if "eb_names" in v:
        raw = v["eb_names"][2]
        names = [raw[i:i + LEN_NAME].rstrip(b"\0").decode() for i in range(0, len(raw), LEN_NAME)]
    cells = []
    for key in sorted((k for k in v if k.startswith("connect")), key=lambda k: int(k[7:] or 0)):
        dtype, ids, data = v[key]
        if dtype != NC_INT:
            raise ParseError("connect must be NC_INT")
        npe = dims[ids[-1]][1]
        name = names[int(key[7:]) - 1]
        if NODES.get(name) != npe:
            raise ParseError("block cell / node count mismatch")
        raw = struct.unpack(f">{len(data) // 4}i", data)
        for e in range(len(raw) // npe):
            nodes = [x - 1 for x in raw[e * npe:(e + 1) * npe]]
            if any(x < 0 or x >= len(coords) for x in nodes):
                raise ParseError("node index out of range")
            cells.append((name, nodes))
    return coords, cells
