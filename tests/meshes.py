"""Seeded test meshes shared by the parity tests (inputs only, no reference logic)."""
import numpy as np

from oracle import oracle as O


def box(n, mn=(0.0, 0.0, 0.0), mx=(1.0, 1.0, 1.0)):
    return O.box_mesh(list(mn), list(mx), list(n))


def jitter(coords, amp, seed, keep_boundary=True):
    """Move interior nodes by up to amp * (cell size) so every element is general."""
    rng = np.random.default_rng(seed)
    c = coords.copy()
    lo, hi = c.min(axis=0), c.max(axis=0)
    d = rng.uniform(-amp, amp, size=c.shape)
    if keep_boundary:
        on_b = np.any((np.abs(c - lo) < 1e-12) | (np.abs(c - hi) < 1e-12), axis=1)
        d[on_b] = 0.0
    return c + d


def quad_grid(nx, ny, lx=1.0, ly=1.0):
    """Structured Quad4 grid: node j*(nx+1)+i at (i*lx/nx, j*ly/ny), counter-clockwise elements."""
    xs = np.arange(nx + 1) * (lx / nx)
    ys = np.arange(ny + 1) * (ly / ny)
    coords = np.array([[x, y] for y in ys for x in xs])
    conn = []
    for j in range(ny):
        for i in range(nx):
            n0 = j * (nx + 1) + i
            conn.append([n0, n0 + 1, n0 + nx + 2, n0 + nx + 1])
    return coords, np.array(conn, dtype=np.int64)


def unit_cube_bcs(coords, dpn=1):
    nodes = set()
    for axis in range(3):
        for coord in (0.0, 1.0):
            nodes |= set(int(i) for i in O.nodes_on_plane(coords, axis, coord, 1e-9))
    return [(n * dpn + k, 0.0) for n in sorted(nodes) for k in range(dpn)]


def tri_grid(nx, ny, lx=1.0, ly=1.0):
    """Structured Tri3 grid: each cell of quad_grid split along alternating
    diagonals into two counter-clockwise triangles."""
    coords, quads = quad_grid(nx, ny, lx, ly)
    tris = []
    for k, (a, b, c, d) in enumerate(quads):
        i, j = k % nx, k // nx
        if (i + j) % 2 == 0:
            tris += [[a, b, c], [a, c, d]]
        else:
            tris += [[a, b, d], [b, c, d]]
    return coords, np.array(tris, dtype=np.int64)
