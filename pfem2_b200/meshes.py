"""Programmatic meshes for the PFEM2 workloads (the cases' build_grid).

The reference builds its meshes with deal.II (GridGenerator::subdivided_hyper_rectangle
with colorize=true in tube_Poiseuille/tube (Vx-driven).cc:91-101 and
tubePoiseuille3D/tube.cc:72-81) or reads UNV files (cylinder2D/cylinder2D.cc:266-277).
Here every mesh is generated in numpy with deal.II's conventions:

* cell vertices in lexicographic order (vertex v has reference coordinate
  bit d of v on axis d), all cells with positive Jacobian;
* face f lies on reference axis f//2 at side f%2; face_boundary_id is -1
  for interior faces;
* colorized boxes: the faces at x=min, x=max, y=min, y=max, z=min, z=max
  get ids 0..5.

A Mesh is (vertices [nv, dim] f64, cells [nc, 2^dim] i32, face_bid [nc, 2 dim] i32).
Cells are ordered along a Morton curve of their centroids and vertices by
first use, which keeps each cell's neighbourhood close in memory.
"""
from dataclasses import dataclass

import numpy as np


@dataclass
class Mesh:
    vertices: np.ndarray
    cells: np.ndarray
    face_bid: np.ndarray

    @property
    def dim(self):
        return self.vertices.shape[1]

    @property
    def n_vertices(self):
        return self.vertices.shape[0]

    @property
    def n_cells(self):
        return self.cells.shape[0]


def _morton_key(pts, bits=20):
    lo = pts.min(axis=0)
    span = np.maximum(pts.max(axis=0) - lo, 1e-300)
    q = np.floor((pts - lo) / span * (2 ** bits - 1)).astype(np.uint64)
    key = np.zeros(len(pts), dtype=np.uint64)
    dim = pts.shape[1]
    for b in range(bits):
        for d in range(dim):
            key |= ((q[:, d] >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * dim + d)
    return key


def _finish(vertices, cells, face_bid, reorder=True):
    """Drops unused vertices, orders cells on a Morton curve and vertices by first use."""
    vertices = np.asarray(vertices, dtype=np.float64)
    cells = np.asarray(cells, dtype=np.int64)
    face_bid = np.asarray(face_bid, dtype=np.int32)
    if reorder:
        cen = vertices[cells].mean(axis=1)
        order = np.argsort(_morton_key(cen), kind="stable")
        cells = cells[order]
        face_bid = face_bid[order]
    used_order = []
    seen = np.full(len(vertices), -1, dtype=np.int64)
    flat = cells.reshape(-1)
    # first-use numbering
    first = np.unique(flat, return_index=True)
    ordv = first[0][np.argsort(first[1], kind="stable")]
    seen[ordv] = np.arange(len(ordv))
    del used_order
    new_cells = seen[cells]
    return Mesh(vertices[ordv].copy(), new_cells.astype(np.int32), face_bid.astype(np.int32))


def _merge_vertices(points, tol=1e-9):
    """Merges coincident points; returns (unique_points, index_map)."""
    scale = np.abs(points).max() + 1.0
    key = np.round(points / (tol * scale)).astype(np.int64)
    _, first, inv = np.unique(key, axis=0, return_index=True, return_inverse=True)
    return points[first], inv.reshape(-1)


def rect_mesh(nx, ny, x0=0.0, x1=1.0, y0=0.0, y1=1.0, reorder=True):
    """subdivided_hyper_rectangle(tria, {nx, ny}, (x0,y0), (x1,y1), colorize=true)."""
    xs = np.linspace(x0, x1, nx + 1)
    ys = np.linspace(y0, y1, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    verts = np.stack([X.ravel(), Y.ravel()], axis=1)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    i = i.ravel(); j = j.ravel()
    v0 = j * (nx + 1) + i
    cells = np.stack([v0, v0 + 1, v0 + nx + 1, v0 + nx + 2], axis=1)
    fb = np.full((len(cells), 4), -1, dtype=np.int32)
    fb[i == 0, 0] = 0
    fb[i == nx - 1, 1] = 1
    fb[j == 0, 2] = 2
    fb[j == ny - 1, 3] = 3
    return _finish(verts, cells, fb, reorder)


def box_mesh(nx, ny, nz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), reorder=True):
    """subdivided_hyper_rectangle in 3D, colorized (ids 0..5)."""
    xs = np.linspace(lo[0], hi[0], nx + 1)
    ys = np.linspace(lo[1], hi[1], ny + 1)
    zs = np.linspace(lo[2], hi[2], nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    verts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i = i.ravel(); j = j.ravel(); k = k.ravel()
    sx, sy = 1, nx + 1
    sz = (nx + 1) * (ny + 1)
    v0 = k * sz + j * sy + i
    cells = np.stack([v0 + ((v & 1) * sx + ((v >> 1) & 1) * sy + ((v >> 2) & 1) * sz) for v in range(8)], axis=1)
    fb = np.full((len(cells), 6), -1, dtype=np.int32)
    fb[i == 0, 0] = 0; fb[i == nx - 1, 1] = 1
    fb[j == 0, 2] = 2; fb[j == ny - 1, 3] = 3
    fb[k == 0, 4] = 4; fb[k == nz - 1, 5] = 5
    return _finish(verts, cells, fb, reorder)


def _graded(n, ratio):
    """n+1 points on [0,1], geometric growth `ratio` between successive cells."""
    if abs(ratio - 1.0) < 1e-12:
        return np.linspace(0.0, 1.0, n + 1)
    w = ratio ** np.arange(n)
    s = np.concatenate([[0.0], np.cumsum(w)])
    return s / s[-1]


def channel_disk_mesh(h=0.0088, length=4.0, height=1.0, center=(0.5, 0.5), radius=0.1,
                      half_square=None, radial_ratio=1.08, reorder=True):
    """2D channel [0,length]x[0,height] with a disk obstacle: an O-grid of 4
    blocks between the circle and a square around it, plus a tensor grid of
    blocks outside the square. Boundary ids follow cylinder2D: 1 inlet (x=0),
    2 outlet (x=length), 3 disk, 4 walls (y=0, y=height).

    `h` is the target cell size away from the disk; ~50k cells at h=0.0088.
    """
    cx, cy = center
    s = half_square if half_square is not None else min(max(0.2, radius + 0.1), 0.45 * min(cy, height - cy) / 0.5)
    s = min(s, cx - 1e-3, cy - 1e-3, height - cy - 1e-3)
    xa, xb = cx - s, cx + s
    ya, yb = cy - s, cy + s
    n_s = max(4, int(round(2 * s / h)))
    n1x = max(1, int(round(xa / h)))
    n3x = max(1, int(round((length - xb) / h)))
    n1y = max(1, int(round(ya / h)))
    n3y = max(1, int(round((height - yb) / h)))
    xs = np.concatenate([np.linspace(0, xa, n1x + 1)[:-1], np.linspace(xa, xb, n_s + 1)[:-1], np.linspace(xb, length, n3x + 1)])
    ys = np.concatenate([np.linspace(0, ya, n1y + 1)[:-1], np.linspace(ya, yb, n_s + 1)[:-1], np.linspace(yb, height, n3y + 1)])
    ix0, ix1 = n1x, n1x + n_s
    iy0, iy1 = n1y, n1y + n_s
    NX, NY = len(xs) - 1, len(ys) - 1
    pts = []
    cells = []
    fbs = []

    def add_pt(p):
        pts.append(p)
        return len(pts) - 1

    # tensor grid outside the square
    gid = np.full((NY + 1, NX + 1), -1, dtype=np.int64)
    for j in range(NY + 1):
        for i in range(NX + 1):
            if ix0 < i < ix1 and iy0 < j < iy1:
                continue
            gid[j, i] = add_pt((xs[i], ys[j]))
    for j in range(NY):
        for i in range(NX):
            if ix0 <= i < ix1 and iy0 <= j < iy1:
                continue
            c = [gid[j, i], gid[j, i + 1], gid[j + 1, i], gid[j + 1, i + 1]]
            fb = [-1, -1, -1, -1]
            if i == 0: fb[0] = 1
            if i == NX - 1: fb[1] = 2
            if j == 0: fb[2] = 4
            if j == NY - 1: fb[3] = 4
            cells.append(c); fbs.append(fb)
    # O-grid: n_s cells along each square side, n_r radial layers
    dist = s * np.sqrt(2.0)
    n_r = max(2, int(round((s - radius) / h * 1.3)))
    rad = _graded(n_r, radial_ratio)
    # square perimeter points, counter-clockwise starting at (xa, ya)
    sq = []
    for t in range(n_s):  # bottom: (xa..xb, ya)
        sq.append((xs[ix0 + t], ya))
    for t in range(n_s):  # right: (xb, ya..yb)
        sq.append((xb, ys[iy0 + t]))
    for t in range(n_s):  # top: (xb..xa, yb)
        sq.append((xs[ix1 - t], yb))
    for t in range(n_s):  # left: (xa, yb..ya)
        sq.append((xa, ys[iy1 - t]))
    sq = np.array(sq)
    nper = len(sq)
    ring = np.zeros((n_r + 1, nper), dtype=np.int64)
    for k in range(nper):
        ps = sq[k]
        d = ps - np.array([cx, cy])
        pc = np.array([cx, cy]) + radius * d / np.linalg.norm(d)
        for l in range(n_r + 1):
            p = pc + (ps - pc) * rad[l]
            ring[l, k] = add_pt((p[0], p[1]))
    del dist
    for l in range(n_r):
        for k in range(nper):
            k1 = (k + 1) % nper
            # local frame: axis 0 outward (away from the disk), axis 1 along
            # the perimeter counter-clockwise -> positive orientation
            c = [ring[l, k], ring[l + 1, k], ring[l, k1], ring[l + 1, k1]]
            fb = [-1, -1, -1, -1]
            if l == 0:
                fb[0] = 3
            cells.append(c); fbs.append(fb)
    pts = np.array(pts, dtype=np.float64)
    uniq, inv = _merge_vertices(pts)
    cells = inv[np.array(cells, dtype=np.int64)]
    mesh = _finish(uniq, cells, np.array(fbs, dtype=np.int32), reorder)
    _check_orientation(mesh)
    return mesh


def pipe_mesh(ny=64, nz=64, nx=256, length=4.0, radius=0.5, reorder=True):
    """3D pipe along x with a circular cross-section mapped from a square
    (elliptical grid map (u,v) -> (u sqrt(1-v^2/2), v sqrt(1-u^2/2))).
    Boundary ids: 0 inlet (x=0), 1 outlet (x=length), 2 wall."""
    us = np.linspace(-1.0, 1.0, ny + 1)
    vs = np.linspace(-1.0, 1.0, nz + 1)
    xs = np.linspace(0.0, length, nx + 1)
    V, U = np.meshgrid(vs, us, indexing="ij")
    Yc = radius * U * np.sqrt(1.0 - V * V / 2.0)
    Zc = radius * V * np.sqrt(1.0 - U * U / 2.0)
    # vertex (i along x, j along y(u), k along z(v))
    K, J, I = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    verts = np.stack([xs[I.ravel()], Yc[K.ravel(), J.ravel()], Zc[K.ravel(), J.ravel()]], axis=1)
    sx, sy, sz = 1, nx + 1, (nx + 1) * (ny + 1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i = i.ravel(); j = j.ravel(); k = k.ravel()
    v0 = k * sz + j * sy + i
    cells = np.stack([v0 + ((v & 1) * sx + ((v >> 1) & 1) * sy + ((v >> 2) & 1) * sz) for v in range(8)], axis=1)
    fb = np.full((len(cells), 6), -1, dtype=np.int32)
    fb[i == 0, 0] = 0; fb[i == nx - 1, 1] = 1
    fb[j == 0, 2] = 2; fb[j == ny - 1, 3] = 2
    fb[k == 0, 4] = 2; fb[k == nz - 1, 5] = 2
    mesh = _finish(verts, cells, fb, reorder)
    _check_orientation(mesh)
    return mesh


def _check_orientation(mesh):
    """Asserts a positive Jacobian determinant at all cell vertices."""
    X = mesh.vertices[mesh.cells]  # nc, nvc, dim
    dim = mesh.dim
    if dim == 2:
        for v in range(4):
            b = [(v >> d) & 1 for d in range(2)]
            e0 = X[:, v ^ 1] - X[:, v]
            e1 = X[:, v ^ 2] - X[:, v]
            s0 = 1 if b[0] == 0 else -1
            s1 = 1 if b[1] == 0 else -1
            det = s0 * s1 * (e0[:, 0] * e1[:, 1] - e0[:, 1] * e1[:, 0])
            if not np.all(det > 0):
                raise ValueError("mesh has inverted cells")
    else:
        for v in range(8):
            b = [(v >> d) & 1 for d in range(3)]
            es = [(X[:, v ^ (1 << d)] - X[:, v]) * (1 if b[d] == 0 else -1) for d in range(3)]
            det = np.einsum("ij,ij->i", es[0], np.cross(es[1], es[2]))
            if not np.all(det > 0):
                raise ValueError("mesh has inverted cells")


def nearest_vertex(mesh, point):
    d = np.linalg.norm(mesh.vertices - np.asarray(point)[None, :], axis=1)
    return int(np.argmin(d))
