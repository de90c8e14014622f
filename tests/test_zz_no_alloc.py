"""GPU test of pfem2_project_noalloc, the projection entry point for callers
that cannot let the library allocate device memory (their own memory pool,
or work recorded into a CUDA graph). It runs on caller-owned buffers and
keeps its scratch in a fixed device array; its result must equal the
projection of the context-based entry point, call after call.

The file name sorts last on purpose: a run that stops at the first failure
has run every other test before this one. It passes alone in a fresh
process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from pfem2_b200 import _abi as A
from pfem2_b200 import cases
from pfem2_b200.solver import Solver, load_library

pytestmark = pytest.mark.gpu

TOL = 1e-13  # the FP64 projection tolerance of the parity tests


def vertex_cells(mesh):
    """cells around each vertex (ascending) and the vertex's local index there"""
    nvc = mesh.cells.shape[1]
    v = mesh.cells.reshape(-1).astype(np.int64)
    c = np.repeat(np.arange(mesh.n_cells), nvc)
    loc = np.tile(np.arange(nvc), mesh.n_cells)
    order = np.lexsort((c, v))
    ptr = np.concatenate([[0], np.cumsum(np.bincount(v, minlength=mesh.n_vertices))]).astype(np.int32)
    return ptr, c[order].astype(np.int32), loc[order].astype(np.int32)


def wall_flags(mesh, bids):
    """1 on the vertices of boundary faces with the given ids (the context's
    zero_after_projection vertices): face f of a cell lies on axis f // 2 at
    side f % 2, its vertices have that bit of their local index set to f % 2"""
    flag = np.zeros(mesh.n_vertices, np.uint8)
    nvc = mesh.cells.shape[1]
    for f in range(mesh.face_bid.shape[1]):
        on = np.isin(mesh.face_bid[:, f], bids)
        for b in range(nvc):
            if ((b >> (f // 2)) & 1) == f % 2:
                flag[mesh.cells[on, b]] = 1
    return flag


def call_noalloc(lib, torch, mesh, particles, zero_flag=None, incidences=None):
    cell, xi, u = particles
    dim = mesh.dim
    ptr, vc, vl = incidences if incidences is not None else vertex_cells(mesh)
    start = np.concatenate([[0], np.cumsum(np.bincount(cell, minlength=mesh.n_cells))]).astype(np.int32)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    t = [dev(ptr), dev(vc), dev(vl), dev(start), dev(xi.astype(np.float64)), dev(u.astype(np.float64))]
    zf = dev(zero_flag) if zero_flag is not None else None
    node_u = torch.full((mesh.n_vertices, dim), float("nan"), dtype=torch.float64, device="cuda")
    node_w = torch.full((mesh.n_vertices,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    st = lib.pfem2_project_noalloc(dim, mesh.n_cells, mesh.n_vertices, *[C.c_void_p(x.data_ptr()) for x in t],
                                   C.c_void_p(zf.data_ptr() if zf is not None else 0),
                                   C.c_void_p(node_u.data_ptr()), C.c_void_p(node_w.data_ptr()),
                                   C.c_void_p(stream.cuda_stream))
    assert st == A.OK, lib.pfem2_last_error().decode()
    stream.synchronize()
    return node_u.cpu().numpy(), node_w.cpu().numpy()


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("dim", [2, 3])
def test_noalloc_projection_matches_context_twice(dim):
    torch = pytest.importorskip("torch")
    lib = load_library()
    sp = cases.poiseuille_2d(nx=32, ny=12) if dim == 2 else cases.pipe_3d(ny=6, nz=6, nx=12)
    g = Solver(sp, precision=A.PREC_FP64)
    X = sp.mesh.vertices
    fields = [1.0 + 0.3 * np.sin(2.0 * X[:, 1]), 0.2 * np.cos(1.5 * X[:, 0])] + ([0.1 * X[:, 2]] if dim == 3 else [])
    for d in range(dim):
        g.set_field(A.FIELD_VX + d, fields[d])
    q = (4, 4) if dim == 2 else (3, 3, 3)
    g.seed_particles(q, seed=3, jitter=0.1)
    for call in range(2):
        if call == 1:
            # change the carried velocities, then compare again: the shared
            # scratch must not leak the first call's contents
            for d in range(dim):
                g.set_field(A.FIELD_OLD_VX + d, fields[d])
                g.set_field(A.FIELD_VX + d, 0.5 * fields[d] + 0.1 * d)
            g.correct_particles_velocities()
        g.distribute_particle_velocities_to_grid()
        ref_u = np.stack([g.field(A.FIELD_VX + d) for d in range(dim)], axis=1)
        ref_w = g.field(A.FIELD_NODE_WEIGHT)
        nu, nw = call_noalloc(lib, torch, sp.mesh, g.particles())
        assert rel(nw, ref_w) <= TOL
        assert rel(nu, ref_u) <= TOL
    g.close()


def test_noalloc_wall_vertices():
    """a channel whose disk and walls are zeroed after the projection
    (zero_after_projection_mask): with the same zero flags the entry point
    equals the context's projection; without flags the wall vertices keep
    their projected velocity"""
    torch = pytest.importorskip("torch")
    lib = load_library()
    sp = cases.channel_disk(h=0.05, zero_ids=(3, 4))
    g = Solver(sp, precision=A.PREC_FP64)
    X = sp.mesh.vertices
    g.set_field(A.FIELD_VX, 1.0 + 0.3 * np.sin(2.0 * X[:, 1]))
    g.set_field(A.FIELD_VY, 0.2 * np.cos(1.5 * X[:, 0]))
    g.seed_particles(sp.q, seed=4, jitter=0.1)
    g.distribute_particle_velocities_to_grid()
    ref_u = np.stack([g.field(A.FIELD_VX + d) for d in range(2)], axis=1)
    ref_w = g.field(A.FIELD_NODE_WEIGHT)
    flags = wall_flags(sp.mesh, (3, 4))
    assert flags.sum() > 0
    for _ in range(2):
        nu, nw = call_noalloc(lib, torch, sp.mesh, g.particles(), zero_flag=flags)
        assert rel(nw, ref_w) <= TOL
        assert rel(nu, ref_u) <= TOL
    nu, _ = call_noalloc(lib, torch, sp.mesh, g.particles())
    wall = flags != 0
    assert np.array_equal(nu[~wall], call_noalloc(lib, torch, sp.mesh, g.particles(), zero_flag=flags)[0][~wall])
    assert np.abs(nu[wall]).max() > 0.1 and np.all(ref_u[wall] == 0.0)
    g.close()


def test_noalloc_out_of_range_incidence():
    """an incidence naming a cell beyond n_cells makes that vertex NaN and
    leaves the others exact"""
    torch = pytest.importorskip("torch")
    lib = load_library()
    sp = cases.poiseuille_2d(nx=16, ny=6)
    g = Solver(sp, precision=A.PREC_FP64)
    g.set_field(A.FIELD_VX, np.ones(sp.mesh.n_vertices))
    g.seed_particles((3, 3), seed=1, jitter=0.1)
    parts = g.particles()
    good_u, good_w = call_noalloc(lib, torch, sp.mesh, parts)
    ptr, vc, vl = vertex_cells(sp.mesh)
    v = 40
    vc = vc.copy()
    vc[ptr[v]] = sp.mesh.n_cells
    bad_u, bad_w = call_noalloc(lib, torch, sp.mesh, parts, incidences=(ptr, vc, vl))
    assert np.isnan(bad_w[v]) and np.all(np.isnan(bad_u[v]))
    keep = np.arange(sp.mesh.n_vertices) != v
    assert np.array_equal(bad_u[keep], good_u[keep]) and np.array_equal(bad_w[keep], good_w[keep])
    g.close()


def test_noalloc_rejects_too_many_cells():
    torch = pytest.importorskip("torch")
    lib = load_library()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    st = lib.pfem2_project_noalloc(2, 65536 + 1, 4, p, p, p, p, p, p, C.c_void_p(0), p, p, C.c_void_p(0))
    assert st == A.INVALID_ARG
    assert b"PFEM2_NOALLOC_MAX_CELLS" in lib.pfem2_last_error()
