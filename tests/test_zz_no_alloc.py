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


def call_noalloc(lib, torch, mesh, particles):
    cell, xi, u = particles
    dim = mesh.dim
    ptr, vc, vl = vertex_cells(mesh)
    start = np.concatenate([[0], np.cumsum(np.bincount(cell, minlength=mesh.n_cells))]).astype(np.int32)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    t = [dev(ptr), dev(vc), dev(vl), dev(start), dev(xi.astype(np.float64)), dev(u.astype(np.float64))]
    node_u = torch.full((mesh.n_vertices, dim), float("nan"), dtype=torch.float64, device="cuda")
    node_w = torch.full((mesh.n_vertices,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    st = lib.pfem2_project_noalloc(dim, mesh.n_cells, mesh.n_vertices, *[C.c_void_p(x.data_ptr()) for x in t],
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


def test_noalloc_rejects_too_many_cells():
    torch = pytest.importorskip("torch")
    lib = load_library()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    st = lib.pfem2_project_noalloc(2, 65536 + 1, 4, p, p, p, p, p, p, p, p, C.c_void_p(0))
    assert st == A.INVALID_ARG
    assert b"PFEM2_NOALLOC_MAX_CELLS" in lib.pfem2_last_error()
