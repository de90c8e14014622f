"""Parity of the library (through the C ABI) with the FP64 oracle on the
benchmark workloads themselves, not only on toy meshes:

- the 2D Poiseuille channel in full: 64x16 Q1 cells, 4x4 particles per cell
  with +-0.1 jitter (seed 0), dt = 0.005, 200 steps
  (tube_Poiseuille/tube (Vx-driven).cc:48-52 inflow);
- the ~52k-cell channel with a disk obstacle, a few steps;
- the 3D pipe at 32x32x128 hex cells, one step.

The solves run to a relative tolerance of 1e-11 in both implementations, so
that they agree far below the parity bars (1e-12 is at the FP64 floor of the
pipe's solves). Particle membership must be
exact except within 1e-6 (reference units) of a face.
"""
import os

import numpy as np
import pytest

import oracle as O
from pfem2_b200 import _abi as A
from pfem2_b200 import cases
from pfem2_b200.solver import Solver
from tests.helpers import compare_particles, rel_l2

pytestmark = pytest.mark.gpu

THREADS = max(1, min(16, os.cpu_count() or 1))


def tight(sp, rtol=1e-11):
    sp.case.vel_tol = sp.case.p_tol = 0.0
    sp.case.vel_rtol = sp.case.p_rtol = rtol
    return sp


def run_pair(sp, steps, prec=A.PREC_FP64, **kw):
    g = Solver(sp, precision=prec, **kw)
    o = O.Oracle(sp.mesh, sp.case, movement_steps=sp.movement_steps, max_per_part=sp.max_per_part,
                 threads=THREADS)
    g.seed_particles(sp.q, sp.seed, sp.jitter)
    o.seed_particles(sp.q, sp.seed, sp.jitter)
    for _ in range(steps):
        g.step()
        o.step(1)
    return g, o


def fields(dim):
    return [A.FIELD_VX + d for d in range(dim)] + [A.FIELD_P]


def check(g, o, dim, tol, eps_face, xi_tol, u_tol):
    """velocity components against the norm of the whole velocity field (a
    component that is zero up to round-off, like the pipe's cross-flow,
    has no relative error of its own), the pressure against its norm"""
    errs = {}
    vel = [o.field(A.FIELD_VX + d) for d in range(dim)]
    vnorm = float(np.sqrt(sum(np.dot(v, v) for v in vel)))
    for f in fields(dim):
        a, b = g.field(f), o.field(f)
        scale = vnorm if f != A.FIELD_P else float(np.linalg.norm(b))
        errs[f] = float(np.linalg.norm(a - b)) / max(scale, 1e-300)
        assert errs[f] <= tol, (f, errs[f])
    r = compare_particles(o.particles(), g.particles(), eps_face, xi_tol, u_tol)
    return errs, r


def test_poiseuille_full_200_steps():
    """cfg1 exactly as specified, FP64: fields to 1e-8, membership exact
    (no particle flips cell) after 200 steps"""
    sp = tight(cases.poiseuille_2d())
    assert sp.mesh.n_cells == 1024 and sp.q == (4, 4) and sp.jitter == 0.1 and sp.seed == 0
    g, o = run_pair(sp, 200)
    # (after 200 steps the reference coordinates differ by a few 1e-9: the
    # library locates in a cell-local frame, the oracle in global coordinates)
    _, r = check(g, o, 2, 1e-8, 1e-6, 1e-8, 1e-8)
    assert r["flips"] == 0 and r["n_o"] == r["n_g"]
    go, oo = g.stats(), o.stats()
    assert go["deleted"] == oo["deleted"] and go["reseeded"] == oo["reseeded"] and go["removed"] == oo["removed"]
    # the loads of the probe pair agree as well
    # (patch 7 names no boundary: only the probe entry is nonzero)
    gp, op = g.calculate_loads(7)[4], o.calculate_loads(7)[4]
    assert op != 0.0 and abs(gp - op) <= 1e-8 * abs(op)
    g.close()


def test_channel_disk_52k_steps():
    """cfg2's mesh (~52k cells, 25 particles per cell), three steps, FP64"""
    sp = tight(cases.channel_disk())
    assert 45000 < sp.mesh.n_cells < 60000
    g, o = run_pair(sp, 3)
    _, r = check(g, o, 2, 1e-8, 1e-6, 1e-9, 1e-8)
    assert r["flips"] == 0
    gl, ol = g.calculate_loads(3), o.calculate_loads(3)
    assert np.allclose(gl, ol, rtol=1e-7, atol=1e-9), (gl, ol)
    g.close()


def test_pipe_3d_32():
    """cfg4's pipe at 32x32x128 hex cells (27 particles per cell), one step, FP64"""
    sp = tight(cases.pipe_3d(ny=32, nz=32, nx=128))
    g, o = run_pair(sp, 1)
    _, r = check(g, o, 3, 1e-8, 1e-6, 1e-9, 1e-8)
    assert r["flips"] == 0
    g.close()
