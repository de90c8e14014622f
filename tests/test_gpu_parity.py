"""Parity of the CUDA library (through the C ABI) against the FP64 oracle.

Three precision modes (tests/helpers.py MODES): fp64, the default mixed path
(FP32 inner Krylov iterations refined in FP64) and fp32 (every FP32 stage,
FP32 particle coordinates). Membership must match exactly except for
particles within 1e-6 of a cell face (fp64, mixed) or within the measured
2e-5 band of FP32 reference coordinates (fp32); floating point results are
compared with the tolerances written in each test.
"""
import numpy as np
import pytest

import oracle as O
from pfem2_b200 import _abi as A
from pfem2_b200 import cases
from pfem2_b200.solver import Solver
from tests.helpers import MODES, compare_particles, rel_l2, solver_kw

pytestmark = pytest.mark.gpu

PRECS = MODES
FACE_EPS = {"fp64": 1e-6, "mixed": 1e-6, "fp32": 2e-5}
XI_TOL = {"fp64": 1e-11, "mixed": 1e-11, "fp32": 2e-5}


def smooth_field(X, scale=1.0):
    x, y = X[:, 0], X[:, 1]
    ux = scale * (1.0 + 0.4 * np.sin(2.9 * y + 0.3) * np.cos(1.7 * x))
    uy = scale * (0.35 * np.cos(2.3 * x - 0.2) * np.sin(1.1 * y + 0.5))
    if X.shape[1] == 3:
        z = X[:, 2]
        uz = scale * 0.3 * np.sin(1.9 * x + 2.1 * z)
        return [ux, uy, uz]
    return [ux, uy]


def spec_2d(dt=0.03, **kw):
    sp = cases.poiseuille_2d(nx=32, ny=12, **kw)
    sp.case.dt = dt
    sp.case.vel_tol = 1e-13
    sp.case.p_tol = 1e-12
    return sp


def spec_3d(dt=0.02, **kw):
    sp = cases.pipe_3d(ny=6, nz=6, nx=12, **kw)
    sp.case.dt = dt
    sp.case.vel_tol = 1e-13
    sp.case.p_tol = 1e-12
    return sp


def make_pair(sp, prec, **kw):
    """the library in mode `prec` (a MODES name, or a pfem2_precision value
    with fp32_stages in kw) and the oracle on the same spec"""
    if isinstance(prec, str):
        kw = dict(kw, **solver_kw(prec))
    else:
        kw = dict(kw, precision=prec)
    g = Solver(sp, **kw)
    o = O.Oracle(sp.mesh, sp.case, movement_steps=kw.get("movement_steps", sp.movement_steps),
                 max_per_part=kw.get("max_per_part", sp.max_per_part))
    return g, o


def set_vel(g, o, sp, fields, old=None):
    dim = sp.mesh.dim
    for d in range(dim):
        g.set_field(A.FIELD_VX + d, fields[d])
        o.set_field(A.FIELD_VX + d, fields[d])
        ov = old[d] if old is not None else np.zeros_like(fields[d])
        g.set_field(A.FIELD_OLD_VX + d, ov)
        o.set_field(A.FIELD_OLD_VX + d, ov)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("dim", [2, 3])
def test_seed(prec, dim):
    sp = spec_2d() if dim == 2 else spec_3d()
    g, o = make_pair(sp, prec)
    f = smooth_field(sp.mesh.vertices)
    set_vel(g, o, sp, f)
    q = (4, 4) if dim == 2 else (3, 3, 3)
    g.seed_particles(q, seed=7, jitter=0.1)
    o.seed_particles(q, seed=7, jitter=0.1)
    gc, gx, gu = g.particles()
    oc, ox, ou = o.particles()
    assert np.array_equal(gc, oc)
    tol = 1e-6 if prec == "fp32" else 1e-14
    assert np.abs(gx - ox).max() <= tol
    assert np.abs(gu - ou).max() <= tol * 4


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("dim", [2, 3])
def test_correct(prec, dim):
    sp = spec_2d() if dim == 2 else spec_3d()
    g, o = make_pair(sp, prec)
    X = sp.mesh.vertices
    f0 = smooth_field(X)
    set_vel(g, o, sp, f0)
    q = (4, 4) if dim == 2 else (3, 3, 3)
    g.seed_particles(q, seed=3, jitter=0.1)
    o.seed_particles(q, seed=3, jitter=0.1)
    f1 = smooth_field(X[:, ::-1] if dim == 2 else X[:, [2, 0, 1]], 0.7)
    set_vel(g, o, sp, f1, old=f0)
    g.correct_particles_velocities()
    o.correct_particles_velocities()
    gc, gx, gu = g.particles()
    oc, ox, ou = o.particles()
    assert np.array_equal(gc, oc)
    tol = 2e-6 if prec == "fp32" else 1e-13
    assert np.abs(gu - ou).max() <= tol


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("check", [False, True])
def test_move(prec, dim, check):
    """advection with point location (and check_cell_for_empty_parts)."""
    sp = spec_2d(dt=0.03) if dim == 2 else spec_3d(dt=0.015)
    g, o = make_pair(sp, prec)
    X = sp.mesh.vertices
    f = smooth_field(X)
    set_vel(g, o, sp, f)
    q = (4, 4) if dim == 2 else (3, 3, 3)
    g.seed_particles(q, seed=11, jitter=0.1)
    o.seed_particles(q, seed=11, jitter=0.1)
    for _ in range(3):
        if check:
            g.move_particles()
            o.move_particles()
        else:
            g.advect()
            o.advect()
    r = compare_particles(o.particles(), g.particles(), FACE_EPS[prec], XI_TOL[prec],
                          1e-5 if prec == "fp32" else 1e-12)
    gs, os_ = g.stats(), o.stats()
    # membership: exact in fp64 and mixed; with FP32 reference coordinates a
    # particle may change cell only within the band of FACE_EPS (the largest
    # face distance of a flipped particle measured here is reported)
    if prec != "fp32":
        assert r["flips"] == 0
    assert r["max_flip_dist"] <= FACE_EPS[prec]
    assert gs["deleted"] == os_["deleted"]
    if check:
        assert gs["removed"] == os_["removed"] and gs["reseeded"] == os_["reseeded"]
    assert gs["far"] == 0


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("dim", [2, 3])
def test_project(prec, dim):
    sp = spec_2d() if dim == 2 else spec_3d()
    g, o = make_pair(sp, prec)
    X = sp.mesh.vertices
    f = smooth_field(X)
    set_vel(g, o, sp, f)
    q = (4, 4) if dim == 2 else (3, 3, 3)
    g.seed_particles(q, seed=5, jitter=0.1)
    o.seed_particles(q, seed=5, jitter=0.1)
    g.distribute_particle_velocities_to_grid()
    o.distribute_particle_velocities_to_grid()
    tol = 3e-7 if prec == "fp32" else 1e-13
    for d in range(dim):
        assert rel_l2(g.field(A.FIELD_VX + d), o.field(A.FIELD_VX + d)) <= tol
    assert rel_l2(g.field(A.FIELD_NODE_WEIGHT), o.field(A.FIELD_NODE_WEIGHT)) <= tol


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("dim", [2, 3])
def test_fem_step(prec, dim):
    """prediction, pressure Poisson and correction solves from the same state."""
    sp = spec_2d(dt=0.005) if dim == 2 else spec_3d(dt=0.002)
    g, o = make_pair(sp, prec)
    X = sp.mesh.vertices
    f = smooth_field(X, 0.5)
    set_vel(g, o, sp, f)
    g.fem_step()
    o.fem_step(1)
    # both solve to absolute residuals of 1e-13 (velocity) / 1e-12
    # (pressure); fp32: FP32 assembly of the right-hand sides
    tol = {"fp64": 1e-8, "mixed": 1e-8, "fp32": 2e-5}[prec]
    for fld in [A.FIELD_PRED_VX + d for d in range(dim)] + [A.FIELD_P] + [A.FIELD_VX + d for d in range(dim)]:
        e = rel_l2(g.field(fld), o.field(fld))
        assert e <= tol, (fld, e)


@pytest.mark.parametrize("prec", PRECS)
def test_steps_2d(prec):
    """three whole time steps (correct, move, project, FEM) from seeding."""
    sp = spec_2d(dt=0.01)
    g, o = make_pair(sp, prec)
    g.seed_particles(sp.q, seed=0, jitter=0.1)
    o.seed_particles(sp.q, seed=0, jitter=0.1)
    for _ in range(3):
        g.step()
        o.step(1)
    tol = {"fp64": 1e-8, "mixed": 1e-7, "fp32": 1e-4}[prec]
    for fld in (A.FIELD_VX, A.FIELD_VY, A.FIELD_P):
        e = rel_l2(g.field(fld), o.field(fld))
        assert e <= tol, (fld, e)


def test_fused_step_equals_member_calls():
    """pfem2_step (fused kernels, CUDA graph) == the separate member calls, bit for bit."""
    sp = spec_2d(dt=0.01)
    a = Solver(sp, precision=A.PREC_FP64, use_graph=True)
    b = Solver(sp, precision=A.PREC_FP64, use_graph=False)
    for s in (a, b):
        s.seed_particles(sp.q, seed=0, jitter=0.1)
    for _ in range(3):
        a.step()
        b.correct_particles_velocities()
        b.move_particles()
        b.distribute_particle_velocities_to_grid()
        b.fem_step()
    for fld in (A.FIELD_VX, A.FIELD_VY, A.FIELD_P):
        assert np.array_equal(a.field(fld), b.field(fld))
    ca, xa, ua = a.particles()
    cb, xb, ub = b.particles()
    assert np.array_equal(ca, cb) and np.array_equal(xa, xb) and np.array_equal(ua, ub)


def test_batched_equals_single():
    """two instances in one batch give the instances' own results: bit for bit
    in the particle kernels and the Jacobi solves; the pressure solve of a
    batch uses per-instance coarse subdomains of its own size, so there the
    fields agree to the solver tolerance."""
    s1 = spec_2d(dt=0.01)
    s2 = cases.poiseuille_2d(nx=20, ny=8)
    s2.case.dt = 0.008
    s2.case.vel_tol = s2.case.p_tol = 1e-11
    both = Solver([s1, s2], precision=A.PREC_MIXED)
    one = Solver(s1, precision=A.PREC_MIXED)
    two = Solver(s2, precision=A.PREC_MIXED)
    for s in (both, one, two):
        s.seed_particles((4, 4), seed=0, jitter=0.1)
    for _ in range(2):
        for s in (both, one, two):
            s.step()
    for fld in (A.FIELD_VX, A.FIELD_P):
        assert rel_l2(both.field(fld, 0), one.field(fld, 0)) <= 1e-6
        assert rel_l2(both.field(fld, 1), two.field(fld, 0)) <= 1e-6
    assert both.n_particles(0) == one.n_particles(0) and both.n_particles(1) == two.n_particles(0)


def test_deterministic():
    sp = spec_2d(dt=0.01)
    outs = []
    for _ in range(2):
        s = Solver(sp, precision=A.PREC_MIXED)
        s.seed_particles(sp.q, seed=0, jitter=0.1)
        for _ in range(3):
            s.step()
        outs.append([s.field(f) for f in (A.FIELD_VX, A.FIELD_VY, A.FIELD_P)])
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("prec", PRECS)
def test_particles_only_step(prec):
    """the particle-kernel workload: correct -> move -> project on a frozen field"""
    sp = cases.stress_2d(n=24)
    g = Solver(sp, particles_only=True, **solver_kw(prec))
    o = O.Oracle(sp.mesh, sp.case, movement_steps=sp.movement_steps, max_per_part=sp.max_per_part)
    ux, uy = sp.meta["ux"], sp.meta["uy"]
    for f, v in ((A.FIELD_VX, ux), (A.FIELD_VY, uy), (A.FIELD_PRED_VX, ux), (A.FIELD_PRED_VY, uy)):
        g.set_field(f, v)
    o.set_field(A.FIELD_VX, ux)
    o.set_field(A.FIELD_VY, uy)
    g.seed_particles(sp.q, sp.seed, sp.jitter)
    o.seed_particles(sp.q, sp.seed, sp.jitter)
    for _ in range(3):
        g.step()
        o.correct_particles_velocities()
        o.move_particles()
        o.distribute_particle_velocities_to_grid()
        proj = [o.field(A.FIELD_VX), o.field(A.FIELD_VY)]
        o.set_field(A.FIELD_OLD_VX, proj[0])
        o.set_field(A.FIELD_OLD_VY, proj[1])
        o.set_field(A.FIELD_VX, ux)
        o.set_field(A.FIELD_VY, uy)
        oproj = proj
    gproj = [g.field(A.FIELD_OLD_VX), g.field(A.FIELD_OLD_VY)]
    tol = {"fp64": 1e-12, "mixed": 1e-12, "fp32": 1e-4}[prec]
    for d in range(2):
        assert rel_l2(gproj[d], oproj[d]) <= tol
    r = compare_particles(o.particles(), g.particles(), FACE_EPS[prec], XI_TOL[prec],
                          1e-4 if prec == "fp32" else 1e-12)
    if prec != "fp32":
        assert r["flips"] == 0


def test_ensemble_batch_matches_oracle():
    """a batch of four uneven channel instances (2k-6k cells, different
    Reynolds numbers and radii) in one context: every instance equals the
    oracle run of that instance alone (mixed path, solves to 1e-11 relative)"""
    specs = cases.ensemble(n=4, cells_lo=2000, cells_hi=6000)
    for sp in specs:
        sp.case.vel_tol = sp.case.p_tol = 0.0
        sp.case.vel_rtol = sp.case.p_rtol = 1e-11
    assert len({sp.mesh.n_cells for sp in specs}) == 4
    s = Solver(specs, precision=A.PREC_MIXED)
    s.seed_particles(specs[0].q, 2, 0.0)
    for _ in range(2):
        s.step()
    assert s.stats()["status"] == A.OK
    for i, sp in enumerate(specs):
        o = O.Oracle(sp.mesh, sp.case, movement_steps=sp.movement_steps, max_per_part=sp.max_per_part)
        o.seed_particles(specs[0].q, 2, 0.0)
        for _ in range(2):
            o.step(1)
        for fld in (A.FIELD_VX, A.FIELD_VY, A.FIELD_P):
            e = rel_l2(s.field(fld, i), o.field(fld))
            assert e <= 1e-7, (i, fld, e)
        assert s.n_particles(i) == o.n_particles()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_advect_split_equals_one_kernel(monkeypatch, prec):
    """the two-phase advection (the default: lean sub-steps, then each warp's
    queued particles that left their cell) equals the one-pass form bit for
    bit; both chosen here through PFEM2_ADVECT_SPLIT_MIN"""
    sp = spec_2d(dt=0.02)
    outs = []
    for split_min in ("0", str(1 << 40)):
        monkeypatch.setenv("PFEM2_ADVECT_SPLIT_MIN", split_min)
        s = Solver(sp, **solver_kw(prec))
        s.seed_particles(sp.q, seed=0, jitter=0.1)
        for _ in range(3):
            s.step()
        outs.append((s.particles(), [s.field(f) for f in (A.FIELD_VX, A.FIELD_P)], s.stats()["deleted"]))
        s.close()
    (pa, fa, da), (pb, fb, db) = outs
    for x, y in zip(pa, pb):
        assert np.array_equal(x, y)
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y)
    assert da == db


@pytest.mark.parametrize("prec", PRECS)
def test_vorticity(prec):
    """calculate_vorticity on the library's own fields after two steps
    against the oracle's restatement on the same fields (FP64 in both)"""
    sp = cases.channel_disk(h=0.05, dt=0.01)
    g = Solver(sp, **solver_kw(prec))
    g.seed_particles(sp.q, seed=0, jitter=0.1)
    for _ in range(2):
        g.step()
    w = g.calculate_vorticity()
    o = O.Oracle(sp.mesh, sp.case)
    o.set_field(A.FIELD_VX, g.field(A.FIELD_VX))
    o.set_field(A.FIELD_VY, g.field(A.FIELD_VY))
    assert rel_l2(w, o.calculate_vorticity()) <= 1e-12
    assert np.abs(w).max() > 1.0  # the disk sheds vorticity
    g.close()


def test_vorticity_rejects_3d():
    sp = spec_3d()
    g = Solver(sp, precision=A.PREC_FP64)
    with pytest.raises(Exception):
        g.calculate_vorticity()
    g.close()


@pytest.mark.parametrize("prec", PRECS)
def test_wall_pushback_steps(prec):
    """three whole steps of the disk channel with the wall push-back on the
    disk and the channel walls (zero_after_projection), against the oracle"""
    sp = cases.channel_disk(h=0.05, dt=0.01, zero_ids=(3, 4), wall_pushback=1)
    sp.case.vel_tol = 1e-13
    sp.case.p_tol = 1e-12
    g, o = make_pair(sp, prec)
    g.seed_particles(sp.q, seed=0, jitter=0.1)
    o.seed_particles(sp.q, seed=0, jitter=0.1)
    for _ in range(3):
        g.step()
        o.step(1)
    tol = {"fp64": 1e-8, "mixed": 1e-7, "fp32": 1e-4}[prec]
    for fld in (A.FIELD_VX, A.FIELD_VY, A.FIELD_P):
        e = rel_l2(g.field(fld), o.field(fld))
        assert e <= tol, (fld, e)
    # the push-back changed the particles next to the walls: without it
    # the run differs by more than the tolerance
    sp0 = cases.channel_disk(h=0.05, dt=0.01, zero_ids=(3, 4), wall_pushback=0)
    sp0.case.vel_tol, sp0.case.p_tol = 1e-13, 1e-12
    g0 = Solver(sp0, **solver_kw(prec))
    g0.seed_particles(sp0.q, seed=0, jitter=0.1)
    for _ in range(3):
        g0.step()
    assert rel_l2(g0.field(A.FIELD_VX), g.field(A.FIELD_VX)) > 10 * tol
    g.close()
    g0.close()
