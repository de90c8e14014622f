"""Known answers of the oracle's moving-mesh routines (CPU): the restatement
of problem_of_elasticity, reinterpolate_fields and transform_grid with the
particles' relocation (cylinderDyM/cylinderDyM.cc:926-976,
cylinderDyM/pfem2particle.cpp:1144-1261).
"""
import numpy as np

import oracle as O
from pfem2_b200 import _abi as A
from pfem2_b200 import cases


def test_elasticity_rigid_translation():
    """one boundary displaced by d and nothing else held: the elastic
    energy's minimiser is the rigid translation u = d everywhere"""
    sp = cases.poiseuille_2d(nx=12, ny=5)
    o = O.Oracle(sp.mesh, sp.case)
    it, res = o.problem_of_elasticity(1.0, 0.7, [], 0, [0.013, -0.021])
    assert it > 0 and res < 1e-9
    assert np.abs(o.field(A.FIELD_DISP_X) - 0.013).max() < 1e-12
    assert np.abs(o.field(A.FIELD_DISP_Y) + 0.021).max() < 1e-12


def test_elasticity_body_and_fixed_walls():
    """the disk displaced upward, the channel's boundaries held: the
    displacement is the body's on the disk, zero on the outer boundary, in
    between everywhere else"""
    sp = cases.channel_disk(h=0.05)
    o = O.Oracle(sp.mesh, sp.case)
    it, _ = o.problem_of_elasticity(1.0, 1.0, [1, 2, 4], 3, [0.0, 0.01])
    uy = o.field(A.FIELD_DISP_Y)
    m = sp.mesh
    disk = np.unique(np.concatenate([m.cells[c] for c, f in zip(*np.nonzero(m.face_bid == 3))]))
    assert it > 0
    assert uy.max() <= 0.01 + 1e-12 and uy.min() >= -1e-3
    assert np.isclose(uy[disk], 0.01).sum() >= len(disk) // 2


def test_reinterpolation_reproduces_linear_fields():
    """Q1 interpolation is exact for linear fields: every interior vertex
    takes f(x + u), boundary vertices keep f(x)"""
    sp = cases.channel_disk(h=0.05)
    o = O.Oracle(sp.mesh, sp.case)
    X = sp.mesh.vertices
    f = {A.FIELD_VX: lambda P: 1.0 + 0.3 * P[:, 0] - 0.2 * P[:, 1],
         A.FIELD_VY: lambda P: -0.5 + 0.1 * P[:, 0] + 0.4 * P[:, 1],
         A.FIELD_P: lambda P: 2.0 - 0.7 * P[:, 0]}
    for k, fn in f.items():
        o.set_field(k, fn(X))
    o.problem_of_elasticity(1.0, 1.0, [1, 2, 4], 3, [0.0, 0.01])
    U = np.stack([o.field(A.FIELD_DISP_X), o.field(A.FIELD_DISP_Y)], axis=1)
    o.reinterpolate_fields()
    m = sp.mesh
    bnd = np.zeros(m.n_vertices, bool)
    for c, fc in zip(*np.nonzero(m.face_bid >= 0)):
        for v in range(4):
            if ((v >> (fc // 2)) & 1) == fc % 2:
                bnd[m.cells[c, v]] = True
    moved = np.linalg.norm(U, axis=1) > 0
    assert (moved & ~bnd).sum() > 20
    for k, fn in f.items():
        got = o.field(k)
        assert np.abs(got[~bnd] - fn(X + U)[~bnd]).max() < 1e-12
        assert np.array_equal(got[bnd], fn(X)[bnd])


def test_transform_keeps_particle_positions():
    """after transform_grid every particle keeps its physical position and
    is found again in the moved mesh; only particles that the displaced
    disk now covers (outside the fluid) are deleted"""
    sp = cases.channel_disk(h=0.05)
    o = O.Oracle(sp.mesh, sp.case)
    o.seed_particles(sp.q, 0, 0.1)
    before = o.positions()
    n0 = o.n_particles()
    o.problem_of_elasticity(1.0, 1.0, [1, 2, 4], 3, [0.0, 0.004])
    U = np.stack([o.field(A.FIELD_DISP_X), o.field(A.FIELD_DISP_Y)], axis=1)
    o.transform_grid()
    assert np.abs(o.vertices() - (sp.mesh.vertices + U)).max() < 1e-15
    deleted = o.stats()["deleted"]
    assert o.n_particles() == n0 - deleted and deleted < n0 // 100
    cell, xi, _ = o.particles()
    after = o.positions()
    # every kept particle is one of the particles before, at the same place
    key = lambda P: np.round(P, 12)
    b = {tuple(p) for p in key(before)}
    assert all(tuple(p) in b for p in key(after))
    # and its new reference coordinates map back to it in the moved mesh
    for p in range(0, len(cell), 37):
        assert np.abs(o.map_to_real(int(cell[p]), xi[p]) - after[p]).max() < 1e-12
    # the deleted ones lie inside the displaced disk (centre (0.5, 0.504), r 0.1)
    kept = {tuple(q) for q in key(after)}
    gone = [p for p in key(before) if tuple(p) not in kept]
    r = np.linalg.norm(np.array(gone) - [0.5, 0.504], axis=1) if gone else np.zeros(0)
    assert np.all(r < 0.1 + 1e-9)
