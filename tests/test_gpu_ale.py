"""The moving-mesh step (cylinderDyM) through the C ABI against the FP64
oracle: the pseudo-solid elasticity solve for the mesh displacement, the
reinterpolation of the fields, the grid transformation with the particles'
relocation and check_empty_cells, and whole time steps of the reference's
moving-mesh loop (cylinderDyM/cylinderDyM.cc:1146-1160) with a prescribed
body motion in place of its motion ODE.
"""
import numpy as np
import pytest

import oracle as O
from pfem2_b200 import _abi as A
from pfem2_b200 import cases
from pfem2_b200.solver import Pfem2Error, Solver
from tests.helpers import compare_particles, rel_l2, solver_kw

pytestmark = pytest.mark.gpu

LAME = (1.0, 1.0)
FIXED, BODY = (1, 2, 4), 3


def spec(dt=0.01):
    sp = cases.channel_disk(h=0.05, dt=dt)
    sp.case.vel_tol = sp.case.p_tol = 0.0
    sp.case.vel_rtol = sp.case.p_rtol = 1e-11
    return sp


def pair(sp, mode):
    g = Solver(sp, moving_mesh=True, **solver_kw(mode))
    o = O.Oracle(sp.mesh, sp.case, movement_steps=sp.movement_steps, max_per_part=sp.max_per_part)
    return g, o


def smooth(X):
    return [1.0 + 0.3 * np.sin(3.0 * X[:, 1]), 0.2 * np.cos(2.0 * X[:, 0]), 1.0 - 0.5 * X[:, 0]]


def test_elasticity_matches_oracle():
    sp = spec()
    g, o = pair(sp, "fp64")
    it, res = g.problem_of_elasticity(*LAME, FIXED, BODY, [0.003, 0.01], rtol=1e-12)
    oit, ores = o.problem_of_elasticity(*LAME, FIXED, BODY, [0.003, 0.01], rtol=1e-12)
    assert it > 10 and oit > 10
    for f in (A.FIELD_DISP_X, A.FIELD_DISP_Y):
        assert rel_l2(g.field(f), o.field(f)) <= 1e-10
    assert np.abs(g.field(A.FIELD_DISP_Y)).max() == pytest.approx(0.01, rel=1e-12)
    g.close()


def test_elasticity_requires_moving_context():
    sp = spec()
    g = Solver(sp, precision=A.PREC_FP64)
    with pytest.raises(Pfem2Error) as e:
        g.problem_of_elasticity(*LAME, FIXED, BODY, [0.0, 0.01])
    assert e.value.status == A.BAD_STATE
    g.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_move_mesh_matches_oracle(mode):
    """one mesh move of a seeded state: reinterpolated fields, moved
    vertices, relocated particles (membership exact, deletions equal)"""
    sp = spec()
    g, o = pair(sp, mode)
    X = sp.mesh.vertices
    for k, v in zip((A.FIELD_VX, A.FIELD_VY, A.FIELD_P), smooth(X)):
        g.set_field(k, v)
        o.set_field(k, v)
    g.seed_particles(sp.q, 0, 0.1)
    o.seed_particles(sp.q, 0, 0.1)
    g.problem_of_elasticity(*LAME, FIXED, BODY, [0.0, 0.004], rtol=1e-12)
    o.problem_of_elasticity(*LAME, FIXED, BODY, [0.0, 0.004], rtol=1e-12)
    g.move_mesh()
    o.move_mesh()
    assert np.abs(g.vertices() - o.vertices()).max() < 1e-12
    for k in (A.FIELD_VX, A.FIELD_VY, A.FIELD_P):
        assert rel_l2(g.field(k), o.field(k)) <= 1e-10, k
    r = compare_particles(o.particles(), g.particles(), 1e-6, 1e-9, 1e-12)
    assert r["flips"] == 0
    gs, os_ = g.stats(), o.stats()
    assert gs["deleted"] == os_["deleted"] > 0
    assert gs["reseeded"] == os_["reseeded"] and gs["removed"] == os_["removed"]
    g.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_moving_mesh_steps(mode):
    """three steps of the reference's moving-mesh loop: step, loads, the
    body's displacement (prescribed), elasticity, mesh move"""
    sp = spec(dt=0.005)
    g, o = pair(sp, mode)
    g.seed_particles(sp.q, 0, 0.1)
    o.seed_particles(sp.q, 0, 0.1)
    loads = []
    for n in range(3):
        g.step()
        o.step(1)
        loads.append((g.calculate_loads(BODY), o.calculate_loads(BODY)))
        d = [0.0, 0.003 * np.sin(0.7 * (n + 1))]
        g.problem_of_elasticity(*LAME, FIXED, BODY, d, rtol=1e-12)
        o.problem_of_elasticity(*LAME, FIXED, BODY, d, rtol=1e-12)
        g.move_mesh()
        o.move_mesh()
    tol = 1e-8 if mode == "fp64" else 1e-7
    assert np.abs(g.vertices() - o.vertices()).max() < 1e-12
    for k in (A.FIELD_VX, A.FIELD_VY, A.FIELD_P):
        assert rel_l2(g.field(k), o.field(k)) <= tol, k
    for gl, ol in loads:
        assert np.allclose(gl, ol, rtol=1e-6, atol=1e-8), (gl, ol)
    assert g.n_particles() == o.n_particles()
    g.close()
