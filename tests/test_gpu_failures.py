"""Failure paths of the library, made to fire on purpose in forms that
leave the GPU usable: statuses the host reads, never a device fault.

- a Krylov solve that runs out of iterations: PFEM2_NOT_CONVERGED (the
  reference only prints "failed to converge", TurekBenchmarkCuda/TurekBenchmark.cc:742-744);
- particle, per-cell and far-mover capacities too small: PFEM2_PARTICLE_OVERFLOW;
- non-finite host input: PFEM2_INVALID_ARG before anything reaches the device;
- bounded device-side waits (the persistent solver's phase waits, the
  rebin's look-back) given no patience through PFEM2_SPIN_LIMIT: the kernel
  gives up, the call returns PFEM2_TIMEOUT, the context then refuses to step
  (PFEM2_BAD_STATE), and a fresh context on the same GPU works.
"""
import numpy as np
import pytest

from pfem2_b200 import _abi as A
from pfem2_b200 import cases
from pfem2_b200.solver import Pfem2Error, Solver
from tests.test_gpu_parity import smooth_field, spec_2d

pytestmark = pytest.mark.gpu


def status_of(fn, *args):
    try:
        fn(*args)
    except Pfem2Error as e:
        return e.status
    return A.OK


def with_velocity(g, sp, scale=0.5):
    for d, v in enumerate(smooth_field(sp.mesh.vertices, scale)):
        g.set_field(A.FIELD_VX + d, v)
        g.set_field(A.FIELD_OLD_VX + d, np.zeros_like(v))


@pytest.mark.parametrize("kind", [A.SOLVER_CG, A.SOLVER_BICGSTAB])
def test_not_converged(kind):
    sp = spec_2d(dt=0.005)
    sp.case.max_iter = 1
    sp.case.vel_solver = sp.case.p_solver = kind
    g = Solver(sp, precision=A.PREC_FP64)
    with_velocity(g, sp)
    assert status_of(g.fem_step) == A.NOT_CONVERGED
    assert g.stats(check=False)["status"] == A.NOT_CONVERGED
    g.close()


def test_seed_capacity_overflow():
    sp = spec_2d()
    g = Solver(sp, precision=A.PREC_MIXED, capacity_factor=1e-9)
    assert status_of(g.seed_particles, sp.q, 0, 0.1) == A.PARTICLE_OVERFLOW
    g.close()


def test_per_cell_capacity_overflow():
    """16 particles per cell with room for 8 incoming ones per cell"""
    sp = spec_2d()
    g = Solver(sp, precision=A.PREC_MIXED, per_cell_max=8)
    with_velocity(g, sp)
    g.seed_particles((4, 4), 0, 0.1)
    assert status_of(g.move_particles) == A.PARTICLE_OVERFLOW
    g.close()


def test_far_mover_overflow():
    """a uniform flow of 2.4 cells per step: particles leave the 1-ring of
    their cell, more of them than a far-mover capacity of 1"""
    sp = spec_2d(dt=0.3)
    g = Solver(sp, precision=A.PREC_MIXED, far_capacity=1)
    nv = sp.mesh.n_vertices
    g.set_field(A.FIELD_VX, np.ones(nv))
    g.set_field(A.FIELD_VY, np.zeros(nv))
    g.seed_particles((4, 4), 0, 0.1)
    assert status_of(g.move_particles) == A.PARTICLE_OVERFLOW
    g.close()


def test_non_finite_input_rejected():
    sp = spec_2d()
    g = Solver(sp, precision=A.PREC_FP64)
    v = np.zeros(sp.mesh.n_vertices)
    v[3] = np.nan
    assert status_of(g.set_field, A.FIELD_VX, v) == A.INVALID_ARG
    v[3] = np.inf
    assert status_of(g.set_field, A.FIELD_P, v) == A.INVALID_ARG
    g.seed_particles((2, 2), 0, 0.0)
    cell, xi, u = g.particles()
    xi[5, 0] = np.nan
    assert status_of(g.set_particles, [(cell, xi, u)]) == A.INVALID_ARG
    g.close()


def fresh_context_steps():
    sp = spec_2d(dt=0.01)
    g = Solver(sp, precision=A.PREC_MIXED)
    g.seed_particles(sp.q, 0, 0.1)
    g.step()
    assert g.stats()["status"] == A.OK
    g.close()


def test_solver_wait_timeout(monkeypatch):
    """the persistent solver's waits give up at once: PFEM2_TIMEOUT, then
    PFEM2_BAD_STATE for stepping calls; another context runs normally"""
    monkeypatch.setenv("PFEM2_SPIN_LIMIT", "0")
    sp = cases.channel_disk(h=0.02, dt=0.002)
    g = Solver(sp, precision=A.PREC_MIXED)
    monkeypatch.delenv("PFEM2_SPIN_LIMIT")
    with_velocity(g, sp)
    assert status_of(g.fem_step) == A.TIMEOUT
    assert status_of(g.step) == A.BAD_STATE
    assert status_of(g.fem_step) == A.BAD_STATE
    g.close()
    fresh_context_steps()


def test_rebin_lookback_timeout(monkeypatch):
    """the rebin's look-back over 512 tiles gives up at once: PFEM2_TIMEOUT"""
    monkeypatch.setenv("PFEM2_SPIN_LIMIT", "0")
    sp = cases.stress_2d(n=64)
    g = Solver(sp, precision=A.PREC_MIXED, particles_only=True)
    monkeypatch.delenv("PFEM2_SPIN_LIMIT")
    ux, uy = sp.meta["ux"], sp.meta["uy"]
    for f, v in ((A.FIELD_VX, ux), (A.FIELD_VY, uy), (A.FIELD_PRED_VX, ux), (A.FIELD_PRED_VY, uy)):
        g.set_field(f, v)
    g.seed_particles(sp.q, sp.seed, sp.jitter)
    assert status_of(g.move_particles) == A.TIMEOUT
    assert status_of(g.move_particles) == A.BAD_STATE
    g.close()
    fresh_context_steps()
