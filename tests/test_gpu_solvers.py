"""Krylov solver kinds and stopping rules of the library (through the C ABI)
against the FP64 oracle.

The reference solves velocity with BiCGStab + Jacobi and pressure with
BiCGStab + SSOR (cylinder2D/cylinder2D.cc:736-780); the library offers CG
and BiCGStab for every system (pfem2_case.vel_solver / p_solver). Systems
solved to the same tight tolerance by different methods agree to that
tolerance; the relative rule stops at max(tol, rtol |b|).
"""
import numpy as np
import pytest

from pfem2_b200 import _abi as A
from pfem2_b200.solver import Pfem2Error, Solver
from tests.helpers import rel_l2
from tests.test_gpu_parity import make_pair, set_vel, smooth_field, spec_2d, spec_3d

pytestmark = pytest.mark.gpu

# mixed contexts here run only the inner Krylov iterations in FP32, so that
# the solver alone separates them from the FP64 oracle
KRYLOV_ONLY = A.FP32_KRYLOV


def fields_of(dim):
    return [A.FIELD_PRED_VX + d for d in range(dim)] + [A.FIELD_P] + [A.FIELD_VX + d for d in range(dim)]


def solve_once(sp, prec, **kw):
    g, o = make_pair(sp, prec, **kw)
    f = smooth_field(sp.mesh.vertices, 0.5)
    set_vel(g, o, sp, f)
    return g, o


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
@pytest.mark.parametrize("dim", [2, 3])
def test_bicgstab_fem_step(prec, dim):
    """fem_step with BiCGStab for every system (pressure with the Jacobi
    preconditioner) against the oracle's BiCGStab (solve_bicgstab)"""
    sp = spec_2d(dt=0.005) if dim == 2 else spec_3d(dt=0.002)
    sp.case.vel_solver = sp.case.p_solver = A.SOLVER_BICGSTAB
    g, o = solve_once(sp, prec, fp32_stages=KRYLOV_ONLY)
    g.fem_step()
    o.fem_step(0)
    st = g.stats()
    assert st["iters"][3] > 0 and st["iters"][0] > 0
    for fld in fields_of(dim):
        e = rel_l2(g.field(fld), o.field(fld))
        assert e <= 1e-8, (fld, e)
    g.close()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_bicgstab_equals_cg(prec):
    """the same state solved by CG (multigrid pressure) and by BiCGStab
    (Jacobi pressure): the fields agree to the solvers' tolerance"""
    out = []
    for kind in (A.SOLVER_CG, A.SOLVER_BICGSTAB):
        sp = spec_2d(dt=0.005)
        sp.case.vel_solver = sp.case.p_solver = kind
        g = Solver(sp, precision=prec, fp32_stages=KRYLOV_ONLY)
        for d, v in enumerate(smooth_field(sp.mesh.vertices, 0.5)):
            g.set_field(A.FIELD_VX + d, v)
            g.set_field(A.FIELD_OLD_VX + d, np.zeros_like(v))
        g.fem_step()
        out.append([g.field(f) for f in fields_of(2)])
        g.close()
    for a, b in zip(*out):
        assert rel_l2(a, b) <= 1e-8


@pytest.mark.parametrize("kind", [A.SOLVER_CG, A.SOLVER_BICGSTAB])
def test_relative_tolerance(kind):
    """tol = 0 with rtol: the solves stop at rtol |b| (an absolute 0 alone
    would never be reached) and agree with the oracle under the same rule"""
    sp = spec_2d(dt=0.005)
    sp.case.vel_tol = sp.case.p_tol = 0.0
    sp.case.vel_rtol = sp.case.p_rtol = 1e-11
    sp.case.vel_solver = sp.case.p_solver = kind
    g, o = solve_once(sp, A.PREC_FP64)
    g.fem_step()
    o.fem_step(0 if kind == A.SOLVER_BICGSTAB else 1)
    st = g.stats()
    assert st["status"] == A.OK
    assert 0.0 < st["residual"][3]
    for fld in fields_of(2):
        assert rel_l2(g.field(fld), o.field(fld)) <= 1e-8
    g.close()


def test_mixed_solver_kinds_rejected():
    """every instance of a context names the same solver kinds"""
    a, b = spec_2d(), spec_2d()
    b.case.vel_solver = A.SOLVER_BICGSTAB if a.case.vel_solver == A.SOLVER_CG else A.SOLVER_CG
    with pytest.raises(Pfem2Error) as e:
        Solver([a, b], precision=A.PREC_FP64)
    assert e.value.status == A.INVALID_ARG
