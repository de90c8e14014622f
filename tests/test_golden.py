"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py).

The fixtures hold the FP64 oracle's fields, per-cell particle counts and
loads after a few whole time steps of three small seeded workloads (2D
Poiseuille, a coarse channel with disk, a 3D pipe). The CPU test re-runs the
oracle against them (it must not drift); the GPU tests run the library
through the C ABI against them with the tolerances of the parity tests.
"""
import os

import numpy as np
import pytest

from pfem2_b200 import _abi as A
from tests.golden.make_golden import golden_cases, run_oracle
from tests.helpers import MODES, rel_l2, solver_kw

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = list(golden_cases().keys())


def _load(name):
    return dict(np.load(os.path.join(HERE, f"{name}.npz")))


def _fields(dim):
    return ["vx", "vy", "vz"][:dim] + ["p"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_golden(name):
    sp, steps = golden_cases()[name]
    ref = _load(name)
    assert int(ref["steps"]) == steps
    out = run_oracle(sp, steps)
    for f in _fields(sp.mesh.dim):
        assert rel_l2(out[f], ref[f]) <= 1e-12, f
    assert np.array_equal(out["cell_counts"], ref["cell_counts"])
    if ref["loads"].size:
        assert np.allclose(out["loads"], ref["loads"], rtol=1e-10, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", MODES)
@pytest.mark.parametrize("name", CASES)
def test_library_matches_golden(name, prec):
    _check_library(name, prec)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", MODES)
@pytest.mark.parametrize("name", CASES)
def test_library_matches_golden_wide_multigrid(name, prec, monkeypatch):
    """the pressure multigrid of one large system (from PFEM2_MG_WIDE_MIN rows
    on: two blocks per SM, a tile per block), forced on the small cases"""
    monkeypatch.setenv("PFEM2_MG_WIDE_MIN", "0")
    _check_library(name, prec)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", MODES)
@pytest.mark.parametrize("name", CASES)
def test_library_matches_golden_composite_restriction(name, prec, monkeypatch):
    """the restriction to level 2 through the composite R02 inside phase B
    (the form below PFEM2_MG_SPLIT_MIN rows; by default every system uses the
    separate phase b2 = Pt1^T b1)"""
    monkeypatch.setenv("PFEM2_MG_SPLIT_MIN", str(1 << 40))
    _check_library(name, prec)


def _check_library(name, prec):
    from pfem2_b200.solver import Solver

    sp, steps = golden_cases()[name]
    ref = _load(name)
    s = Solver(sp, **solver_kw(prec))
    s.seed_particles(sp.q, seed=sp.seed, jitter=sp.jitter)
    loads = []
    for _ in range(steps):
        s.step()
        if sp.case.load_patch_id >= 0:
            loads.append(s.calculate_loads(sp.case.load_patch_id))
    tol = {"fp64": 1e-8, "mixed": 1e-7, "fp32": 1e-4}[prec]
    for f in _fields(sp.mesh.dim):
        fld = {"vx": A.FIELD_VX, "vy": A.FIELD_VY, "vz": A.FIELD_VZ, "p": A.FIELD_P}[f]
        e = rel_l2(s.field(fld), ref[f])
        assert e <= tol, (f, e)
    # membership: the per-cell particle counts are exact in fp64 and mixed
    # (FP64 coordinates); with FP32 coordinates a particle within rounding of
    # a face may sit in the neighbour cell
    counts = np.bincount(s.particles()[0], minlength=sp.mesh.n_cells)
    if prec == "fp32":
        assert abs(int(counts.sum()) - int(ref["cell_counts"].sum())) <= max(2, ref["cell_counts"].sum() // 1000)
        assert np.mean(counts != ref["cell_counts"]) <= 0.005
    else:
        assert np.array_equal(counts, ref["cell_counts"])
    if ref["loads"].size:
        got = np.array(loads).reshape(-1, 5)
        ltol = {"fp64": 1e-6, "mixed": 1e-6, "fp32": 1e-2}[prec]
        scale = np.abs(ref["loads"]).max()
        assert np.abs(got - ref["loads"]).max() <= ltol * scale
    s.close()
