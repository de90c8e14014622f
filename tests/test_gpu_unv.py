"""A mesh from a UNV file through the library: the reference's cylinder2D
case (cylinder2D/cylinder2D.cc:266-277 reads its mesh with GridIn::read_unv;
boundary groups 1 inlet, 2 outlet, 3 cylinder, 4 walls) on a synthetic
channel-with-cylinder mesh written to UNV by pfem2_b200/unv.py and read
back, run for three whole steps on the GPU against the FP64 oracle.
"""
import numpy as np
import pytest

import oracle as O
from pfem2_b200 import _abi as A
from pfem2_b200 import cases, meshes, unv
from pfem2_b200.solver import Solver
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
def test_unv_cylinder_case_matches_oracle(tmp_path, prec):
    src = meshes.channel_disk_mesh(h=0.05)
    path = tmp_path / "cylinder.unv"
    unv.write_unv(src, path)
    sp = cases.cylinder2d_unv(str(path), dt=0.01)
    assert sp.mesh.n_cells == src.n_cells
    assert sorted(np.unique(sp.mesh.face_bid[sp.mesh.face_bid >= 0]).tolist()) == [1, 2, 3, 4]
    sp.case.vel_tol = sp.case.p_tol = 0.0
    sp.case.vel_rtol = sp.case.p_rtol = 1e-11
    g = Solver(sp, precision=prec)
    o = O.Oracle(sp.mesh, sp.case, movement_steps=sp.movement_steps, max_per_part=sp.max_per_part)
    g.seed_particles(sp.q, 0, 0.1)
    o.seed_particles(sp.q, 0, 0.1)
    for _ in range(3):
        g.step()
        o.step(1)
    tol = 1e-8 if prec == A.PREC_FP64 else 1e-7
    for f in (A.FIELD_VX, A.FIELD_VY, A.FIELD_P):
        assert rel_l2(g.field(f), o.field(f)) <= tol, f
    gl, ol = g.calculate_loads(3), o.calculate_loads(3)
    assert np.all(np.isfinite(gl)) and gl[0] + gl[1] != 0.0
    assert np.allclose(gl, ol, rtol=1e-6, atol=1e-9)
    g.close()
