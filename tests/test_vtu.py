"""VTK XML output (output_results): the written files decode back to the
mesh, the fields and the particles; the asynchronous writer produces one
file per snapshot and the .pvd collection."""
import base64
import xml.etree.ElementTree as ET
from types import SimpleNamespace

import numpy as np
import pytest

from pfem2_b200 import _abi as A
from pfem2_b200 import cases
from pfem2_b200 import meshes as M
from pfem2_b200 import vtu

_NP = {"Float64": np.float64, "Float32": np.float32, "Int32": np.int32, "Int64": np.int64, "UInt8": np.uint8}


def _decode(el):
    raw = base64.b64decode(el.text)
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    return np.frombuffer(raw[8:8 + n], _NP[el.get("type")])


def _read(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    pts = _decode(piece.find("Points/DataArray")).reshape(-1, 3)
    cells = {a.get("Name"): _decode(a) for a in piece.find("Cells")}
    pdata = {a.get("Name"): _decode(a) for a in piece.find("PointData")}
    return piece, pts, cells, pdata


@pytest.mark.parametrize("maker", [lambda: M.channel_disk_mesh(h=0.1), lambda: M.pipe_mesh(4, 4, 6)])
def test_vtu_decodes_to_mesh_and_fields(maker, tmp_path):
    m = maker()
    rng = np.random.default_rng(0)
    f = {"P": rng.standard_normal(m.n_vertices), "V": rng.standard_normal((m.n_vertices, 3))}
    p = tmp_path / "m.vtu"
    vtu.write_vtu(p, m, f)
    piece, pts, cells, pdata = _read(p)
    assert int(piece.get("NumberOfPoints")) == m.n_vertices and int(piece.get("NumberOfCells")) == m.n_cells
    assert np.array_equal(pts[:, :m.dim], m.vertices)
    order = [0, 1, 3, 2, 4, 5, 7, 6] if m.dim == 3 else [0, 1, 3, 2]
    assert np.array_equal(cells["connectivity"].reshape(m.n_cells, -1), m.cells[:, order])
    assert np.all(cells["types"] == (12 if m.dim == 3 else 9))
    assert np.array_equal(pdata["P"], f["P"]) and np.array_equal(pdata["V"].reshape(-1, 3), f["V"])


def test_particle_positions_follow_the_q1_map(tmp_path):
    m = M.rect_mesh(4, 2, 0.0, 4.0, 0.0, 1.0)
    rng = np.random.default_rng(1)
    cell = rng.integers(0, m.n_cells, 50)
    xi = rng.random((50, 2))
    x = vtu.particle_positions(m, cell, xi)
    lo = m.vertices[m.cells[cell, 0]]
    assert np.allclose(x, lo + xi * np.array([1.0, 0.5]))
    p = tmp_path / "p.vtu"
    vtu.write_particles_vtu(p, x, xi)
    _, pts, cells, pdata = _read(p)
    assert np.allclose(pts[:, :2], x) and np.array_equal(pdata["velocity"].reshape(-1, 2), xi)


def test_async_writer_with_a_solver_stand_in(tmp_path):
    sp = cases.poiseuille_2d(nx=4, ny=2)
    m = sp.mesh
    fake = SimpleNamespace(
        specs=[sp],
        field=lambda f, inst=0: np.full(m.n_vertices, float(f)),
        particles=lambda inst=0: (np.array([0, 1], np.int32), np.full((2, 2), 0.5), np.ones((2, 2))))
    w = vtu.AsyncWriter(fake, str(tmp_path), particles=True)
    for k in range(3):
        w.snapshot(k, 0.1 * k)
    w.close()
    for k in range(3):
        _, _, _, pdata = _read(tmp_path / f"solution-{k:06d}.vtu")
        assert np.all(pdata["Vx"] == A.FIELD_VX) and np.all(pdata["P"] == A.FIELD_P)
        assert (tmp_path / f"solution-{k:06d}-particles.vtu").exists()
    coll = ET.parse(tmp_path / "solution.pvd").getroot()
    assert [d.get("file") for d in coll.iter("DataSet")] == [f"solution-{k:06d}.vtu" for k in range(3)]


@pytest.mark.gpu
def test_async_writer_with_the_library(tmp_path):
    from pfem2_b200.solver import Solver

    sp = cases.channel_disk(h=0.05, dt=0.01)
    s = Solver(sp)
    s.seed_particles(sp.q, 0, 0.0)
    w = vtu.AsyncWriter(s, str(tmp_path), particles=True)
    for k in range(2):
        s.step()
        w.snapshot(k, (k + 1) * sp.case.dt)
    w.close()
    _, _, _, pdata = _read(tmp_path / "solution-000001.vtu")
    assert np.allclose(pdata["Vx"], s.field(A.FIELD_VX)) and np.allclose(pdata["P"], s.field(A.FIELD_P))
    _, pts, _, _ = _read(tmp_path / "solution-000001-particles.vtu")
    assert len(pts) == s.n_particles()
    s.close()
