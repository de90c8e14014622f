"""UNV mesh input (the reference's GridIn::read_unv path): round trips of
programmatic meshes through write_unv / read_unv, orientation repair, and
(when the reference tree is present) its own cylinder mesh."""
import os

import numpy as np
import pytest

from pfem2_b200 import meshes as M
from pfem2_b200 import unv


@pytest.mark.parametrize("maker", [
    lambda: M.rect_mesh(6, 3, 0.0, 4.0, 0.0, 1.0),
    lambda: M.channel_disk_mesh(h=0.1, radius=0.1),
    lambda: M.box_mesh(3, 2, 2),
    lambda: M.pipe_mesh(4, 4, 6),
])
def test_round_trip_is_exact(maker, tmp_path):
    m = maker()
    p = tmp_path / "m.unv"
    unv.write_unv(m, p)
    r = unv.read_unv(p)
    assert np.array_equal(r.vertices, m.vertices)
    assert np.array_equal(r.cells, m.cells)
    assert np.array_equal(r.face_bid, m.face_bid)


def test_clockwise_quads_are_reoriented(tmp_path):
    m = M.rect_mesh(3, 2, 0.0, 3.0, 0.0, 2.0, reorder=False)
    p = tmp_path / "cw.unv"
    unv.write_unv(m, p)
    # reverse the corner order of every quad (clockwise) in the file
    lines = p.read_text().splitlines()
    i = lines.index("  2412") + 1
    while lines[i].strip() != "-1":
        rec = lines[i].split()
        if rec[1] == "44":
            v = lines[i + 1].split()
            lines[i + 1] = "".join(f"{int(t):10d}" for t in v[::-1])
        i += 2 if rec[1] == "44" else 3
    p.write_text("\n".join(lines) + "\n")
    r = unv.read_unv(p, reorder=False)
    X = r.vertices
    for cv in r.cells:
        d1, d2 = X[cv[1]] - X[cv[0]], X[cv[2]] - X[cv[0]]
        assert d1[0] * d2[1] - d1[1] * d2[0] > 0
    # the same cells (as sets of corner coordinates) with the same boundary faces
    def key(mesh):
        out = []
        for c, cv in enumerate(mesh.cells):
            corners = tuple(sorted(map(tuple, np.round(mesh.vertices[cv], 12))))
            faces = []
            for f in range(4):
                ax, side = f // 2, f % 2
                fv = [cv[v] for v in range(4) if ((v >> ax) & 1) == side]
                faces.append((tuple(sorted(map(tuple, np.round(mesh.vertices[fv], 12)))), int(mesh.face_bid[c, f])))
            out.append((corners, tuple(sorted(faces))))
        return sorted(out)
    assert key(r) == key(m)


# the reference's own cylinder2D mesh, read where the reference tree is
# checked out (PFEM2_REFERENCE_DIR); skipped without it
REF_MESH = os.path.join(os.environ.get("PFEM2_REFERENCE_DIR", ""), "cylinder2D", "scaled3.unv")


@pytest.mark.skipif(not os.environ.get("PFEM2_REFERENCE_DIR") or not os.path.exists(REF_MESH),
                    reason="PFEM2_REFERENCE_DIR does not name the reference tree")
def test_reference_cylinder_mesh():
    """the reference's cylinder2D mesh: 7050 quads, boundary groups 1-4
    (inlet, outlet, cylinder, walls) with 75, 75, 60 and 170 faces"""
    m = unv.read_unv(REF_MESH)
    assert m.dim == 2 and m.n_cells == 7050
    ids, counts = np.unique(m.face_bid[m.face_bid >= 0], return_counts=True)
    assert dict(zip(ids.tolist(), counts.tolist())) == {1: 75, 2: 75, 3: 60, 4: 170}
    X = m.vertices
    for cv in m.cells:
        d1, d2 = X[cv[1]] - X[cv[0]], X[cv[2]] - X[cv[0]]
        assert d1[0] * d2[1] - d1[1] * d2[0] > 0


@pytest.mark.skipif(not os.environ.get("PFEM2_REFERENCE_DIR") or not os.path.exists(REF_MESH),
                    reason="PFEM2_REFERENCE_DIR does not name the reference tree")
def test_reference_cylinder_case_runs_in_the_oracle():
    """the reference's cylinder2D case on its own mesh: three oracle steps
    give finite fields, a drag on the cylinder and the inlet velocity kept"""
    import oracle as O
    from pfem2_b200 import _abi as A
    from pfem2_b200 import cases

    sp = cases.cylinder2d_unv(REF_MESH)
    o = O.Oracle(sp.mesh, sp.case)
    o.seed_particles(sp.q, 0, 0.0)
    for _ in range(3):
        o.step(1)
    vx, p = o.field(A.FIELD_VX), o.field(A.FIELD_P)
    assert np.all(np.isfinite(vx)) and np.all(np.isfinite(p))
    inlet = np.unique(sp.mesh.cells[np.nonzero(sp.mesh.face_bid == 1)[0]][:, [0, 2]].ravel())
    assert np.isclose(np.median(vx[inlet]), 1.0)
    loads = o.calculate_loads(3)
    assert np.all(np.isfinite(loads)) and loads[0] + loads[1] != 0.0


def test_repair_drops_preamble_and_unlisted_elements(tmp_path):
    """repairMesh: the datasets before the nodes and the line elements no
    group lists (an internal boundary here) go; the mesh read back is the same"""
    m = M.rect_mesh(4, 2, 0.0, 4.0, 0.0, 1.0)
    p = tmp_path / "m.unv"
    unv.write_unv(m, p)
    lines = p.read_text().splitlines()
    # a header dataset in front, and an unlisted internal line element
    head = ["    -1", "   164", "METER", "    -1", "    -1", "  2420", "         1", "SMESH_Auxiliary_Cartesian_System",
            "    -1"]
    i = lines.index("  2412") + 1
    extra = [f"{99999:10d}{11:10d}{2:10d}{1:10d}{7:10d}{2:10d}", f"{0:10d}{1:10d}{1:10d}",
             f"{int(m.cells[0, 1]) + 1:10d}{int(m.cells[0, 3]) + 1:10d}"]
    lines = head + lines[:i] + extra + lines[i:]
    p.write_text("\n".join(lines) + "\n")
    q = tmp_path / "repaired.unv"
    kept, dropped = unv.repair_unv(p, q)
    assert dropped == 1 and kept == m.n_cells + int((m.face_bid >= 0).sum())
    assert "2420" not in q.read_text() and "164" not in q.read_text().split("2411")[0]
    a, b = unv.read_unv(p), unv.read_unv(q)
    assert np.array_equal(a.cells, b.cells) and np.array_equal(a.face_bid, b.face_bid)
    assert np.array_equal(a.face_bid, m.face_bid)


@pytest.mark.skipif(not os.environ.get("PFEM2_REFERENCE_DIR") or not os.path.exists(REF_MESH),
                    reason="PFEM2_REFERENCE_DIR does not name the reference tree")
def test_repair_reference_mesh(tmp_path):
    q = tmp_path / "repaired.unv"
    kept, dropped = unv.repair_unv(REF_MESH, q)
    assert (kept, dropped) == (7050 + 380, 0)  # every line element of that file is in a group
    a, b = unv.read_unv(REF_MESH), unv.read_unv(q)
    assert np.array_equal(a.cells, b.cells) and np.array_equal(a.face_bid, b.face_bid)
