"""UNV (I-DEAS universal file) mesh reader, the reference's mesh input.

The reference's drivers read their meshes with deal.II's GridIn::read_unv
(cylinder2D/cylinder2D.cc:266-277, TurekBenchmarkCuda/TurekBenchmark.cc:273-276).
This module restates what that reader takes from a file written by Salome:

* dataset 2411: nodes (label, three coordinate systems/colour, then x y z);
* dataset 2412: elements (label, FE descriptor, two property tables, colour,
  node count; beam-type descriptors carry one more record), then node labels;
  cells are linear quads (descriptor 44) in 2D and linear bricks (115) in 3D,
  boundary faces are rods (11) in 2D and quads (44) in 3D;
* dataset 2467: permanent groups (number, ..., entity count; the name; then
  entity records of four integers, two per line). A group's name is its
  number: on a boundary element it becomes the boundary id of that face (on
  a cell it would be a material id, which the PFEM2 path does not use).

Cells are brought to deal.II's lexicographic vertex order with a positive
Jacobian, faces the reader does not name get boundary id 0 (deal.II's
default), interior faces -1, and the mesh is then ordered like the
programmatic meshes (pfem2_b200/meshes.py).
"""
import numpy as np

from pfem2_b200 import meshes as M

_BEAMS = {11, 21, 22, 23, 24}  # FE descriptors with a beam-orientation record


def _datasets(lines):
    """yields (dataset id, its lines) for every '-1' delimited block"""
    i, n = 0, len(lines)
    while i < n:
        if lines[i].strip() == "-1" and i + 1 < n and lines[i + 1].strip() not in ("", "-1"):
            did = int(lines[i + 1].split()[0])
            j = i + 2
            while j < n and lines[j].strip() != "-1":
                j += 1
            yield did, lines[i + 2:j]
            i = j + 1
        else:
            i += 1


def _floats(line):
    return [float(t.replace("D", "E").replace("d", "e")) for t in line.split()]


def read_unv(path, reorder=True):
    """Mesh of a UNV file (see the module docstring). Raises ValueError on
    content the PFEM2 path cannot use (mixed cell types, a non-numeric
    group name, a boundary element that matches no cell face)."""
    with open(path) as f:
        lines = f.read().splitlines()
    nodes, elems, groups = {}, {}, []
    for did, blk in _datasets(lines):
        if did == 2411:
            for k in range(0, len(blk) - 1, 2):
                nodes[int(blk[k].split()[0])] = _floats(blk[k + 1])[:3]
        elif did == 2412:
            k = 0
            while k < len(blk):
                rec = [int(t) for t in blk[k].split()]
                label, fe, nn = rec[0], rec[1], rec[5]
                k += 1
                if fe in _BEAMS:
                    k += 1
                conn = []
                while len(conn) < nn:
                    conn += [int(t) for t in blk[k].split()]
                    k += 1
                elems[label] = (fe, conn[:nn])
        elif did in (2467, 2477, 2452, 2435):
            k = 0
            while k < len(blk):
                head = [int(t) for t in blk[k].split()]
                name = blk[k + 1].strip()
                count = head[-1]
                k += 2
                ents = []
                while len(ents) < count:
                    v = [int(t) for t in blk[k].split()]
                    for a in range(0, len(v), 4):
                        ents.append((v[a], v[a + 1]))
                    k += 1
                groups.append((name, ents[:count]))
    dim = 3 if any(fe == 115 for fe, _ in elems.values()) else 2
    cell_fe, face_fe = (115, 44) if dim == 3 else (44, 11)
    labels = sorted(nodes)
    index = {lab: i for i, lab in enumerate(labels)}
    X = np.array([nodes[lab][:dim] for lab in labels], dtype=np.float64)
    cell_labels = sorted(lab for lab, (fe, _) in elems.items() if fe == cell_fe)
    if not cell_labels:
        raise ValueError("no quad (2D) or brick (3D) cells in the file")
    cells = []
    for lab in cell_labels:
        v = [index[n] for n in elems[lab][1]]
        cells.append(_lexicographic(X, v, dim))
    cells = np.array(cells, dtype=np.int64)
    # faces of every cell, keyed by their vertex set
    nf = 2 * dim
    fb = np.full((len(cells), nf), -1, dtype=np.int32)
    owner = {}
    for c, cv in enumerate(cells):
        for f in range(nf):
            key = tuple(sorted(_face_vertices(cv, f, dim)))
            owner.setdefault(key, []).append((c, f))
    for key, lst in owner.items():
        if len(lst) == 1:
            fb[lst[0]] = 0
    cell_set = set(cell_labels)
    for name, ents in groups:
        try:
            bid = int(name)
        except ValueError:
            raise ValueError(f"group name {name!r} is not a number (it is the boundary id)")
        for etype, tag in ents:
            if etype != 8 or tag in cell_set or tag not in elems:
                continue
            fe, conn = elems[tag]
            if fe != face_fe:
                continue
            key = tuple(sorted(index[n] for n in conn))
            if key not in owner:
                raise ValueError(f"boundary element {tag} matches no cell face")
            for c, f in owner[key]:
                fb[c, f] = bid
    return M._finish(X, cells.astype(np.int32), fb, reorder)


def _face_vertices(cv, f, dim):
    ax, side = f // 2, f % 2
    return [cv[v] for v in range(1 << dim) if ((v >> ax) & 1) == side]


def _lexicographic(X, v, dim):
    """UNV corner order (quad: counter-clockwise; brick: bottom quad, then
    top quad) to lexicographic order with a positive Jacobian"""
    if dim == 2:
        a, b, c, d = v
        area = 0.0
        ring = [a, b, c, d]
        for k in range(4):
            p, q = X[ring[k]], X[ring[(k + 1) % 4]]
            area += p[0] * q[1] - q[0] * p[1]
        if area < 0:
            a, b, c, d = a, d, c, b
        return [a, b, d, c]
    lex = [v[0], v[1], v[3], v[2], v[4], v[5], v[7], v[6]]
    P = X[lex]
    J = np.stack([P[1] - P[0], P[2] - P[0], P[4] - P[0]])
    if np.linalg.det(J) < 0:
        lex = lex[4:] + lex[:4]
    return lex


def repair_unv(src, dst):
    """What the reference's repairMesh tool does (repairMesh/repairMesh.cc)
    for deal.II import: drop every dataset before the nodes, keep the nodes,
    the cells and only those line (2D) / face (3D) elements that a group
    lists (internal boundaries and leftovers go), keep the groups. Returns
    (elements kept, elements dropped). read_unv gives the same mesh for the
    original and the repaired file."""
    with open(src) as f:
        lines = f.read().splitlines()
    out = []
    listed = set()
    blocks = list(_datasets(lines))
    for did, blk in blocks:
        if did in (2467, 2477, 2452, 2435):
            k = 0
            while k < len(blk):
                count = int(blk[k].split()[-1])
                k += 2
                n = 0
                while n < count:
                    v = [int(t) for t in blk[k].split()]
                    for a in range(0, len(v), 4):
                        if v[a] == 8:
                            listed.add(v[a + 1])
                    n += len(v) // 4
                    k += 1
    kept = dropped = 0
    bricks = any(did == 2412 and any(len(l.split()) == 6 and l.split()[1] == "115" for l in blk)
                 for did, blk in blocks)
    cell_fe = 115 if bricks else 44
    for did, blk in blocks:
        if did == 2411:
            out += ["    -1", "  2411"] + blk + ["    -1"]
        elif did == 2412:
            body = []
            k = 0
            while k < len(blk):
                rec = [int(t) for t in blk[k].split()]
                label, fe, nn = rec[0], rec[1], rec[5]
                n_lines = 1 + (1 if fe in _BEAMS else 0) + (nn + 7) // 8
                if fe == cell_fe or label in listed:
                    body += blk[k:k + n_lines]
                    kept += 1
                else:
                    dropped += 1
                k += n_lines
            out += ["    -1", "  2412"] + body + ["    -1"]
        elif did in (2467, 2477, 2452, 2435):
            out += ["    -1", f"  {did}"] + blk + ["    -1"]
    with open(dst, "w") as f:
        f.write("\n".join(out) + "\n")
    return kept, dropped


def write_unv(mesh, path, groups=None):
    """Writes a mesh as UNV (nodes, cells, boundary elements, groups): the
    inverse of read_unv for round-trip tests. groups: {boundary id: [(cell,
    face), ...]}; by default every named boundary face of the mesh."""
    dim = mesh.dim
    cells = np.asarray(mesh.cells)
    if groups is None:
        groups = {}
        for c, f in zip(*np.nonzero(mesh.face_bid >= 0)):
            groups.setdefault(int(mesh.face_bid[c, f]), []).append((int(c), int(f)))
    out = ["    -1", "  2411"]
    for i, x in enumerate(mesh.vertices):
        xyz = list(x) + [0.0] * (3 - dim)
        out.append(f"{i + 1:10d}{1:10d}{1:10d}{11:10d}")
        out.append("".join(f"{t:25.16E}" for t in xyz))
    out += ["    -1", "    -1", "  2412"]
    cell_fe, face_fe = (115, 44) if dim == 3 else (44, 11)
    unv_order = [0, 1, 3, 2, 4, 5, 7, 6] if dim == 3 else [0, 1, 3, 2]
    label = 0
    for cv in cells:
        label += 1
        out.append(f"{label:10d}{cell_fe:10d}{2:10d}{1:10d}{7:10d}{len(cv):10d}")
        out.append("".join(f"{int(cv[k]) + 1:10d}" for k in unv_order))
    face_labels = {}
    face_order = [0, 1, 3, 2] if dim == 3 else [0, 1]
    for bid in sorted(groups):
        for c, f in groups[bid]:
            label += 1
            fv = _face_vertices(cells[c], f, dim)
            nn = len(fv)
            out.append(f"{label:10d}{face_fe:10d}{2:10d}{1:10d}{7:10d}{nn:10d}")
            if face_fe in _BEAMS:
                out.append(f"{0:10d}{1:10d}{1:10d}")
            out.append("".join(f"{int(fv[k]) + 1:10d}" for k in face_order))
            face_labels.setdefault(bid, []).append(label)
    out += ["    -1", "    -1", "  2467"]
    for g, bid in enumerate(sorted(face_labels)):
        labs = face_labels[bid]
        out.append(f"{g + 1:10d}" + f"{0:10d}" * 6 + f"{len(labs):10d}")
        out.append(str(bid))
        for k in range(0, len(labs), 2):
            out.append("".join(f"{8:10d}{lab:10d}{0:10d}{0:10d}" for lab in labs[k:k + 2]))
    out.append("    -1")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
