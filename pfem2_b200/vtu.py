"""VTK XML output of fields and particles (the reference's output_results,
TurekBenchmarkCuda/TurekBenchmark.cc:802-928, writes VTU/PVTU with deal.II's
DataOut; here the same data from the library's host copies).

* write_vtu: the mesh (Q1 quads / hexes) with nodal fields as point data;
* write_particles_vtu: particle positions as vertices with their velocity;
* write_pvd: a time-series collection of such files;
* AsyncWriter: takes host copies of the fields after a step and writes the
  files on a background thread, so the encoding and the file I/O overlap the
  next steps on the GPU.

Arrays are written inline as base64 binary with a UInt64 length header
(ParaView and VTK read it).
"""
import base64
import os
import queue
import threading

import numpy as np

_VTK_QUAD, _VTK_HEX, _VTK_VERTEX = 9, 12, 1
_TYPES = {np.dtype(np.float64): "Float64", np.dtype(np.float32): "Float32", np.dtype(np.int32): "Int32",
          np.dtype(np.int64): "Int64", np.dtype(np.uint8): "UInt8"}


def _array(name, a, ncomp=1):
    a = np.ascontiguousarray(a)
    raw = a.tobytes()
    data = base64.b64encode(np.uint64(len(raw)).tobytes() + raw).decode("ascii")
    nm = f' Name="{name}"' if name else ""
    return (f'<DataArray type="{_TYPES[a.dtype]}"{nm} NumberOfComponents="{ncomp}" format="binary">'
            f"{data}</DataArray>")


def _points3(x):
    x = np.asarray(x, dtype=np.float64)
    if x.shape[1] == 2:
        x = np.hstack([x, np.zeros((len(x), 1))])
    return x


def _write(path, npts, ncells, points, conn, offsets, types, point_data):
    parts = ['<?xml version="1.0"?>',
             '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
             "<UnstructuredGrid>", f'<Piece NumberOfPoints="{npts}" NumberOfCells="{ncells}">',
             "<Points>", _array(None, points, 3), "</Points>",
             "<Cells>", _array("connectivity", conn), _array("offsets", offsets), _array("types", types), "</Cells>",
             "<PointData>"]
    for name, a in point_data.items():
        a = np.asarray(a)
        parts.append(_array(name, a, 1 if a.ndim == 1 else a.shape[1]))
    parts += ["</PointData>", "</Piece>", "</UnstructuredGrid>", "</VTKFile>"]
    tmp = f"{path}.tmp"
    with open(tmp, "w") as f:
        f.write("\n".join(parts) + "\n")
    os.replace(tmp, path)


def write_vtu(path, mesh, point_data):
    """mesh: pfem2_b200.meshes.Mesh; point_data: {name: [nv] or [nv, k]}"""
    dim = mesh.dim
    order = [0, 1, 3, 2, 4, 5, 7, 6] if dim == 3 else [0, 1, 3, 2]
    nvc = len(order)
    conn = np.asarray(mesh.cells, dtype=np.int64)[:, order].ravel()
    offsets = np.arange(1, mesh.n_cells + 1, dtype=np.int64) * nvc
    types = np.full(mesh.n_cells, _VTK_HEX if dim == 3 else _VTK_QUAD, dtype=np.uint8)
    _write(path, mesh.n_vertices, mesh.n_cells, _points3(mesh.vertices), conn, offsets, types, point_data)


def particle_positions(mesh, cell, xi):
    """x = sum_v N_v(xi) X_v of every particle (Q1 map, lexicographic corners)"""
    dim = mesh.dim
    xi = np.asarray(xi, dtype=np.float64)
    X = mesh.vertices[np.asarray(mesh.cells)[cell]]  # [np, 2^dim, dim]
    N = np.ones((len(cell), 1 << dim))
    for v in range(1 << dim):
        for d in range(dim):
            N[:, v] *= xi[:, d] if (v >> d) & 1 else 1.0 - xi[:, d]
    return np.einsum("pv,pvd->pd", N, X)


def write_particles_vtu(path, positions, velocity):
    n = len(positions)
    _write(path, n, n, _points3(positions), np.arange(n, dtype=np.int64), np.arange(1, n + 1, dtype=np.int64),
           np.full(n, _VTK_VERTEX, dtype=np.uint8), {"velocity": np.asarray(velocity, dtype=np.float64)})


def write_pvd(path, entries):
    """entries: [(time, file name relative to path's directory)]"""
    lines = ['<?xml version="1.0"?>', '<VTKFile type="Collection" version="1.0">', "<Collection>"]
    lines += [f'<DataSet timestep="{t!r}" file="{f}"/>' for t, f in entries]
    lines += ["</Collection>", "</VTKFile>"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


class AsyncWriter:
    """Writes field (and optionally particle) snapshots of a Solver on a
    background thread: snapshot() copies the data to the host (the only part
    on the caller's thread) and queues the encoding and the file I/O."""

    def __init__(self, solver, directory, prefix="solution", instance=0, particles=False):
        self.s, self.dir, self.prefix, self.inst, self.particles = solver, directory, prefix, instance, particles
        self.mesh = solver.specs[instance].mesh
        self.entries = []
        self.q = queue.Queue()
        self.err = None
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def snapshot(self, step, time):
        from pfem2_b200 import _abi as A

        dim = self.mesh.dim
        names = ["Vx", "Vy", "Vz"][:dim] + ["P"]
        fids = [A.FIELD_VX, A.FIELD_VY, A.FIELD_VZ][:dim] + [A.FIELD_P]
        data = {n: self.s.field(f, self.inst) for n, f in zip(names, fids)}
        parts = self.s.particles(self.inst) if self.particles else None
        name = f"{self.prefix}-{step:06d}.vtu"
        self.entries.append((time, name))
        self.q.put((name, data, parts))

    def _run(self):
        while True:
            job = self.q.get()
            if job is None:
                return
            try:
                name, data, parts = job
                write_vtu(os.path.join(self.dir, name), self.mesh, data)
                if parts is not None:
                    cell, xi, u = parts
                    write_particles_vtu(os.path.join(self.dir, name.replace(".vtu", "-particles.vtu")),
                                        particle_positions(self.mesh, cell, xi), u)
            except Exception as e:  # reported by close()
                self.err = e

    def close(self):
        """waits for the queued files, writes the .pvd collection"""
        self.q.put(None)
        self.t.join()
        if self.err is not None:
            raise self.err
        write_pvd(os.path.join(self.dir, f"{self.prefix}.pvd"), self.entries)
