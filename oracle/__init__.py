"""ctypes wrapper of the FP64 CPU oracle (oracle/pfem2_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker. The product library never
loads it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from pfem2_b200 import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_bp = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    lib.or_create.restype = vp
    lib.or_create.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _ip, _ip, C.POINTER(A.Case), C.c_int, C.c_int]
    lib.or_destroy.argtypes = [vp]
    lib.or_set_threads.argtypes = [vp, C.c_int]
    lib.or_seed.argtypes = [vp, _up, C.c_uint64, C.c_double]
    lib.or_uniform.restype = C.c_double
    lib.or_uniform.argtypes = [C.c_uint64, C.c_uint64, C.c_int]
    for fn in ("or_correct", "or_advect", "or_check_empty", "or_move", "or_project", "or_assemble_matrices"):
        getattr(lib, fn).argtypes = [vp]
    lib.or_fem_step.argtypes = [vp, C.c_int]
    lib.or_fem_step.restype = C.c_int
    lib.or_step.argtypes = [vp, C.c_int]
    lib.or_step.restype = C.c_int
    lib.or_loads.argtypes = [vp, C.c_int, _dp]
    lib.or_vorticity.argtypes = [vp]
    lib.or_vorticity.restype = C.c_int
    lib.or_n_particles.argtypes = [vp]
    lib.or_n_particles.restype = C.c_int
    lib.or_nnz.argtypes = [vp]
    lib.or_nnz.restype = C.c_int
    lib.or_get_particles.argtypes = [vp, _ip, _dp, _dp]
    lib.or_get_positions.argtypes = [vp, _dp]
    lib.or_set_particles.argtypes = [vp, C.c_int, _ip, _dp, _dp, C.c_void_p]
    lib.or_get_field.argtypes = [vp, C.c_int, _dp]
    lib.or_set_field.argtypes = [vp, C.c_int, _dp]
    lib.or_get_stats.argtypes = [vp, _ip, _dp]
    lib.or_get_matrix.argtypes = [vp, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.or_get_matrix.restype = C.c_int
    lib.or_shape_values.argtypes = [C.c_int, _dp, _dp]
    lib.or_map_to_unit.argtypes = [vp, C.c_int, _dp, _dp]
    lib.or_map_to_unit.restype = C.c_int
    lib.or_map_to_real.argtypes = [vp, C.c_int, _dp, _dp]
    lib.or_measure.argtypes = [vp]
    lib.or_measure.restype = C.c_double
    lib.or_boundary_measure.argtypes = [vp, C.c_int, _dp]
    lib.or_boundary_measure.restype = C.c_double
    lib.or_rhs.argtypes = [vp, C.c_int, _dp]
    lib.or_get_dirichlet.argtypes = [vp, C.c_int, _bp, _dp]
    lib.or_elasticity.argtypes = [vp, C.c_double, C.c_double, C.c_uint, C.c_int, _dp, C.c_double, C.c_double,
                                  C.c_int, C.POINTER(C.c_double)]
    lib.or_elasticity.restype = C.c_int
    lib.or_reinterpolate.argtypes = [vp]
    lib.or_transform_grid.argtypes = [vp]
    lib.or_get_vertices.argtypes = [vp, _dp]
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _load()
    return _LIB


def uniform(seed, ordinal, axis):
    return lib().or_uniform(seed, ordinal, axis)


class Oracle:
    """FP64 CPU model of one flow instance, with the pfem2Solver member names."""

    def __init__(self, mesh, case, movement_steps=3, max_per_part=3, threads=1):
        self.L = lib()
        self.dim = mesh.dim
        self.mesh = mesh
        self.case = case
        self.nv = mesh.n_vertices
        self._X = np.ascontiguousarray(mesh.vertices, dtype=np.float64).reshape(-1)
        self._cv = np.ascontiguousarray(mesh.cells, dtype=np.int32).reshape(-1)
        self._fb = np.ascontiguousarray(mesh.face_bid, dtype=np.int32).reshape(-1)
        self.h = self.L.or_create(self.dim, mesh.n_vertices, mesh.n_cells, self._X, self._cv, self._fb,
                                  C.byref(case), movement_steps, max_per_part)
        self.L.or_set_threads(self.h, threads)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_destroy(self.h)
            self.h = None

    # pfem2Solver members
    def seed_particles(self, q, seed=0, jitter=0.0):
        qq = np.array(list(q) + [1] * (3 - len(q)), dtype=np.uint32)
        self.L.or_seed(self.h, qq, seed, jitter)

    def correct_particles_velocities(self):
        self.L.or_correct(self.h)

    def move_particles(self):
        self.L.or_move(self.h)

    def advect(self):
        self.L.or_advect(self.h)

    def check_empty(self):
        self.L.or_check_empty(self.h)

    def distribute_particle_velocities_to_grid(self):
        self.L.or_project(self.h)

    def fem_step(self, precond_p=1):
        return self.L.or_fem_step(self.h, precond_p)

    def calculate_loads(self, patch_id):
        out = np.zeros(5)
        self.L.or_loads(self.h, patch_id, out)
        return out

    def calculate_vorticity(self):
        """nodal vorticity (2D), cylinderDyM/pfem2particle.cpp:1000-1050"""
        if self.L.or_vorticity(self.h) != 0:
            raise ValueError("the vorticity is computed for 2D meshes only")
        return self.field(A.FIELD_VORTICITY)

    def step(self, precond_p=1):
        return self.L.or_step(self.h, precond_p)

    # moving mesh (cylinderDyM)
    def problem_of_elasticity(self, lam, mu, fixed_ids, body_id, disp, tol=0.0, rtol=1e-12, max_iter=10000):
        """mesh displacement into FIELD_DISP_*; returns (iterations, residual)"""
        mask = 0
        for b in fixed_ids:
            mask |= 1 << b
        d = np.zeros(3)
        d[:len(disp)] = disp
        res = C.c_double()
        it = self.L.or_elasticity(self.h, lam, mu, mask, body_id, d, tol, rtol, max_iter, C.byref(res))
        return it, res.value

    def reinterpolate_fields(self):
        self.L.or_reinterpolate(self.h)

    def transform_grid(self):
        """moves the mesh by FIELD_DISP_* and relocates the particles"""
        self.L.or_transform_grid(self.h)

    def move_mesh(self):
        """reinterpolate_fields, transform_grid, sort_particles_into_subdomains_and_cells,
        check_empty_cells (cylinderDyM/cylinderDyM.cc:1157-1160)"""
        self.reinterpolate_fields()
        self.transform_grid()
        self.check_empty()

    def vertices(self):
        out = np.zeros(self.nv * self.dim)
        self.L.or_get_vertices(self.h, out)
        return out.reshape(self.nv, self.dim)

    # state
    def n_particles(self):
        return self.L.or_n_particles(self.h)

    def particles(self):
        n = self.n_particles()
        cell = np.zeros(n, np.int32)
        xi = np.zeros((n, self.dim))
        u = np.zeros((n, self.dim))
        self.L.or_get_particles(self.h, cell, xi.reshape(-1), u.reshape(-1))
        return cell, xi, u

    def positions(self):
        x = np.zeros((self.n_particles(), self.dim))
        self.L.or_get_positions(self.h, x.reshape(-1))
        return x

    def set_particles(self, cell, xi, u, q=None):
        cell = np.ascontiguousarray(cell, np.int32)
        xi = np.ascontiguousarray(xi, np.float64).reshape(-1)
        u = np.ascontiguousarray(u, np.float64).reshape(-1)
        qa = None
        if q is not None:
            qa = np.array(list(q) + [1] * (3 - len(q)), dtype=np.uint32)
        self.L.or_set_particles(self.h, len(cell), cell, xi, u,
                                qa.ctypes.data_as(C.c_void_p) if qa is not None else None)
        self._qkeep = qa

    def field(self, f):
        out = np.zeros(self.nv)
        self.L.or_get_field(self.h, f, out)
        return out

    def set_field(self, f, v):
        self.L.or_set_field(self.h, f, np.ascontiguousarray(v, np.float64))

    def stats(self):
        ints = np.zeros(11, np.int32)
        res = np.zeros(7)
        self.L.or_get_stats(self.h, ints, res)
        return {"n_particles": int(ints[0]), "deleted": int(ints[1]), "removed": int(ints[2]),
                "reseeded": int(ints[3]), "iters": ints[4:].tolist(), "residual": res.tolist()}

    def matrix(self, which):
        nnz = self.L.or_nnz(self.h)
        rp = np.zeros(self.nv + 1, np.int32)
        ci = np.zeros(nnz, np.int32)
        val = np.zeros(nnz)
        self.L.or_get_matrix(self.h, which, rp.ctypes.data_as(C.c_void_p), ci.ctypes.data_as(C.c_void_p),
                             val.ctypes.data_as(C.c_void_p))
        return rp, ci, val

    def assemble_matrices(self):
        self.L.or_assemble_matrices(self.h)

    def rhs(self, which):
        out = np.zeros(self.nv)
        self.L.or_rhs(self.h, which, out)
        return out

    def dirichlet(self, field):
        isd = np.zeros(self.nv, np.uint8)
        val = np.zeros(self.nv)
        self.L.or_get_dirichlet(self.h, field, isd, val)
        return isd.astype(bool), val

    def measure(self):
        return self.L.or_measure(self.h)

    def boundary_measure(self, b):
        n = np.zeros(self.dim)
        s = self.L.or_boundary_measure(self.h, b, n)
        return s, n

    def map_to_unit(self, cell, x):
        xi = np.zeros(self.dim)
        ok = self.L.or_map_to_unit(self.h, cell, np.ascontiguousarray(x, np.float64), xi)
        return bool(ok), xi

    def map_to_real(self, cell, xi):
        x = np.zeros(self.dim)
        self.L.or_map_to_real(self.h, cell, np.ascontiguousarray(xi, np.float64), x)
        return x


def shape_values(dim, xi):
    N = np.zeros(1 << dim)
    lib().or_shape_values(dim, np.ascontiguousarray(xi, np.float64), N)
    return N
