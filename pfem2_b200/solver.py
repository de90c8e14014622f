"""Python mirror of the reference's pfem2Solver interface over libpfem2b.so.

Method names follow the reference members (TurekBenchmark/pfem2particle.h:139-243):
seed_particles, correct_particles_velocities, move_particles,
distribute_particle_velocities_to_grid, calculate_loads, plus fem_step
(assemble_system / fem_step of the case drivers) and step (one run() iteration).
Every call goes through the C ABI of include/pfem2.h; a failing status raises
Pfem2Error. There is no CPU fallback: without the built library or a CUDA
device the constructor raises.
"""
import ctypes as C
import os

import numpy as np

from . import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfem2b.so")


class Pfem2Error(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{A.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_LIB = None
N_STAGES = 7
STAGE_NAMES = ["advect", "rebin", "project_nodes", "prediction", "pressure_rhs", "pressure_solve", "correction"]

# every entry point declared in include/pfem2.h
EXPORTS = [
    "pfem2_create", "pfem2_destroy", "pfem2_add_instance", "pfem2_setup", "pfem2_seed", "pfem2_correct",
    "pfem2_move", "pfem2_advect", "pfem2_check_empty", "pfem2_project", "pfem2_fem_step", "pfem2_loads",
    "pfem2_step", "pfem2_step_and_read", "pfem2_get_field", "pfem2_set_field", "pfem2_particle_count",
    "pfem2_get_particles", "pfem2_set_particles", "pfem2_get_stats", "pfem2_get_time", "pfem2_synchronize",
    "pfem2_launch_count", "pfem2_stage_times", "pfem2_enable_stage_timing", "pfem2_get_stream",
    "pfem2_last_error", "pfem2_abi_version", "pfem2_project_noalloc", "pfem2_solver_sizes",
    "pfem2_calculate_vorticity", "pfem2_set_tuning", "pfem2_get_tuning", "pfem2_tuning_key",
    "pfem2_mesh_elasticity", "pfem2_move_mesh", "pfem2_get_vertices",
]


def load_library(path=LIB_PATH):
    """Loads the in-tree libpfem2b.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise Pfem2Error(A.NO_DEVICE, f"{path} not built (run pfem2_b200/build.py)")
    lib = C.CDLL(path)
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    st = C.c_int
    sig = {
        "pfem2_create": [C.POINTER(A.Config), C.POINTER(vp)],
        "pfem2_destroy": [vp],
        "pfem2_add_instance": [vp, C.POINTER(A.MeshView), C.POINTER(A.Case), ip],
        "pfem2_setup": [vp],
        "pfem2_seed": [vp, C.c_int32, C.POINTER(C.c_uint32), C.c_uint64, C.c_double],
        "pfem2_correct": [vp], "pfem2_move": [vp], "pfem2_advect": [vp], "pfem2_check_empty": [vp],
        "pfem2_project": [vp], "pfem2_fem_step": [vp], "pfem2_step": [vp],
        "pfem2_loads": [vp, C.c_int32, C.c_int32, dp],
        "pfem2_step_and_read": [vp, dp, ip, C.c_int32, dp],
        "pfem2_get_field": [vp, C.c_int32, C.c_int32, dp],
        "pfem2_set_field": [vp, C.c_int32, C.c_int32, dp],
        "pfem2_particle_count": [vp, C.c_int32, ip],
        "pfem2_get_particles": [vp, C.c_int32, ip, dp, dp],
        "pfem2_set_particles": [vp, ip, ip, dp, dp],
        "pfem2_get_stats": [vp, C.POINTER(A.Stats)],
        "pfem2_get_time": [vp, dp, ip],
        "pfem2_synchronize": [vp],
        "pfem2_launch_count": [vp, C.POINTER(C.c_int64)],
        "pfem2_stage_times": [vp, dp, C.c_int32],
        "pfem2_solver_sizes": [vp, C.POINTER(C.c_int64)],
        "pfem2_calculate_vorticity": [vp],
        "pfem2_enable_stage_timing": [vp, C.c_int32],
        "pfem2_get_stream": [vp, C.POINTER(vp)],
        "pfem2_set_tuning": [vp, C.POINTER(A.Tuning)],
        "pfem2_get_tuning": [vp, C.POINTER(A.Tuning)],
        "pfem2_tuning_key": [vp, C.c_char_p, C.c_int32],
        "pfem2_mesh_elasticity": [vp, C.c_int32, C.POINTER(A.Elasticity), dp, ip, dp],
        "pfem2_move_mesh": [vp],
        "pfem2_get_vertices": [vp, C.c_int32, dp],
    }
    sig["pfem2_project_noalloc"] = [C.c_int32, C.c_int32, C.c_int32] + [vp] * 9 + [vp]
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = st
    lib.pfem2_last_error.restype = C.c_char_p
    lib.pfem2_last_error.argtypes = []
    lib.pfem2_abi_version.restype = C.c_int32
    _LIB = lib
    return lib


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class Solver:
    """pfem2Solver over a batch of instances (one instance = one case)."""

    def __init__(self, specs, precision=A.PREC_MIXED, device=0, movement_steps=None, max_per_part=None,
                 use_graph=True, capacity_factor=2.0, per_cell_max=0, particles_only=False, fp32_stages=0,
                 far_capacity=0, tuning=None, moving_mesh=False):
        """tuning: a dict of pfem2_tuning fields (launch shapes) set before
        setup; unset or 0 fields come from the tuning cache named by
        PFEM2_TUNING_CACHE, else from the sizes"""
        if not isinstance(specs, (list, tuple)):
            specs = [specs]
        self.L = load_library()
        self.specs = list(specs)
        self.dim = specs[0].mesh.dim
        cfg = A.Config()
        cfg.dim = self.dim
        cfg.precision = precision
        cfg.device = device
        cfg.movement_steps = movement_steps if movement_steps is not None else specs[0].movement_steps
        cfg.max_particles_per_cell_part = max_per_part if max_per_part is not None else specs[0].max_per_part
        cfg.particles_per_cell_max = per_cell_max
        cfg.particle_capacity_factor = capacity_factor
        cfg.far_mover_capacity = far_capacity
        cfg.use_graph = 1 if use_graph else 0
        cfg.particles_only = 1 if particles_only else 0
        cfg.fp32_stages = fp32_stages
        cfg.moving_mesh = 1 if moving_mesh else 0
        self.cfg = cfg
        h = C.c_void_p()
        self._check(self.L.pfem2_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self._keep = []
        for sp in self.specs:
            m = sp.mesh
            X = np.ascontiguousarray(m.vertices, np.float64)
            cv = np.ascontiguousarray(m.cells, np.int32)
            fb = np.ascontiguousarray(m.face_bid, np.int32)
            self._keep += [X, cv, fb]
            mv = A.MeshView(m.n_vertices, m.n_cells, _dptr(X), _iptr(cv), _iptr(fb))
            inst = C.c_int32()
            self._check(self.L.pfem2_add_instance(self.h, C.byref(mv), C.byref(sp.case), C.byref(inst)))
        if tuning:
            t = A.Tuning()
            for k, v in tuning.items():
                setattr(t, k, int(v))
            self._check(self.L.pfem2_set_tuning(self.h, C.byref(t)))
        self._check(self.L.pfem2_setup(self.h))
        self._keep = []

    def _check(self, s):
        if s != A.OK:
            raise Pfem2Error(s, self.L.pfem2_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.pfem2_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- pfem2Solver members
    def seed_particles(self, q, seed=0, jitter=0.0, instance=-1):
        qq = (C.c_uint32 * 3)(*(list(q) + [1] * (3 - len(q))))
        self._check(self.L.pfem2_seed(self.h, instance, qq, seed, jitter))

    def correct_particles_velocities(self):
        self._check(self.L.pfem2_correct(self.h))

    def move_particles(self):
        self._check(self.L.pfem2_move(self.h))

    def advect(self):
        self._check(self.L.pfem2_advect(self.h))

    def check_empty(self):
        self._check(self.L.pfem2_check_empty(self.h))

    def distribute_particle_velocities_to_grid(self):
        self._check(self.L.pfem2_project(self.h))

    def fem_step(self):
        self._check(self.L.pfem2_fem_step(self.h))

    def calculate_loads(self, patch_id, instance=0):
        out = np.zeros(5)
        self._check(self.L.pfem2_loads(self.h, instance, patch_id, _dptr(out)))
        return out

    def calculate_vorticity(self, instance=0):
        """calculate_vorticity (cylinderDyM/pfem2particle.cpp:1000-1050), 2D:
        the nodal vorticity of every instance; returns the given instance's."""
        self._check(self.L.pfem2_calculate_vorticity(self.h))
        return self.field(A.FIELD_VORTICITY, instance)

    def step(self):
        self._check(self.L.pfem2_step(self.h))

    # ---- moving mesh (cylinderDyM)
    def problem_of_elasticity(self, lam, mu, fixed_ids, body_id, disp, tol=0.0, rtol=1e-12, max_iter=10000):
        """problem_of_elasticity + solveU (cylinderDyM/cylinderDyM.cc:926-976,
        886-903): the mesh displacement into FIELD_DISP_*; returns
        (iterations, residual)"""
        e = A.Elasticity()
        e.lam, e.mu, e.body_id, e.tol, e.rtol, e.max_iter = lam, mu, body_id, tol, rtol, max_iter
        mask = 0
        for b in fixed_ids:
            mask |= 1 << b
        e.fixed_mask = mask
        d = np.zeros(3)
        d[:len(disp)] = disp
        it, res = C.c_int32(), C.c_double()
        self._check(self.L.pfem2_mesh_elasticity(self.h, 0, C.byref(e), _dptr(d), C.byref(it), C.byref(res)))
        return it.value, res.value

    def move_mesh(self):
        """reinterpolate_fields, transform_grid, sort_particles_into_subdomains_and_cells
        and check_empty_cells (cylinderDyM/cylinderDyM.cc:1157-1160)"""
        self._check(self.L.pfem2_move_mesh(self.h))

    def step_and_read(self, fields=(A.FIELD_VX, A.FIELD_VY, A.FIELD_P), loads=None, out=None):
        n_inst = len(self.specs)
        if loads is None:
            loads = np.zeros(5 * n_inst)
        f = np.asarray(fields, np.int32)
        if out is None:
            out = np.zeros(sum(sp.mesh.n_vertices for sp in self.specs) * len(f))
        self._check(self.L.pfem2_step_and_read(self.h, _dptr(loads), _iptr(f), len(f), _dptr(out)))
        return loads, out

    # ---- state
    def field(self, f, instance=0):
        out = np.zeros(self.specs[instance].mesh.n_vertices)
        self._check(self.L.pfem2_get_field(self.h, instance, f, _dptr(out)))
        return out

    def set_field(self, f, values, instance=0):
        v = np.ascontiguousarray(values, np.float64)
        self._check(self.L.pfem2_set_field(self.h, instance, f, _dptr(v)))

    def vertices(self, instance=0):
        """vertex coordinates [n_vertices, dim] (moved by move_mesh)"""
        out = np.zeros(self.specs[instance].mesh.n_vertices * self.dim)
        self._check(self.L.pfem2_get_vertices(self.h, instance, _dptr(out)))
        return out.reshape(-1, self.dim)

    def n_particles(self, instance=0):
        n = C.c_int32()
        self._check(self.L.pfem2_particle_count(self.h, instance, C.byref(n)))
        return n.value

    def particles(self, instance=0):
        n = self.n_particles(instance)
        cell = np.zeros(n, np.int32)
        xi = np.zeros((n, self.dim))
        u = np.zeros((n, self.dim))
        if n:
            self._check(self.L.pfem2_get_particles(self.h, instance, _iptr(cell), _dptr(xi), _dptr(u)))
        return cell, xi, u

    def set_particles(self, per_instance):
        """per_instance: list of (cell, xi, u) tuples, one per instance."""
        counts = np.array([len(p[0]) for p in per_instance], np.int32)
        cell = np.ascontiguousarray(np.concatenate([p[0] for p in per_instance]), np.int32)
        xi = np.ascontiguousarray(np.concatenate([p[1] for p in per_instance]), np.float64)
        u = np.ascontiguousarray(np.concatenate([p[2] for p in per_instance]), np.float64)
        self._check(self.L.pfem2_set_particles(self.h, _iptr(counts), _iptr(cell), _dptr(xi), _dptr(u)))

    def stats(self, check=True):
        """Counters of the last particle pass and the last Krylov solves. With
        check=False a failing status (e.g. NOT_CONVERGED) is returned in the
        dict under 'status' instead of raised."""
        s = A.Stats()
        st = self.L.pfem2_get_stats(self.h, C.byref(s))
        if check:
            self._check(st)
        return {"n_particles": s.n_particles, "deleted": s.n_deleted_last_move,
                "removed": s.n_removed_last_check, "reseeded": s.n_reseeded_last_check,
                "far": s.n_far_movers_last_move, "iters": list(s.iters), "residual": list(s.residual),
                "refinements_p": s.refinements_p, "status": st}

    def synchronize(self):
        self._check(self.L.pfem2_synchronize(self.h))

    def launch_count(self):
        n = C.c_int64()
        self._check(self.L.pfem2_launch_count(self.h, C.byref(n)))
        return n.value

    def sizes(self):
        """Rows (vertices), CSR nonzeros and arithmetic-type bytes of the batch."""
        rows = nnz = 0
        for sp in self.specs:
            cv = sp.mesh.cells.astype(np.int64)
            nvc = cv.shape[1]
            a = np.repeat(cv, nvc, axis=1).reshape(-1)
            b = np.tile(cv, (1, nvc)).reshape(-1)
            nnz += len(np.unique(a * sp.mesh.n_vertices + b))
            rows += sp.mesh.n_vertices
        return {"rows": rows, "nnz": nnz, "real_bytes": 4 if A.FP32_KRYLOV & self.fp32_stages() else 8}

    def fp32_stages(self):
        """The PFEM2_FP32_* stages this context runs in FP32."""
        if self.cfg.precision != A.PREC_MIXED:
            return 0
        return self.cfg.fp32_stages or A.FP32_DEFAULT

    def tuning(self):
        """the launch shapes in use (pfem2_get_tuning)"""
        t = A.Tuning()
        self._check(self.L.pfem2_get_tuning(self.h, C.byref(t)))
        return {k: getattr(t, k) for k in A.TUNING_FIELDS}

    def tuning_key(self):
        """the key this context looks the tuning cache up with"""
        buf = C.create_string_buffer(512)
        self._check(self.L.pfem2_tuning_key(self.h, buf, 512))
        return buf.value.decode()

    def enable_stage_timing(self, on=True):
        self._check(self.L.pfem2_enable_stage_timing(self.h, 1 if on else 0))

    def solver_sizes(self):
        """Multigrid hierarchy of the pressure solve (pfem2_solver_sizes)."""
        out = (C.c_int64 * 12)()
        self._check(self.L.pfem2_solver_sizes(self.h, out))
        keys = ("n0", "n1", "n2", "n3", "r01", "r02", "c3", "p0", "j1", "p1", "j2", "p2")
        return dict(zip(keys, (int(v) for v in out)))

    def stage_times(self, reset=False):
        ms = np.zeros(N_STAGES)
        self._check(self.L.pfem2_stage_times(self.h, _dptr(ms), 1 if reset else 0))
        return ms

    def stream(self):
        s = C.c_void_p()
        self._check(self.L.pfem2_get_stream(self.h, C.byref(s)))
        return s.value
