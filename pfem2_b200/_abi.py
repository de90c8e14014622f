"""ctypes mirror of the structs and enums in include/pfem2.h.

The layouts here must match the C header field for field; the CPU test
suite checks sizeof() of each against values the library itself reports.
"""
import ctypes as C

PFEM2_MAX_BC = 8

# pfem2_status
OK, INVALID_ARG, CUDA_ERROR, NOT_CONVERGED, TIMEOUT, PARTICLE_OVERFLOW, NO_DEVICE, BAD_STATE, MESH_ERROR = range(9)
STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARG", 2: "CUDA_ERROR", 3: "NOT_CONVERGED", 4: "TIMEOUT",
    5: "PARTICLE_OVERFLOW", 6: "NO_DEVICE", 7: "BAD_STATE", 8: "MESH_ERROR",
}

PREC_FP64, PREC_MIXED = 0, 1
# PFEM2_FP32_* stage bits of Config.fp32_stages
FP32_PARTICLES, FP32_ASSEMBLY, FP32_KRYLOV, FP32_PRESSURE_RHS = 1, 2, 4, 8
FP32_ALL = FP32_PARTICLES | FP32_ASSEMBLY | FP32_KRYLOV | FP32_PRESSURE_RHS
FP32_DEFAULT = FP32_KRYLOV

(FIELD_VX, FIELD_VY, FIELD_VZ, FIELD_P, FIELD_OLD_VX, FIELD_OLD_VY, FIELD_OLD_VZ, FIELD_OLD_P,
 FIELD_PRED_VX, FIELD_PRED_VY, FIELD_PRED_VZ, FIELD_NODE_WEIGHT, FIELD_VORTICITY,
 FIELD_DISP_X, FIELD_DISP_Y, FIELD_DISP_Z) = range(16)
N_FIELDS = 16
ABI_VERSION = 3  # PFEM2_ABI_VERSION of include/pfem2.h

BC_CONSTANT, BC_PARABOLA = 0, 1
SOLVER_CG, SOLVER_BICGSTAB = 0, 1


class Dirichlet(C.Structure):
    _fields_ = [
        ("boundary_id", C.c_int32), ("kind", C.c_int32), ("axis", C.c_int32), ("pad_", C.c_int32),
        ("value", C.c_double), ("a", C.c_double), ("b", C.c_double),
    ]


class Case(C.Structure):
    _fields_ = [
        ("mu", C.c_double), ("rho", C.c_double), ("dt", C.c_double),
        ("n_dirichlet", C.c_int32 * 4),
        ("dirichlet", (Dirichlet * PFEM2_MAX_BC) * 4),
        ("open_boundary_mask", C.c_uint32),
        ("open_boundary_pressure_flux", C.c_double),
        ("zero_after_projection_mask", C.c_uint32),
        ("load_patch_id", C.c_int32), ("probe_a", C.c_int32), ("probe_b", C.c_int32),
        ("outer_corrections", C.c_int32),
        ("load_diam", C.c_double), ("load_umean", C.c_double),
        ("vel_tol", C.c_double), ("p_tol", C.c_double),
        ("max_iter", C.c_int32), ("vel_solver", C.c_int32), ("p_solver", C.c_int32),
        ("reassemble_every_step", C.c_int32),
        ("wall_pushback", C.c_int32), ("pad_", C.c_int32),
        ("vel_rtol", C.c_double), ("p_rtol", C.c_double),
    ]


class MeshView(C.Structure):
    _fields_ = [
        ("n_vertices", C.c_int32), ("n_cells", C.c_int32),
        ("vertices", C.POINTER(C.c_double)), ("cells", C.POINTER(C.c_int32)),
        ("face_boundary_id", C.POINTER(C.c_int32)),
    ]


class Config(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32),
        ("movement_steps", C.c_int32), ("max_particles_per_cell_part", C.c_int32),
        ("particles_per_cell_max", C.c_int32),
        ("particle_capacity_factor", C.c_double),
        ("far_mover_capacity", C.c_int32), ("use_graph", C.c_int32),
        ("particles_only", C.c_int32), ("fp32_stages", C.c_int32),
        ("moving_mesh", C.c_int32), ("pad_", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("n_particles", C.c_int32), ("n_deleted_last_move", C.c_int32),
        ("n_removed_last_check", C.c_int32), ("n_reseeded_last_check", C.c_int32),
        ("n_far_movers_last_move", C.c_int32),
        ("iters", C.c_int32 * 7), ("residual", C.c_double * 7),
        ("refinements_p", C.c_int32), ("pad_", C.c_int32),
    ]


class Tuning(C.Structure):
    """pfem2_tuning: launch shapes (0 = automatic)"""
    _fields_ = [
        ("advect_blocks_per_sm", C.c_int32), ("advect_split", C.c_int32),
        ("rebin_blocks_per_sm", C.c_int32), ("vel_tile_slices", C.c_int32),
        ("p_blocks_per_sm", C.c_int32), ("vel_blocks_per_sm", C.c_int32),
    ]


TUNING_FIELDS = ["advect_blocks_per_sm", "advect_split", "rebin_blocks_per_sm", "vel_tile_slices", "p_blocks_per_sm",
                 "vel_blocks_per_sm"]


class Elasticity(C.Structure):
    """pfem2_elasticity: the mesh's pseudo-solid and its CG controls"""
    _fields_ = [
        ("lam", C.c_double), ("mu", C.c_double), ("fixed_mask", C.c_uint32), ("body_id", C.c_int32),
        ("tol", C.c_double), ("rtol", C.c_double), ("max_iter", C.c_int32), ("pad_", C.c_int32),
    ]
