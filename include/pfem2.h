/*
 * pfem2.h -- C ABI of the B200-native PFEM2 time-step library (libpfem2b.so).
 *
 * The reference (andreyypopov/pfem2) exposes its hot path as the member
 * functions of `class pfem2Solver` (TurekBenchmarkCuda/pfem2particle.h:126-233,
 * TurekBenchmark/pfem2particle.h:139-243, tubePoiseuille3D/pfem2particle.h).
 * Every function below replaces one of those members (cited beside it); the
 * header-only C++ class in pfem2_solver.hpp forwards the reference's member
 * names to these entry points so a case driver keeps its run() order:
 *
 *     correct_particles_velocities -> move_particles ->
 *     distribute_particle_velocities_to_grid -> fem_step -> calculate_loads
 *
 * Conventions
 *  - Plain pointers and sizes only; every entry point returns pfem2_status.
 *  - A context owns all device memory and one CUDA stream. Calls on one
 *    context are not re-entrant; distinct contexts are independent.
 *  - A context holds a BATCH of independent flow instances (a single case is
 *    a batch of one). Cells, vertices (= Q1 DoFs) and particles of all
 *    instances are concatenated; per-instance arrays passed to or returned by
 *    the API use the instance's own local numbering.
 *  - Vertex order inside a cell and face numbering follow deal.II
 *    (lexicographic): vertex v has reference coordinate bit d of v along axis
 *    d; face f lies on axis f/2 at side f%2.
 *  - Host buffers passed in are copied; nothing is retained after return.
 */
#ifndef PFEM2_H
#define PFEM2_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define PFEM2_ABI_VERSION 3

typedef enum {
  PFEM2_OK = 0,
  PFEM2_INVALID_ARG = 1,
  PFEM2_CUDA_ERROR = 2,
  PFEM2_NOT_CONVERGED = 3,      /* a Krylov solve hit max_iter (reference only prints this) */
  PFEM2_TIMEOUT = 4,            /* a bounded device-side wait gave up */
  PFEM2_PARTICLE_OVERFLOW = 5,  /* particle / per-cell / far-mover capacity exceeded */
  PFEM2_NO_DEVICE = 6,
  PFEM2_BAD_STATE = 7,          /* call order violated (e.g. step before setup) */
  PFEM2_MESH_ERROR = 8          /* inverted cell, bad connectivity */
} pfem2_status;

typedef enum {
  PFEM2_PREC_FP64 = 0,   /* everything FP64 ("plain" path) */
  PFEM2_PREC_MIXED = 1   /* the stages of pfem2_config.fp32_stages in FP32; FP64 refinement, dots, loads */
} pfem2_precision;

/* Stages that a PFEM2_PREC_MIXED context runs in FP32 (pfem2_config.fp32_stages,
 * a bit mask; 0 selects PFEM2_FP32_DEFAULT). Everything not listed stays FP64:
 * the nodal fields, the Krylov residual refinement, dot products and norms,
 * the load integrals. The default keeps the fields within 1e-6 relative L2
 * of the FP64 path: only the inner Krylov iterations run in FP32, their
 * result refined in FP64 to the FP64 tolerance. Each further stage in FP32
 * moves the fields by 1e-5 to 4e-4 relative L2 after 25 steps of the 52k-cell
 * disk channel (particles: 8e-6 vx, 4e-5 p; prediction/correction right-hand
 * sides: 2e-5 vx, 2e-4 p; pressure right-hand side: 7e-6 vx, 4e-4 p). */
#define PFEM2_FP32_PARTICLES 1  /* particle state (reference coordinates, velocities) and the particle kernels */
#define PFEM2_FP32_ASSEMBLY 2   /* right-hand sides of the prediction and correction systems */
#define PFEM2_FP32_KRYLOV 4     /* inner Krylov iterations (FP64 reliable updates to the FP64 tolerance) */
#define PFEM2_FP32_PRESSURE_RHS 8 /* right-hand side of the pressure Poisson system */
#define PFEM2_FP32_ALL 15       /* every stage above */
#define PFEM2_FP32_DEFAULT PFEM2_FP32_KRYLOV

typedef enum {
  PFEM2_FIELD_VX = 0, PFEM2_FIELD_VY = 1, PFEM2_FIELD_VZ = 2, PFEM2_FIELD_P = 3,
  PFEM2_FIELD_OLD_VX = 4, PFEM2_FIELD_OLD_VY = 5, PFEM2_FIELD_OLD_VZ = 6, PFEM2_FIELD_OLD_P = 7,
  PFEM2_FIELD_PRED_VX = 8, PFEM2_FIELD_PRED_VY = 9, PFEM2_FIELD_PRED_VZ = 10,
  PFEM2_FIELD_NODE_WEIGHT = 11,  /* sum of shape values from the last projection */
  PFEM2_FIELD_VORTICITY = 12,    /* nodal vorticity from the last pfem2_calculate_vorticity (2D) */
  PFEM2_FIELD_DISP_X = 13,       /* mesh displacement of the last pfem2_mesh_elasticity */
  PFEM2_FIELD_DISP_Y = 14,
  PFEM2_FIELD_DISP_Z = 15,
  PFEM2_N_FIELDS = 16
} pfem2_field;

typedef enum {
  PFEM2_BC_CONSTANT = 0,   /* value */
  PFEM2_BC_PARABOLA = 1    /* value * 4 (s-a)(b-s)/(b-a)^2, s = vertex coordinate `axis` */
} pfem2_bc_kind;

typedef enum {
  PFEM2_SOLVER_CG = 0,
  PFEM2_SOLVER_BICGSTAB = 1
} pfem2_solver_kind;

/* One Dirichlet condition: all vertices of boundary faces with `boundary_id`.
 * Conditions of a field are applied in array order; a vertex on several
 * listed boundaries takes the last one (as successive
 * MatrixTools::apply_boundary_values calls do, cylinder2D/cylinder2D.cc:459-466). */
typedef struct {
  int32_t boundary_id;
  int32_t kind;      /* pfem2_bc_kind */
  int32_t axis;      /* PARABOLA only */
  int32_t pad_;
  double value;
  double a, b;       /* PARABOLA only */
} pfem2_dirichlet;

#define PFEM2_MAX_BC 8

/* Physics, boundary conditions and solver controls of one instance.
 * Field index for bc arrays: 0..dim-1 = velocity components, 3 = pressure. */
typedef struct {
  double mu, rho, dt;
  int32_t n_dirichlet[4];
  pfem2_dirichlet dirichlet[4][PFEM2_MAX_BC];
  /* Boundary ids (bit mask) that are inflow/outflow sections: the prediction
   * stress face terms and the pressure flux face term are integrated there
   * (cylinder2D/cylinder2D.cc:432-447,582-597; tubePoiseuille3D/tube.cc:253-273,496-510). */
  uint32_t open_boundary_mask;
  /* Neumann pressure term G * n_x integrated over open faces
   * (tubePoiseuille3D/tube.cc:509 uses G = -10); 0 in 2D cases. */
  double open_boundary_pressure_flux;
  /* Boundary ids whose vertices are set to zero velocity right after the
   * particle->grid projection (wallsAndBodyDoFs, TurekBenchmarkCuda/pfem2particle.cu:866-869). */
  uint32_t zero_after_projection_mask;
  /* Loads (calculate_loads): obstacle patch id, reference diameter and mean
   * velocity for the coefficients, and the two probe vertices of the
   * pressure difference (-1 = unused), TurekBenchmark/pfem2particle.cpp:920-970. */
  int32_t load_patch_id;
  int32_t probe_a, probe_b;
  int32_t outer_corrections;      /* nOuterCorr (cylinder2D/cylinder2D.cc:395) */
  double load_diam, load_umean;
  /* Krylov controls: SolverControl(max_iter, tol) with the absolute
   * unpreconditioned residual norm as in deal.II (cylinder2D/cylinder2D.cc:736-779). */
  double vel_tol, p_tol;
  int32_t max_iter;
  /* pfem2_solver_kind of the velocity systems (prediction and correction):
   * CG or BiCGStab, both with the Jacobi preconditioner of the reference's
   * velocity solves (cylinder2D/cylinder2D.cc:736-758). */
  int32_t vel_solver;
  /* pfem2_solver_kind of the pressure system: CG with the algebraic multigrid
   * preconditioner (the reference's Trilinos cases use AMG,
   * TurekBenchmarkCuda/TurekBenchmark.cc:731-797), or BiCGStab with the
   * Jacobi preconditioner (the reference's serial cases use BiCGStab with
   * SSOR, cylinder2D/cylinder2D.cc:760-779). Every instance of a context
   * must name the same kinds (PFEM2_INVALID_ARG otherwise). */
  int32_t p_solver;
  int32_t reassemble_every_step;  /* 1: rebuild matrices each step like the reference */
  /* 1: wall push-back after the projection (nacaAirfoil/pfem2particle.cpp:
   * 919-952): for every zero_after_projection vertex whose projected
   * velocity has a component above 1e-5 in magnitude, every particle of the
   * cells around it loses N_vertex(xi_p) times that velocity, before the
   * vertex is set to zero. 0: the vertex is only set to zero. */
  int32_t wall_pushback;
  int32_t pad_;
  /* Relative tolerances (0 = off): a solve stops once its residual norm is
   * <= max(tol, rtol * |b|), |b| the norm of its right-hand side (deal.II's
   * SolverControl with the tolerance scaled by the right-hand side). Tight
   * values make two runs that differ only in arithmetic comparable. */
  double vel_rtol, p_rtol;
} pfem2_case;

/* A mesh of one instance (host arrays, copied by pfem2_add_instance). */
typedef struct {
  int32_t n_vertices;
  int32_t n_cells;
  const double* vertices;          /* [n_vertices][dim] */
  const int32_t* cells;            /* [n_cells][2^dim], deal.II vertex order */
  const int32_t* face_boundary_id; /* [n_cells][2*dim], -1 = interior face */
} pfem2_mesh_view;

typedef struct {
  int32_t dim;                     /* 2 or 3 */
  int32_t precision;               /* pfem2_precision */
  int32_t device;                  /* CUDA ordinal */
  int32_t movement_steps;          /* PARTICLES_MOVEMENT_STEPS (pfem2particle.h:4), 1 .. 65535 */
  int32_t max_particles_per_cell_part; /* MAX_PARTICLES_PER_CELL_PART (pfem2particle.h:5) */
  int32_t particles_per_cell_max;  /* per-cell capacity of the rebin pass (0 = auto) */
  double particle_capacity_factor; /* particle storage = factor * seeded count (0 = 2.0) */
  int32_t far_mover_capacity;      /* particles that leave the 1-ring of their cell in one step (0 = 16384, the most) */
  int32_t use_graph;               /* capture pfem2_step as a CUDA graph */
  /* 1: no FEM (no matrices are set up; pfem2_fem_step is refused). pfem2_step
   * then runs correct -> move -> project on a frozen velocity field held in
   * PFEM2_FIELD_PRED_V*: after each step V is reset to the frozen field and
   * V_old to the new projection (the particle-kernel stress workload). */
  int32_t particles_only;
  /* PFEM2_PREC_MIXED only: the PFEM2_FP32_* stages that run in FP32
   * (0 = PFEM2_FP32_DEFAULT). Ignored by PFEM2_PREC_FP64. */
  int32_t fp32_stages;
  /* 1: the mesh moves (pfem2_mesh_elasticity / pfem2_move_mesh, 2D, one
   * instance): the matrices are reassembled every step and the pressure is
   * solved without the multigrid hierarchy, which is built once on the host
   * (CG with Jacobi, or BiCGStab with Jacobi as p_solver says). */
  int32_t moving_mesh;
  int32_t pad_;
} pfem2_config;

typedef struct pfem2_ctx pfem2_ctx;

typedef struct {
  int32_t n_particles;
  int32_t n_deleted_last_move;     /* left the mesh or found in no patch cell */
  int32_t n_removed_last_check;    /* over MAX_PARTICLES_PER_CELL_PART */
  int32_t n_reseeded_last_check;   /* one per empty sub-cell */
  int32_t n_far_movers_last_move;
  int32_t iters[7];                /* last Krylov iterations: pred x,y,z, p, corr x,y,z */
  double residual[7];              /* last absolute residual norms */
  int32_t refinements_p;           /* FP64 refinement sweeps of the last pressure solve */
  int32_t pad_;
} pfem2_stats;

/* ---- lifecycle (pfem2Solver::pfem2Solver, build_grid, setup_system) ---- */
pfem2_status pfem2_create(const pfem2_config* cfg, pfem2_ctx** out);
pfem2_status pfem2_destroy(pfem2_ctx* ctx);
/* Adds one instance (build_grid; cases' GridIn / GridGenerator calls). */
pfem2_status pfem2_add_instance(pfem2_ctx* ctx, const pfem2_mesh_view* mesh,
                                const pfem2_case* cs, int32_t* instance_out);
/* Builds DoF maps, sparsity, boundary tables, vertex->cell maps and assembles
 * the step-invariant matrices (setup_system, TurekBenchmarkCuda/TurekBenchmark.cc:282-403;
 * pfem2ParticleHandler::initialize_maps, TurekBenchmark/pfem2particle.cpp:215-219). */
pfem2_status pfem2_setup(pfem2_ctx* ctx);

/* ---- the pfem2Solver member functions ---- */
/* seed_particles (TurekBenchmark/pfem2particle.cpp:701-721,774-790): q[d]
 * particles per axis per cell at sub-cell centres, plus a uniform jitter of
 * +-jitter (reference units) from a counter-based SplitMix64 stream keyed by
 * (seed, global particle ordinal, axis). instance < 0: all instances. */
pfem2_status pfem2_seed(pfem2_ctx* ctx, int32_t instance, const uint32_t q[3],
                        uint64_t seed, double jitter);
/* correct_particles_velocities (TurekBenchmark/pfem2particle.cpp:792-811). */
pfem2_status pfem2_correct(pfem2_ctx* ctx);
/* move_particles incl. point location and check_cell_for_empty_parts
 * (TurekBenchmark/pfem2particle.cpp:813-856, :276-507, :723-772). */
pfem2_status pfem2_move(pfem2_ctx* ctx);
/* move_particles without the final check (advection + location + re-sort). */
pfem2_status pfem2_advect(pfem2_ctx* ctx);
/* check_cells_for_empty_parts alone (TurekBenchmarkCuda/pfem2particle.cu:360-416). */
pfem2_status pfem2_check_empty(pfem2_ctx* ctx);
/* distribute_particle_velocities_to_grid (TurekBenchmark/pfem2particle.cpp:858-918). */
pfem2_status pfem2_project(pfem2_ctx* ctx);
/* fem_step / assemble_system: prediction, pressure Poisson, correction
 * (cylinder2D/cylinder2D.cc:385-731, tubePoiseuille3D/tube.cc:165-715). */
pfem2_status pfem2_fem_step(pfem2_ctx* ctx);
/* calculate_loads (TurekBenchmark/pfem2particle.cpp:920-970): out[5] =
 * {Cx_nu, Cx_p, Cy_nu, Cy_p, p(probe_a) - p(probe_b)} (2D). In 3D out =
 * {Fx_p, Fy_p, Fz_p, 0, p_probe} with p_probe the mean pressure over the
 * probe vertices that are set (tubePoiseuille3D/pfem2particle.cpp:693-737). */
pfem2_status pfem2_loads(pfem2_ctx* ctx, int32_t instance, int32_t patch_id, double out[5]);
/* calculate_vorticity (cylinderDyM/pfem2particle.cpp:1000-1050), 2D: at the
 * QGauss(2) points of every cell w = sum_i (dN_i/dx Vy_i - dN_i/dy Vx_i),
 * and at every vertex the sum over its cells and their points of N_vertex w
 * divided by the sum of N_vertex; into PFEM2_FIELD_VORTICITY of every
 * instance (read it with pfem2_get_field). INVALID_ARG in 3D. */
pfem2_status pfem2_calculate_vorticity(pfem2_ctx* ctx);
/* One whole time step: correct -> move -> project -> fem_step, with fused
 * kernels (and a CUDA graph if cfg.use_graph); advances time by dt. */
pfem2_status pfem2_step(pfem2_ctx* ctx);
/* Same as pfem2_step, then loads of every instance into out[5*n_instances]
 * and a host read of all instances' nodal fields listed in `fields`
 * (n_fields entries) into `host_fields` (instance-major, field, vertex). */
pfem2_status pfem2_step_and_read(pfem2_ctx* ctx, double* loads_out,
                                 const int32_t* fields, int32_t n_fields,
                                 double* host_fields);

/* ---- moving mesh (cylinderDyM) ----
 * The reference's moving-mesh driver advances, per time step
 * (cylinderDyM/cylinderDyM.cc:1146-1160): correct -> move -> distribute ->
 * fem_step -> calculate_loads -> the body displacement from its motion ODE
 * (the driver's own code) -> problem_of_elasticity -> reinterpolate_fields
 * -> transform_grid -> sort_particles_into_subdomains_and_cells ->
 * check_empty_cells. The two calls below replace the members from
 * problem_of_elasticity on; they need pfem2_config.moving_mesh. */
typedef struct {
  double lambda, mu;     /* Lame parameters of the mesh's pseudo-solid */
  uint32_t fixed_mask;   /* boundary ids (bit mask) held at zero displacement */
  int32_t body_id;       /* boundary id displaced by body_disp (-1: none) */
  double tol, rtol;      /* CG stops at |r| <= max(tol, rtol |b|) */
  int32_t max_iter;
  int32_t pad_;
} pfem2_elasticity;
/* problem_of_elasticity + solveU (cylinderDyM/cylinderDyM.cc:926-976,
 * 886-903): the displacement of every vertex from the linear elasticity
 * system sum_q [lambda d_ci N_a d_cj N_b + mu d_cj N_a d_ci N_b
 * + delta_ci,cj mu grad N_a . grad N_b] JxW on the current mesh, u = 0 on
 * fixed_mask, u = body_disp on body_id, solved by CG (Jacobi) into
 * PFEM2_FIELD_DISP_X/Y; iterations and the final residual norm out
 * (either may be NULL). NOT_CONVERGED past max_iter. */
pfem2_status pfem2_mesh_elasticity(pfem2_ctx* ctx, int32_t instance, const pfem2_elasticity* e,
                                   const double body_disp[3], int32_t* iterations, double* residual);
/* reinterpolate_fields + transform_grid + sort_particles_into_subdomains_and_
 * cells + check_empty_cells (cylinderDyM/pfem2particle.cpp:1144-1261): every
 * interior vertex takes Vx, Vy, P interpolated at its displaced position in
 * the old mesh (boundary vertices keep theirs), the vertices move by the
 * displacement, every particle keeps its physical position and is located
 * in the moved mesh (its cell, else the reference's vertex-patch search
 * along the direction it moved relative to the mesh; deleted when found
 * nowhere), then the empty sub-cells are refilled. PFEM2_MESH_ERROR if a
 * cell turned inside out. */
pfem2_status pfem2_move_mesh(pfem2_ctx* ctx);

/* ---- state access (public data members of pfem2Solver) ---- */
pfem2_status pfem2_get_field(pfem2_ctx* ctx, int32_t instance, int32_t field, double* host);
pfem2_status pfem2_set_field(pfem2_ctx* ctx, int32_t instance, int32_t field, const double* host);
pfem2_status pfem2_particle_count(pfem2_ctx* ctx, int32_t instance, int32_t* n);
/* Vertex coordinates of an instance [n_vertices][dim] (they change with
 * pfem2_move_mesh; the reference's Triangulation vertices). */
pfem2_status pfem2_get_vertices(pfem2_ctx* ctx, int32_t instance, double* host);
/* Particles of an instance in storage order (sorted by cell): local cell id,
 * reference coordinates [n][dim] and velocity [n][dim]. */
pfem2_status pfem2_get_particles(pfem2_ctx* ctx, int32_t instance, int32_t* cell,
                                 double* xi, double* u);
/* Replaces the particles of ALL instances: n particles with instance-local
 * cells given per instance by counts[n_instances] (instance-major order);
 * the library sorts them (stable) by cell. */
pfem2_status pfem2_set_particles(pfem2_ctx* ctx, const int32_t* counts, const int32_t* cell,
                                 const double* xi, const double* u);
pfem2_status pfem2_get_stats(pfem2_ctx* ctx, pfem2_stats* out);
pfem2_status pfem2_get_time(pfem2_ctx* ctx, double* time, int32_t* timestep_number);
pfem2_status pfem2_synchronize(pfem2_ctx* ctx);
/* Device kernel launches issued by this context so far (for accounting). */
pfem2_status pfem2_launch_count(pfem2_ctx* ctx, int64_t* n);
/* Device time (ms) of the stages of pfem2_step accumulated since the last
 * reset (PFEM2_N_STAGES values): 0 correct+advect+locate, 1 rebin (re-sort,
 * check_cell_for_empty_parts, projection partials), 2 projection node gather,
 * 3 prediction rhs + solves, 4 pressure rhs, 5 pressure solve, 6 correction
 * rhs + solves + update. Needs pfem2_enable_stage_timing; synchronizes. */
#define PFEM2_N_STAGES 7
pfem2_status pfem2_stage_times(pfem2_ctx* ctx, double* ms, int32_t reset);
/* Enable per-stage CUDA-event timing of pfem2_step (off by default). */
pfem2_status pfem2_enable_stage_timing(pfem2_ctx* ctx, int32_t on);
/* The CUDA stream (cudaStream_t) all work of the context is issued on. */
pfem2_status pfem2_get_stream(pfem2_ctx* ctx, void** stream);
/* Sizes of the pressure solver's multigrid hierarchy after pfem2_setup
 * (diagnostics; no counterpart in the reference). out[0..3]: unknowns per
 * level; out[4..11]: stored nonzeros of R01, R02, the b3 contribution rows,
 * the level-0 prolongator, and the J1, Pt1, J2, Pt2 rows of all blocks'
 * coarse lists (halo rows counted once per block that evaluates them).
 * All zero without a hierarchy. */
#define PFEM2_N_SOLVER_SIZES 12
pfem2_status pfem2_solver_sizes(pfem2_ctx* ctx, int64_t* out);
const char* pfem2_last_error(void);
int32_t pfem2_abi_version(void);

/* ---- launch shapes and their autotuning ----
 * No counterpart in the reference (its kernels have fixed launch shapes).
 * Each field 0 = automatic. None of them changes the particle kernels'
 * arithmetic (their results are bitwise the same under every setting); the
 * velocity tile size and blocks per SM change the order of the solver's
 * partial sums and the pressure width its preconditioner, all within the
 * solver tolerance. */
typedef struct {
  int32_t advect_blocks_per_sm;  /* advection grid in 256-thread blocks per SM (sets particles per block) */
  int32_t advect_split;          /* 1: one advection pass, 2: stayers, then each block's queued leavers */
  int32_t rebin_blocks_per_sm;   /* re-sort grid in 256-thread blocks per SM (tiles of 8 cells) */
  int32_t vel_tile_slices;       /* velocity solves: SELL slices of 32 rows per Krylov tile */
  int32_t p_blocks_per_sm;       /* pressure multigrid of a single system: 1 or 2 blocks per SM */
  int32_t vel_blocks_per_sm;     /* velocity solves: 1 or 2 blocks per SM */
} pfem2_tuning;
/* Sets the launch shapes (before pfem2_setup). Fields left at 0 are taken
 * from the tuning cache named by the environment variable PFEM2_TUNING_CACHE
 * (written by the autotuner, pfem2_b200/autotune.py) when it holds an entry
 * for this context's key, else chosen by size. */
pfem2_status pfem2_set_tuning(pfem2_ctx* ctx, const pfem2_tuning* t);
/* The launch shapes in use (after pfem2_setup: every field resolved). */
pfem2_status pfem2_get_tuning(pfem2_ctx* ctx, pfem2_tuning* t);
/* The key of the tuning cache for this context (after pfem2_add_instance):
 * "<device name> <dim> <fp32 stages, -1 for FP64> <log2 cells> <log2 instances>". */
pfem2_status pfem2_tuning_key(pfem2_ctx* ctx, char* buf, int32_t len);

/* ---- projection without allocation ----
 * No counterpart in the reference. For callers that cannot let the library
 * call cudaMalloc (a host code that owns all device memory through its own
 * pool, or work being recorded into a CUDA graph): the particle -> grid
 * projection of distribute_particle_velocities_to_grid on caller-owned
 * device buffers, FP64, allocating nothing. Its per-cell scratch is a fixed
 * device array of PFEM2_NOALLOC_MAX_CELLS cells held by every GPU that loads
 * the library; larger meshes are rejected with PFEM2_INVALID_ARG. A call on
 * a stream that is not being captured looks the array's device address up
 * (the first call on a device must come before any stream capture, which
 * then reuses the address; PFEM2_BAD_STATE otherwise); calls that overlap on
 * the GPU race on the shared array.
 *   vertex_cell_ptr [n_vertices+1], vertex_cell / vertex_cell_local: cells
 *   around each vertex (ascending) and the vertex's local index there, each
 *   in [0, n_cells) / [0, 2^dim) (a vertex with an entry out of range gets
 *   NaN in node_u and node_w, nothing else is read for it);
 *   cell_start [n_cells+1]: particle offsets (non-decreasing, within xi and
 *   u), particles sorted by cell; xi, u [n_particles][dim];
 *   zero_flag [n_vertices] or NULL: vertices whose velocity is set to 0 after
 *   the projection (the wall DoFs of pfem2_case.zero_after_projection_mask,
 *   TurekBenchmarkCuda/pfem2particle.cu:866-869; NULL zeroes none);
 *   out node_u [n_vertices][dim], node_w [n_vertices] (node_u = 0 where
 *   node_w = 0); stream: a cudaStream_t or NULL. */
#define PFEM2_NOALLOC_MAX_CELLS 65536
pfem2_status pfem2_project_noalloc(int32_t dim, int32_t n_cells, int32_t n_vertices,
                                   const int32_t* vertex_cell_ptr, const int32_t* vertex_cell,
                                   const int32_t* vertex_cell_local, const int32_t* cell_start,
                                   const double* xi, const double* u, const uint8_t* zero_flag,
                                   double* node_u, double* node_w, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* PFEM2_H */
