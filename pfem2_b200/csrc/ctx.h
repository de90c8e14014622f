// ctx.h -- host-side context of libpfem2b: device buffers of a batch of
// PFEM2 instances and the launchers shared by the .cu translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/pfem2.h"

namespace pfem2 {

constexpr int kSlice = 32;          // SELL slice height (rows per warp)
constexpr int kMaxPatch = 32;       // max cells around a vertex
constexpr int kMaxRing = 64;        // max cells sharing a vertex with a cell
constexpr int kNumSys = 7;          // pred x,y,z, pressure, mass x,y,z
constexpr int kFarMax = 16384;      // far-mover list capacity (sorted in 128 KB of shared memory)

// Per-instance parameters visible to kernels.
struct DevInst {
  double mu, rho, dt, open_flux;
  double dt_sub;  // dt / PARTICLES_MOVEMENT_STEPS
  unsigned open_mask;
  int q[3];
  double h[3];  // sub-cell widths 1.0 / q of check_cell_for_empty_parts
  unsigned long long qm[3];  // ceil(2^32 / q): t / q = (t * qm) >> 32 exactly for t, q < 2^16
  int max_per_part;
  int v_off, nv_pad, c_off, nc;
};

struct HostInst {
  int nv = 0, nc = 0;
  int v_off = 0, nv_pad = 0, c_off = 0;
  pfem2_case cs{};
  unsigned q[3] = {0, 0, 0};
  std::vector<double> X;
  std::vector<int> cells, fb;
};

// Krylov tile: a run of SELL slices of one system.
struct Tile {
  int sys;        // system id inside the phase
  int comp;       // component slot (vector block)
  int s0, s1;     // slice range
  int slot;       // partial-sum slot (the slots of a system are contiguous)
  int lk;         // index of the system among the systems of the tile's block
};

struct Ctx {
  pfem2_config cfg{};
  int dim = 2;
  // FP32 stages (pfem2_config.fp32_stages of a mixed context): particle
  // state and kernels, prediction/correction right-hand sides, pressure
  // right-hand side, inner Krylov iterations
  bool pmixed = false, amixed = false, prmixed = false, kmixed = false;
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  std::vector<HostInst> inst;
  bool setup_done = false;
  bool seeded = false;
  double time = 0.0;
  int timestep = 1;
  long long launches = 0;

  // sizes (nv includes per-instance padding to a multiple of kSlice)
  int nv = 0, nc = 0, ninc = 0, nnz = 0, nslices = 0, nell = 0;

  // mesh
  double* X = nullptr;
  int* cv = nullptr;
  signed char* fb = nullptr;
  int* cell_inst = nullptr;
  int* vert_inst = nullptr;
  int* v2c_ptr = nullptr;
  int* v2c_cell = nullptr;
  unsigned char* v2c_loc = nullptr;
  double* v2c_dir = nullptr;
  void* v2c_dir_r = nullptr;  // Real copy for the particle kernels
  void* cell_geo = nullptr;   // [nc] CellGeo<dim, Real>: local frame, inverse Jacobian, affine flag
  int* ring_ptr = nullptr;
  int* ring_cell = nullptr;
  int* ring_rev = nullptr;       // [ring entry (c, k)] position of c in the ring of ring_cell[k]
  unsigned* dest_mask = nullptr; // [nc] per old cell: ring positions that received movers (reset per advection)
  DevInst* d_inst = nullptr;
  std::vector<DevInst> h_inst;

  // loads: boundary faces of a patch (global cell * faces-per-cell + face),
  // built on first use per (instance, patch)
  struct LoadFaces {
    int inst, patch, n;
    int* d;
  };
  std::vector<LoadFaces> load_faces;
  double* loads_dev = nullptr;   // [7 * instances]: 5 load sums, then the two probe pressures
  double* loads_host = nullptr;  // pinned copy of loads_dev

  // sparsity: CSR (setup, tests) and SELL-32 (solvers)
  int* rp = nullptr;
  int* ci = nullptr;
  int* inc_slot = nullptr;  // [ninc][NV] -> SELL entry index
  int* sl_ptr = nullptr;    // [nslices+1] entry offset of each slice
  int* sl_len = nullptr;    // [nslices] entries per row in the slice
  int* sl_col = nullptr;    // [nell] column (padding: the row itself with value 0)
  std::vector<int> h_sl_ptr;

  // matrices in SELL layout (values only), FP64 master + FP32 copy
  double* A64[kNumSys] = {};
  float* A32[kNumSys] = {};
  double* dinv64[kNumSys] = {};
  float* dinv32[kNumSys] = {};

  // Dirichlet tables: fields 0..2 velocity, 3 pressure
  unsigned char* isdir[4] = {};
  double* dirval[4] = {};
  double* shift[4] = {};
  unsigned char* zero_flag = nullptr;
  // wall push-back: projected values of the zero-flag vertices before they
  // are zeroed ([dim][nv]) and the cells touching such vertices in
  // instances with wall_pushback (ascending)
  double* wall_dv = nullptr;
  int* wall_cells = nullptr;
  int n_wall_cells = 0;

  // nodal fields (FP64 masters) and Real mirrors for particle kernels
  double* F[PFEM2_N_FIELDS] = {};
  double* corr[3] = {};
  double* rhs[3] = {};
  void* Vr = nullptr;   // [dim][nv] Real
  void* dVr = nullptr;  // [dim][nv] Real, V - V_old

  // particles (SoA, double buffered)
  int pcap = 0;
  int* pcell[2] = {};
  void* pxi[2] = {};
  void* pu[2] = {};
  int cur = 0;
  int* newcell = nullptr;
  // particle capacity from which the advection runs in two phases per warp
  // (stayers, then the warp's queued leavers; measured faster than the
  // one-pass kernel on every bench workload, the smallest 1.3M particles);
  // the environment variable PFEM2_ADVECT_SPLIT_MIN overrides it at creation
  long long adv_split_min = 0;
  int* cell_start[2] = {};
  unsigned long long* rebin_tiles = nullptr;  // ticket + status words of the rebin's single-pass scan
  int* d_np = nullptr;       // [2] particle count of buffer 0/1
  int far_cap = 0;
  unsigned long long* far_keys = nullptr;
  int* d_counters = nullptr;  // see enum Counter
  void* partial = nullptr;    // [nc][NV][dim+1] Real projection partials

  int ring_max = 0;
  int list_cap = 0;           // per-cell incoming particle capacity in the rebin pass
  int nbucket_max = 0;

  // Krylov workspace
  void* kws = nullptr;
  size_t kws_bytes = 0;
  Tile* d_tiles[2] = {};      // [0] 1 component phase, [1] dim component phase
  int ntiles[2] = {};
  int tile_slices = 0;         // Krylov tile size in slices (0 = automatic)
  double* sys_scalars = nullptr;
  double* tile_part = nullptr;
  int* d_sysinfo = nullptr;
  unsigned* barrier = nullptr;   // count, gen
  int* d_err = nullptr;         // abort flag of the running solve (reset per launch)
  int* d_err_sticky = nullptr;  // bits of the solves' exit codes since the host last read them
  // polls of a bounded device-side wait before it gives up (PFEM2_TIMEOUT);
  // the environment variable PFEM2_SPIN_LIMIT lowers it at creation (tests)
  unsigned spin_limit = 1u << 26;
  // a wait timed out: the device state is not trusted, stepping calls
  // return PFEM2_BAD_STATE until the context is destroyed
  bool failed = false;
  int coop_blocks = 0;
  int solve_threads = 256;
  int solve_blocks_per_sm = 1;  // persistent Krylov grid: blocks per SM
  long long mg_wide_min = 262144;  // rows from which one pressure system runs two blocks per SM
  // rows of the largest pressure system from which the restriction to
  // level 2 is a phase of its own (b2 = Pt1^T b1 after b1 is complete)
  // instead of the composite R02 in phase B: from every size, since the
  // composite's rows reach far beyond a block's own rows (on the 52k-row
  // channel 1,981 other rows per block against 381 own) and the extra phase
  // costs less (channel pressure solve 1.29 -> 1.15 ms, 64-instance batch
  // 27.0 -> 21.5 ms); PFEM2_MG_SPLIT_MIN overrides it at creation
  long long mg_split_min = 0;
  bool two_level = true;        // pressure: multigrid preconditioner (else Jacobi)
  bool vel_bicg = false;        // velocity systems solved by BiCGStab (else CG)
  bool p_bicg = false;          // pressure solved by BiCGStab with Jacobi (else CG with multigrid)
  double refine_eta = 1e-3;     // mixed: inner residual reduction per FP64 refinement

  // moving mesh (pfem2_config.moving_mesh): boundary vertices, the
  // elasticity blocks K[a * dim + b] on the SELL pattern, constraint table,
  // right-hand side / inverse diagonal ([dim][nv]), CG vectors, particle
  // positions before a move ([dim][pcap] FP64), reinterpolated fields, and
  // the device status word of the mesh kernels (1: a cell turned inside out)
  bool moving = false;
  unsigned char* ale_bnd = nullptr;
  double* ale_K[9] = {};
  unsigned char* ale_fix = nullptr;
  double* ale_g = nullptr;
  double* ale_rhs = nullptr;
  double* ale_dinv = nullptr;
  double* ale_vec = nullptr;   // x, r, z, q, p[2]: 6 [dim][nv] blocks
  double* ale_part = nullptr;  // [2][grid][4] partial sums of the CG
  int* ale_out = nullptr;      // [2] iterations, converged; ale_res: residual and tolerance
  double* ale_res = nullptr;
  double* ale_xphys = nullptr;
  size_t ale_xphys_cap = 0;
  double* ale_new = nullptr;   // [4][nv]
  int* ale_flag = nullptr;
  int ale_grid = 0;

  // launch shapes: as set by the caller (0 = automatic) and as resolved at
  // setup (caller, else the tuning cache, else by size)
  pfem2_tuning tune_req{};
  pfem2_tuning tune{};
  std::string tune_source = "size";  // "caller", "cache" or "size" (per field: the first that set it)
  std::string device_name;

  // graph
  cudaGraphExec_t graph = nullptr;
  bool graph_valid = false;
  bool timing = false;
  cudaEvent_t ev[8] = {};
  double stage_ms[PFEM2_N_STAGES] = {};
  bool ev_pending = false;

  pfem2_stats stats{};
};

// device counters of the particle passes: statistics of the last pass
// (reset at every advection), then error flags that stay set until the
// host reads them (check_counters), so that a failure inside a run of
// graph-launched steps is still reported
enum Counter {
  CNT_DELETED = 0,
  CNT_REMOVED = 1,
  CNT_RESEEDED = 2,
  CNT_FAR = 3,
  CNT_ZERO_WEIGHT = 4,
  CNT_N_STATS = 5,
  CNT_LIST_OVERFLOW = 5,
  CNT_CAP_OVERFLOW = 6,
  CNT_FAR_OVERFLOW = 7,
  CNT_SCAN_TIMEOUT = 8,
  CNT_N = 9
};

// error reporting
void set_error(const std::string& s);
pfem2_status cuda_status(cudaError_t e, const char* where);
#define PFEM2_CUDA(call)                                              \
  do {                                                                \
    cudaError_t e_ = (call);                                          \
    if (e_ != cudaSuccess) return ::pfem2::cuda_status(e_, #call);    \
  } while (0)

#define PFEM2_TRY(x)                         \
  do {                                       \
    pfem2_status s_ = (x);                   \
    if (s_ != PFEM2_OK) return s_;           \
  } while (0)

inline int grid_for(const Ctx& c, long long n, int threads, int per_sm = 8) {
  long long b = (n + threads - 1) / threads;
  long long cap = (long long)c.num_sms * per_sm;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

// launchers (particles.cu)
pfem2_status launch_seed(Ctx& c, int instance, const uint32_t q[3], uint64_t seed, double jitter);
pfem2_status launch_correct(Ctx& c);
pfem2_status launch_advect(Ctx& c, bool fuse_correct);
pfem2_status launch_rebin(Ctx& c, bool do_check, bool fuse_project, bool from_advect);
pfem2_status launch_project(Ctx& c, bool partials_ready);
pfem2_status launch_sync_real_fields(Ctx& c);
pfem2_status launch_set_particles(Ctx& c, const int* counts, const int* cell, const double* xi, const double* u);
pfem2_status read_particles(Ctx& c, int instance, int* cell, double* xi, double* u, int* n);

// fem.cu
pfem2_status assemble_matrices(Ctx& c);
pfem2_status launch_rhs_prediction(Ctx& c);
pfem2_status launch_rhs_pressure(Ctx& c);
pfem2_status launch_rhs_correction(Ctx& c);
pfem2_status launch_finish_fem(Ctx& c);
pfem2_status launch_restore_frozen(Ctx& c);
pfem2_status launch_loads(Ctx& c, int instance, int patch, double* out_dev);
pfem2_status launch_vorticity(Ctx& c);

// ale.cu (moving mesh)
pfem2_status ale_setup(Ctx& c);
pfem2_status ale_elasticity(Ctx& c, const pfem2_elasticity& e, const double* body_disp, int* iters, double* res);
pfem2_status ale_move_mesh(Ctx& c);
void ale_free(Ctx& c);
// particles.cu: positions before the mesh moves, relocation after it
pfem2_status launch_particle_positions(Ctx& c, double* xphys);
pfem2_status launch_relocate(Ctx& c, const double* xphys);
pfem2_status launch_cell_geo(Ctx& c, int* flag);
pfem2_status far_sort_setup(Ctx& c);

// krylov.cu
pfem2_status krylov_setup(Ctx& c);
pfem2_status krylov_setup_precond(Ctx& c);
void krylov_free(Ctx& c);
// which: 0 prediction (dim systems per instance), 1 pressure, 2 correction
pfem2_status krylov_solve(Ctx& c, int which);
pfem2_status krylov_read_stats(Ctx& c);
void krylov_sizes(Ctx& c, long long* out12);

}  // namespace pfem2
