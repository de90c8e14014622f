// capi.cu -- the C ABI of libpfem2b (include/pfem2.h): context, mesh
// preprocessing (setup_system / initialize_maps), the pfem2Solver member
// functions and the whole-step path with its CUDA graphs.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "common.cuh"
#include "ctx.h"

namespace pfem2 {

static thread_local std::string g_last_error;

void set_error(const std::string& s) { g_last_error = s; }

pfem2_status cuda_status(cudaError_t e, const char* where) {
  set_error(std::string(where) + ": " + cudaGetErrorString(e));
  return PFEM2_CUDA_ERROR;
}

template <typename T>
static pfem2_status dalloc(T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * n);
  if (e != cudaSuccess) return cuda_status(e, "cudaMalloc");
  e = cudaMemset(*p, 0, sizeof(T) * n);
  if (e != cudaSuccess) return cuda_status(e, "cudaMemset");
  return PFEM2_OK;
}

template <typename T>
static pfem2_status upload(T** p, const std::vector<T>& v) {
  pfem2_status s = dalloc(p, v.size());
  if (s != PFEM2_OK) return s;
  if (!v.empty()) PFEM2_CUDA(cudaMemcpy(*p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return PFEM2_OK;
}



// host pinned mirror of the step counters (deferred error reporting)
struct StepMirror {
  int counters[CNT_N];
  int np[2];
};

static double bc_value(const pfem2_dirichlet& d, const double* x) {
  if (d.kind == PFEM2_BC_PARABOLA) {
    const double s = x[d.axis], L = d.b - d.a;
    return d.value * 4.0 * (s - d.a) * (d.b - s) / (L * L);
  }
  return d.value;
}

// per-cell geometry records of the particle kernels (FP64 math, stored in R)
template <int DIM, typename R>
static pfem2_status upload_cell_geo(Ctx& c, const std::vector<double>& X, const std::vector<int>& cv) {
  constexpr int NV = 1 << DIM;
  std::vector<CellGeo<DIM, R>> geo(c.nc);
  for (int ce = 0; ce < c.nc; ++ce) {
    CellGeo<DIM, R>& g = geo[ce];
    double D[NV][DIM];
    const int g0 = cv[(size_t)ce * NV];
    for (int a = 0; a < DIM; ++a) g.x0[a] = X[(size_t)g0 * DIM + a];
    double scale = 0.0;
    for (int v = 0; v < NV; ++v)
      for (int a = 0; a < DIM; ++a) {
        D[v][a] = X[(size_t)cv[(size_t)ce * NV + v] * DIM + a] - g.x0[a];
        scale = std::max(scale, std::fabs(D[v][a]));
        if (v > 0) g.D[v - 1][a] = (R)D[v][a];
      }
    // Jacobian at the centre: dx_a/dxi_b = sum_v D_v,a dN_v/dxi_b (xi = 1/2)
    double J[DIM * DIM] = {};
    for (int v = 0; v < NV; ++v)
      for (int b = 0; b < DIM; ++b) {
        const double sgn = ((v >> b) & 1) ? 1.0 : -1.0;
        const double w = sgn * std::pow(0.5, DIM - 1);
        for (int a = 0; a < DIM; ++a) J[a * DIM + b] += D[v][a] * w;
      }
    double Ji[DIM * DIM];
    double det;
    if (DIM == 2) {
      det = J[0] * J[3] - J[1] * J[2];
      Ji[0] = J[3] / det; Ji[1] = -J[1] / det; Ji[2] = -J[2] / det; Ji[3] = J[0] / det;
    } else {
      const double a = J[0], b = J[1], cc = J[2], d = J[3], e = J[4], f = J[5], gg = J[6], h = J[7], i = J[8];
      const double A = e * i - f * h, B = -(d * i - f * gg), Cc = d * h - e * gg;
      det = a * A + b * B + cc * Cc;
      Ji[0] = A / det; Ji[1] = -(b * i - cc * h) / det; Ji[2] = (b * f - cc * e) / det;
      Ji[3] = B / det; Ji[4] = (a * i - cc * gg) / det; Ji[5] = -(a * f - cc * d) / det;
      Ji[6] = Cc / det; Ji[7] = -(a * h - b * gg) / det; Ji[8] = (a * e - b * d) / det;
    }
    if (!(det > 0.0)) {
      set_error("mesh: a cell has a non-positive Jacobian");
      return PFEM2_MESH_ERROR;
    }
    for (int k = 0; k < DIM * DIM; ++k) g.Ji[k] = (R)Ji[k];
    // affine: every vertex offset is the sum of the edge offsets of its bits
    bool aff = true;
    for (int v = 0; v < NV && aff; ++v)
      for (int a = 0; a < DIM; ++a) {
        double s = 0.0;
        for (int b = 0; b < DIM; ++b)
          if ((v >> b) & 1) s += D[1 << b][a];
        if (std::fabs(D[v][a] - s) > 1e-13 * scale) { aff = false; break; }
      }
    g.affine = aff ? 1 : 0;
  }
  CellGeo<DIM, R>* dptr = nullptr;
  const pfem2_status st = upload(&dptr, geo);
  if (st != PFEM2_OK) return st;
  c.cell_geo = dptr;
  return PFEM2_OK;
}

// ------------------------------------------------------- launch shapes
// key of the tuning cache: device name (spaces as '_'), dim, FP32 stages
// (-1 for an FP64 context), floor(log2(cells)), floor(log2(instances))
static std::string tuning_key(const Ctx& c) {
  long long cells = 0;
  for (const auto& in : c.inst) cells += in.nc;
  int lc = 0, li = 0;
  while ((2LL << lc) <= cells) ++lc;
  while ((2LL << li) <= (long long)c.inst.size()) ++li;
  const int stages = c.cfg.precision == PFEM2_PREC_FP64
                         ? -1
                         : (c.cfg.fp32_stages ? c.cfg.fp32_stages : PFEM2_FP32_DEFAULT);
  std::string name = c.device_name;
  for (char& ch : name)
    if (ch == ' ' || ch == '\t') ch = '_';
  char buf[256];
  snprintf(buf, sizeof(buf), "%s %d %d %d %d", name.c_str(), c.dim, stages, lc, li);
  return buf;
}

// The tuning cache (PFEM2_TUNING_CACHE): one entry per line,
//   <device> <dim> <stages> <log2 cells> <log2 instances>
//   <advect bps> <advect split> <rebin bps> <vel tile slices> <p bps> [<vel bps>] [ms per step]
// (the launch-shape values are integers, the time has a decimal point; a
// missing value is automatic). '#' starts a comment; the last entry with
// this context's key wins. Its values fill the fields the caller left at 0.
constexpr int kTuneVals = 6;

static void apply_tuning_cache(Ctx& c) {
  c.tune = c.tune_req;
  c.tune_source = "caller";
  const char* path = getenv("PFEM2_TUNING_CACHE");
  if (!path || !*path) return;
  FILE* f = fopen(path, "r");
  if (!f) return;
  const std::string key = tuning_key(c);
  char line[512];
  int best[kTuneVals] = {};
  bool found = false;
  while (fgets(line, sizeof(line), f)) {
    if (line[0] == '#') continue;
    std::vector<std::string> tok;
    char* save = nullptr;
    for (char* t = strtok_r(line, " \t\r\n", &save); t; t = strtok_r(nullptr, " \t\r\n", &save))
      tok.emplace_back(t);
    if (tok.size() < 5 + 5) continue;
    const std::string k = tok[0] + " " + tok[1] + " " + tok[2] + " " + tok[3] + " " + tok[4];
    if (key != k) continue;
    int v[kTuneVals] = {};
    bool ok = true;
    int nv = 0;
    for (size_t q = 5; q < tok.size() && nv < kTuneVals; ++q) {
      if (tok[q].find('.') != std::string::npos) break;  // the time
      char* end = nullptr;
      const long x = strtol(tok[q].c_str(), &end, 10);
      if (!end || *end) {
        ok = false;
        break;
      }
      v[nv++] = (int)x;
    }
    if (!ok || nv < 5) continue;
    std::copy(v, v + kTuneVals, best);
    found = true;
  }
  fclose(f);
  if (!found) return;
  int32_t* dst[kTuneVals] = {&c.tune.advect_blocks_per_sm, &c.tune.advect_split, &c.tune.rebin_blocks_per_sm,
                             &c.tune.vel_tile_slices, &c.tune.p_blocks_per_sm, &c.tune.vel_blocks_per_sm};
  for (int i = 0; i < kTuneVals; ++i)
    if (*dst[i] == 0 && best[i] > 0) *dst[i] = best[i];
  c.tune_source = "cache";
}

static pfem2_status check_tuning(const pfem2_tuning& t) {
  if (t.advect_blocks_per_sm < 0 || t.advect_blocks_per_sm > 32 || t.advect_split < 0 || t.advect_split > 2 ||
      t.rebin_blocks_per_sm < 0 || t.rebin_blocks_per_sm > 32 || t.vel_tile_slices < 0 || t.vel_tile_slices > 4096 ||
      t.p_blocks_per_sm < 0 || t.p_blocks_per_sm > 2 || t.vel_blocks_per_sm < 0 || t.vel_blocks_per_sm > 2) {
    set_error("tuning: a field is out of range");
    return PFEM2_INVALID_ARG;
  }
  return PFEM2_OK;
}

// --------------------------------------------------------------- setup
static pfem2_status do_setup(Ctx& c) {
  apply_tuning_cache(c);
  if (!c.tune.advect_blocks_per_sm) c.tune.advect_blocks_per_sm = 16;
  if (!c.tune.rebin_blocks_per_sm) c.tune.rebin_blocks_per_sm = 8;
  const int dim = c.dim, NV = 1 << dim, NF = 2 * dim;
  // offsets
  int v = 0, cc = 0;
  for (auto& in : c.inst) {
    in.v_off = v;
    in.nv_pad = (in.nv + kSlice - 1) / kSlice * kSlice;
    in.c_off = cc;
    v += in.nv_pad;
    cc += in.nc;
  }
  c.nv = v;
  c.nc = cc;
  const int nv = c.nv, nc = c.nc;
  std::vector<double> X((size_t)nv * dim, 0.0);
  std::vector<int> cv((size_t)nc * NV), cinst(nc), vinst(nv, 0);
  std::vector<signed char> fb((size_t)nc * NF);
  for (size_t i = 0; i < c.inst.size(); ++i) {
    auto& in = c.inst[i];
    std::copy(in.X.begin(), in.X.end(), X.begin() + (size_t)in.v_off * dim);
    for (int k = 0; k < in.nv_pad; ++k) vinst[in.v_off + k] = (int)i;
    for (int k = 0; k < in.nc; ++k) {
      cinst[in.c_off + k] = (int)i;
      for (int b = 0; b < NV; ++b) {
        int g = in.cells[(size_t)k * NV + b];
        if (g < 0 || g >= in.nv) {
          set_error("mesh: vertex index out of range");
          return PFEM2_MESH_ERROR;
        }
        cv[(size_t)(in.c_off + k) * NV + b] = g + in.v_off;
      }
      for (int f = 0; f < NF; ++f) {
        int b = in.fb[(size_t)k * NF + f];
        if (b < -1 || b > 127) {
          set_error("mesh: boundary id must be in [-1, 127]");
          return PFEM2_MESH_ERROR;
        }
        fb[(size_t)(in.c_off + k) * NF + f] = (signed char)b;
      }
    }
  }
  // vertex -> cells (ascending cell index), local index, centre directions
  std::vector<int> v2c_ptr(nv + 1, 0);
  for (int k = 0; k < nc * NV; ++k) v2c_ptr[cv[k] + 1]++;
  for (int i = 0; i < nv; ++i) v2c_ptr[i + 1] += v2c_ptr[i];
  c.ninc = v2c_ptr[nv];
  std::vector<int> v2c_cell(c.ninc), fill(nv, 0);
  std::vector<unsigned char> v2c_loc(c.ninc);
  for (int ce = 0; ce < nc; ++ce)
    for (int b = 0; b < NV; ++b) {
      int g = cv[(size_t)ce * NV + b];
      int k = v2c_ptr[g] + fill[g]++;
      v2c_cell[k] = ce;
      v2c_loc[k] = (unsigned char)b;
    }
  for (int i = 0; i < nv; ++i)
    if (v2c_ptr[i + 1] - v2c_ptr[i] > kMaxPatch) {
      set_error("mesh: more than 32 cells around a vertex");
      return PFEM2_MESH_ERROR;
    }
  std::vector<double> v2c_dir((size_t)c.ninc * dim);
  std::vector<float> v2c_dirf((size_t)c.ninc * dim);
  for (int i = 0; i < nv; ++i)
    for (int k = v2c_ptr[i]; k < v2c_ptr[i + 1]; ++k) {
      int ce = v2c_cell[k];
      double ctr[3] = {0, 0, 0}, nn = 0;
      for (int b = 0; b < NV; ++b)
        for (int a = 0; a < dim; ++a) ctr[a] += X[(size_t)cv[(size_t)ce * NV + b] * dim + a];
      for (int a = 0; a < dim; ++a) {
        ctr[a] = ctr[a] / NV - X[(size_t)i * dim + a];
        nn += ctr[a] * ctr[a];
      }
      nn = std::sqrt(nn);
      for (int a = 0; a < dim; ++a) {
        v2c_dir[(size_t)k * dim + a] = ctr[a] / nn;
        v2c_dirf[(size_t)k * dim + a] = (float)(ctr[a] / nn);
      }
    }
  // 1-ring of each cell (cells sharing a vertex), ascending
  std::vector<int> ring_ptr(nc + 1, 0), ring_cell;
  ring_cell.reserve((size_t)nc * (dim == 2 ? 9 : 27));
  std::vector<int> tmp;
  c.ring_max = 0;
  for (int ce = 0; ce < nc; ++ce) {
    tmp.clear();
    for (int b = 0; b < NV; ++b) {
      int g = cv[(size_t)ce * NV + b];
      for (int k = v2c_ptr[g]; k < v2c_ptr[g + 1]; ++k) tmp.push_back(v2c_cell[k]);
    }
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    ring_cell.insert(ring_cell.end(), tmp.begin(), tmp.end());
    ring_ptr[ce + 1] = (int)ring_cell.size();
    c.ring_max = std::max(c.ring_max, (int)tmp.size());
  }
  // sparsity: per row diagonal first, then ascending columns; SELL-32
  // (not needed without FEM)
  std::vector<std::vector<int>> rows(c.cfg.particles_only ? 0 : nv);
  int maxlen = 1;
  for (int i = 0; i < (int)rows.size(); ++i) {
    tmp.clear();
    for (int k = v2c_ptr[i]; k < v2c_ptr[i + 1]; ++k)
      for (int b = 0; b < NV; ++b) tmp.push_back(cv[(size_t)v2c_cell[k] * NV + b]);
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    auto& r = rows[i];
    r.push_back(i);
    for (int j : tmp)
      if (j != i) r.push_back(j);
    maxlen = std::max(maxlen, (int)r.size());
  }
  c.nslices = c.cfg.particles_only ? 0 : nv / kSlice;
  std::vector<int> sl_ptr(c.nslices + 1, 0), sl_len(c.nslices);
  for (int s = 0; s < c.nslices; ++s) {
    int L = 1;
    for (int l = 0; l < kSlice; ++l) L = std::max(L, (int)rows[s * kSlice + l].size());
    sl_len[s] = L;
    sl_ptr[s + 1] = sl_ptr[s] + L * kSlice;
  }
  c.nell = sl_ptr[c.nslices];
  c.h_sl_ptr = sl_ptr;
  std::vector<int> sl_col(c.nell);
  std::vector<std::map<int, int>> where(0);
  c.nnz = 0;
  for (int s = 0; s < c.nslices; ++s)
    for (int l = 0; l < kSlice; ++l) {
      int row = s * kSlice + l;
      auto& r = rows[row];
      c.nnz += (int)r.size();
      for (int j = 0; j < sl_len[s]; ++j) sl_col[sl_ptr[s] + j * kSlice + l] = j < (int)r.size() ? r[j] : row;
    }
  std::vector<int> inc_slot(c.cfg.particles_only ? 0 : (size_t)c.ninc * NV);
  for (int i = 0; i < (int)rows.size(); ++i) {
    auto& r = rows[i];
    int s = i / kSlice, l = i % kSlice;
    for (int k = v2c_ptr[i]; k < v2c_ptr[i + 1]; ++k)
      for (int b = 0; b < NV; ++b) {
        int col = cv[(size_t)v2c_cell[k] * NV + b];
        int j = (int)(std::find(r.begin(), r.end(), col) - r.begin());
        inc_slot[(size_t)k * NV + b] = sl_ptr[s] + j * kSlice + l;
      }
  }
  // Dirichlet tables and zero-after-projection flags
  std::vector<unsigned char> isd[4];
  std::vector<double> dval[4];
  for (int f = 0; f < 4; ++f) {
    isd[f].assign(nv, 0);
    dval[f].assign(nv, 0.0);
  }
  std::vector<unsigned char> zflag(nv, 0);
  for (auto& in : c.inst) {
    for (int k = in.nv; k < in.nv_pad; ++k)
      for (int f = 0; f < 4; ++f) isd[f][in.v_off + k] = 1;
    for (int f = 0; f < 4; ++f) {
      if (f >= dim && f < 3) continue;
      for (int k = 0; k < in.cs.n_dirichlet[f]; ++k) {
        const pfem2_dirichlet& d = in.cs.dirichlet[f][k];
        for (int ce = in.c_off; ce < in.c_off + in.nc; ++ce)
          for (int fc = 0; fc < NF; ++fc) {
            if (fb[(size_t)ce * NF + fc] != d.boundary_id) continue;
            for (int b = 0; b < NV; ++b) {
              if (((b >> (fc / 2)) & 1) != fc % 2) continue;
              int g = cv[(size_t)ce * NV + b];
              isd[f][g] = 1;
              dval[f][g] = bc_value(d, &X[(size_t)g * dim]);
            }
          }
      }
    }
    if (in.cs.zero_after_projection_mask)
      for (int ce = in.c_off; ce < in.c_off + in.nc; ++ce)
        for (int fc = 0; fc < NF; ++fc) {
          int b = fb[(size_t)ce * NF + fc];
          if (b < 0 || b > 31 || !((in.cs.zero_after_projection_mask >> b) & 1u)) continue;
          for (int vb = 0; vb < NV; ++vb)
            if (((vb >> (fc / 2)) & 1) == fc % 2) zflag[cv[(size_t)ce * NV + vb]] = 1;
        }
  }
  // solver kinds: one per system kind for the whole batch
  for (auto& in : c.inst) {
    const pfem2_case& k0 = c.inst[0].cs;
    const bool okk = (in.cs.vel_solver == PFEM2_SOLVER_CG || in.cs.vel_solver == PFEM2_SOLVER_BICGSTAB) &&
                     (in.cs.p_solver == PFEM2_SOLVER_CG || in.cs.p_solver == PFEM2_SOLVER_BICGSTAB);
    if (!okk || in.cs.vel_solver != k0.vel_solver || in.cs.p_solver != k0.p_solver) {
      set_error("vel_solver / p_solver: PFEM2_SOLVER_CG or PFEM2_SOLVER_BICGSTAB, the same in every instance");
      return PFEM2_INVALID_ARG;
    }
    if (!(in.cs.vel_rtol >= 0.0) || !(in.cs.p_rtol >= 0.0) || !(in.cs.vel_tol >= 0.0) || !(in.cs.p_tol >= 0.0)) {
      set_error("solver tolerances must be >= 0");
      return PFEM2_INVALID_ARG;
    }
  }
  c.vel_bicg = c.inst[0].cs.vel_solver == PFEM2_SOLVER_BICGSTAB;
  c.p_bicg = c.inst[0].cs.p_solver == PFEM2_SOLVER_BICGSTAB;
  if (c.p_bicg) c.two_level = false;
  if (c.moving) {
    // the matrices follow the mesh: reassembled every step; the multigrid
    // hierarchy (built once on the host) is not used
    if (c.inst.size() != 1 || c.dim != 2 || c.cfg.particles_only) {
      set_error("moving_mesh: one 2D instance with the FEM");
      return PFEM2_INVALID_ARG;
    }
    c.two_level = false;
    c.inst[0].cs.reassemble_every_step = 1;
  }
  // instance table
  c.h_inst.resize(c.inst.size());
  std::vector<double> tols(4 * c.inst.size());
  std::vector<int> maxit(c.inst.size());
  for (size_t i = 0; i < c.inst.size(); ++i) {
    auto& in = c.inst[i];
    DevInst& d = c.h_inst[i];
    d.mu = in.cs.mu; d.rho = in.cs.rho; d.dt = in.cs.dt; d.open_flux = in.cs.open_boundary_pressure_flux;
    d.open_mask = in.cs.open_boundary_mask;
    d.q[0] = d.q[1] = d.q[2] = 1;
    d.h[0] = d.h[1] = d.h[2] = 1.0;
    d.qm[0] = d.qm[1] = d.qm[2] = 1ull << 32;
    d.max_per_part = c.cfg.max_particles_per_cell_part;
    d.dt_sub = in.cs.dt / c.cfg.movement_steps;
    d.v_off = in.v_off; d.nv_pad = in.nv_pad; d.c_off = in.c_off; d.nc = in.nc;
    const size_t ni = c.inst.size();
    tols[i] = in.cs.vel_tol;
    tols[ni + i] = in.cs.p_tol;
    tols[2 * ni + i] = in.cs.vel_rtol;
    tols[3 * ni + i] = in.cs.p_rtol;
    maxit[i] = in.cs.max_iter > 0 ? in.cs.max_iter : 10000;
  }
  // uploads
  PFEM2_TRY(upload(&c.X, X));
  PFEM2_TRY(upload(&c.cv, cv));
  PFEM2_TRY(upload(&c.fb, fb));
  PFEM2_TRY(upload(&c.cell_inst, cinst));
  PFEM2_TRY(upload(&c.vert_inst, vinst));
  PFEM2_TRY(upload(&c.v2c_ptr, v2c_ptr));
  PFEM2_TRY(upload(&c.v2c_cell, v2c_cell));
  PFEM2_TRY(upload(&c.v2c_loc, v2c_loc));
  PFEM2_TRY(upload(&c.v2c_dir, v2c_dir));
  if (c.pmixed) {
    float* p = nullptr;
    PFEM2_TRY(upload(&p, v2c_dirf));
    c.v2c_dir_r = p;
  } else {
    c.v2c_dir_r = c.v2c_dir;
  }
  if (dim == 2) PFEM2_TRY((c.pmixed ? upload_cell_geo<2, float>(c, X, cv) : upload_cell_geo<2, double>(c, X, cv)));
  else PFEM2_TRY((c.pmixed ? upload_cell_geo<3, float>(c, X, cv) : upload_cell_geo<3, double>(c, X, cv)));
  PFEM2_TRY(upload(&c.ring_ptr, ring_ptr));
  PFEM2_TRY(upload(&c.ring_cell, ring_cell));
  {
    // position of each cell in the rings of its ring cells (rings are
    // symmetric: s is in ring(c) iff c is in ring(s)); 32 and beyond share
    // the mask's all-ones code
    std::vector<int> rev(ring_cell.size(), 0);
    for (int ce = 0; ce < nc; ++ce)
      for (int k = ring_ptr[ce]; k < ring_ptr[ce + 1]; ++k) {
        const int s = ring_cell[k];
        const int* b = ring_cell.data() + ring_ptr[s];
        const int* e = ring_cell.data() + ring_ptr[s + 1];
        const int* it = std::lower_bound(b, e, ce);
        rev[k] = (it != e && *it == ce) ? (int)(it - b) : 32;
      }
    PFEM2_TRY(upload(&c.ring_rev, rev));
    PFEM2_TRY(dalloc(&c.dest_mask, (size_t)nc));
  }
  PFEM2_TRY(upload(&c.sl_ptr, sl_ptr));
  PFEM2_TRY(upload(&c.sl_len, sl_len));
  PFEM2_TRY(upload(&c.sl_col, sl_col));
  PFEM2_TRY(upload(&c.inc_slot, inc_slot));
  for (int f = 0; f < 4; ++f) {
    PFEM2_TRY(upload(&c.isdir[f], isd[f]));
    PFEM2_TRY(upload(&c.dirval[f], dval[f]));
    PFEM2_TRY(dalloc(&c.shift[f], nv));
  }
  PFEM2_TRY(upload(&c.zero_flag, zflag));
  {
    // cells that the wall push-back visits
    std::vector<int> wc;
    for (auto& in : c.inst)
      if (in.cs.wall_pushback)
        for (int ce = in.c_off; ce < in.c_off + in.nc; ++ce) {
          bool touch = false;
          for (int b = 0; b < NV; ++b) touch |= zflag[cv[(size_t)ce * NV + b]] != 0;
          if (touch) wc.push_back(ce);
        }
    c.n_wall_cells = (int)wc.size();
    if (!wc.empty()) {
      PFEM2_TRY(upload(&c.wall_cells, wc));
      PFEM2_TRY(dalloc(&c.wall_dv, (size_t)dim * nv));
    }
  }
  PFEM2_TRY(upload(&c.d_inst, c.h_inst));
  {
    double* t = nullptr;
    PFEM2_TRY(upload(&t, tols));
    c.sys_scalars = t;
    PFEM2_TRY(upload(&c.d_sysinfo, maxit));
  }
  for (int k = 0; k < kNumSys && !c.cfg.particles_only; ++k) {
    PFEM2_TRY(dalloc(&c.A64[k], c.nell));
    PFEM2_TRY(dalloc(&c.A32[k], c.nell));
    PFEM2_TRY(dalloc(&c.dinv64[k], nv));
    PFEM2_TRY(dalloc(&c.dinv32[k], nv));
  }
  for (int f = 0; f < PFEM2_N_FIELDS; ++f) PFEM2_TRY(dalloc(&c.F[f], nv));
  for (int k = 0; k < 3; ++k) {
    PFEM2_TRY(dalloc(&c.corr[k], nv));
    PFEM2_TRY(dalloc(&c.rhs[k], nv));
  }
  const size_t rs = c.pmixed ? 4 : 8;
  {
    void* p;
    PFEM2_CUDA(cudaMalloc(&p, rs * 3 * nv));
    PFEM2_CUDA(cudaMemset(p, 0, rs * 3 * nv));
    c.Vr = p;
    PFEM2_CUDA(cudaMalloc(&p, rs * 3 * nv));
    PFEM2_CUDA(cudaMemset(p, 0, rs * 3 * nv));
    c.dVr = p;
    PFEM2_CUDA(cudaMalloc(&p, rs * (size_t)nc * NV * (dim + 1)));
    PFEM2_CUDA(cudaMemset(p, 0, rs * (size_t)nc * NV * (dim + 1)));
    c.partial = p;
  }
  for (int b = 0; b < 2; ++b) PFEM2_TRY(dalloc(&c.cell_start[b], nc + 1));
  PFEM2_TRY(dalloc(&c.rebin_tiles, (size_t)nc / 8 + 2));
  PFEM2_TRY(dalloc(&c.d_np, 2));
  PFEM2_TRY(dalloc(&c.d_counters, CNT_N));
  // far movers are sorted by one CTA in shared memory (8 B per key)
  c.far_cap = c.cfg.far_mover_capacity > 0 ? std::min(c.cfg.far_mover_capacity, kFarMax) : kFarMax;
  PFEM2_TRY(far_sort_setup(c));
  PFEM2_TRY(dalloc(&c.far_keys, c.far_cap));
  PFEM2_TRY(dalloc(&c.barrier, 2));
  PFEM2_TRY(dalloc(&c.d_err, 1));
  PFEM2_TRY(dalloc(&c.d_err_sticky, 1));
  PFEM2_TRY(dalloc(&c.loads_dev, 7 * c.inst.size()));
  PFEM2_CUDA(cudaMallocHost(&c.loads_host, sizeof(double) * 7 * c.inst.size()));
  c.list_cap = c.cfg.particles_per_cell_max > 0 ? c.cfg.particles_per_cell_max : (dim == 2 ? 512 : 1024);
  if (c.moving) PFEM2_TRY(ale_setup(c));
  if (!c.cfg.particles_only) {
    PFEM2_TRY(krylov_setup(c));
    PFEM2_TRY(assemble_matrices(c));
    PFEM2_CUDA(cudaStreamSynchronize(c.stream));
    PFEM2_TRY(krylov_setup_precond(c));
  }
  PFEM2_CUDA(cudaGetLastError());
  c.setup_done = true;
  return PFEM2_OK;
}

static pfem2_status alloc_particles(Ctx& c, size_t seeded) {
  double f = c.cfg.particle_capacity_factor > 0 ? c.cfg.particle_capacity_factor : 2.0;
  size_t cap = (size_t)std::ceil(seeded * f) + 1024;
  if (cap > (size_t)2000000000) cap = 2000000000;
  if ((int)cap <= c.pcap) return PFEM2_OK;
  const size_t rs = c.pmixed ? 4 : 8;
  for (int b = 0; b < 2; ++b) {
    if (c.pcell[b]) cudaFree(c.pcell[b]);
    if (c.pxi[b]) cudaFree(c.pxi[b]);
    if (c.pu[b]) cudaFree(c.pu[b]);
    PFEM2_CUDA(cudaMalloc(&c.pcell[b], sizeof(int) * cap));
    PFEM2_CUDA(cudaMalloc(&c.pxi[b], rs * c.dim * cap));
    PFEM2_CUDA(cudaMalloc(&c.pu[b], rs * c.dim * cap));
  }
  if (c.newcell) cudaFree(c.newcell);
  PFEM2_CUDA(cudaMalloc(&c.newcell, sizeof(int) * cap));
  c.pcap = (int)cap;
  c.graph_valid = false;
  return PFEM2_OK;
}

// deferred checks of the counters of the last particle pass
static pfem2_status check_counters(Ctx& c, bool sync) {
  if (sync) PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  int cnt[CNT_N];
  int np[2];
  PFEM2_CUDA(cudaMemcpy(cnt, c.d_counters, sizeof(cnt), cudaMemcpyDeviceToHost));
  PFEM2_CUDA(cudaMemcpy(np, c.d_np, sizeof(np), cudaMemcpyDeviceToHost));
  c.stats.n_particles = np[c.cur];
  c.stats.n_deleted_last_move = cnt[CNT_DELETED];
  c.stats.n_removed_last_check = cnt[CNT_REMOVED];
  c.stats.n_reseeded_last_check = cnt[CNT_RESEEDED];
  c.stats.n_far_movers_last_move = cnt[CNT_FAR];
  // the error flags are read once: clear them for the passes to come
  if (cnt[CNT_LIST_OVERFLOW] | cnt[CNT_CAP_OVERFLOW] | cnt[CNT_FAR_OVERFLOW] | cnt[CNT_SCAN_TIMEOUT])
    PFEM2_CUDA(cudaMemset(c.d_counters + CNT_N_STATS, 0, sizeof(int) * (CNT_N - CNT_N_STATS)));
  if (cnt[CNT_LIST_OVERFLOW]) {
    set_error("rebin: more incoming particles than the per-cell capacity (particles_per_cell_max)");
    return PFEM2_PARTICLE_OVERFLOW;
  }
  if (cnt[CNT_SCAN_TIMEOUT]) {
    set_error("rebin: a wait of the single-pass scan timed out");
    c.failed = true;
    return PFEM2_TIMEOUT;
  }
  if (cnt[CNT_FAR_OVERFLOW]) {
    set_error("advect: more far movers than far_mover_capacity");
    return PFEM2_PARTICLE_OVERFLOW;
  }
  if (np[c.cur] > c.pcap) {
    set_error("rebin: particle storage capacity exceeded");
    return PFEM2_PARTICLE_OVERFLOW;
  }
  return PFEM2_OK;
}

// ------------------------------------------------------------ FEM step
// stage boundary event; external so that it becomes a timing node when the
// step is being captured into a CUDA graph
static void mark(Ctx& c, int k) {
  if (c.timing) cudaEventRecordWithFlags(c.ev[k], c.stream, cudaEventRecordExternal);
}

static pfem2_status fem_step_launch(Ctx& c) {
  for (int d = 0; d < c.dim; ++d)
    PFEM2_CUDA(cudaMemcpyAsync(c.F[PFEM2_FIELD_OLD_VX + d], c.F[PFEM2_FIELD_VX + d], sizeof(double) * c.nv,
                               cudaMemcpyDeviceToDevice, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(c.F[PFEM2_FIELD_OLD_P], c.F[PFEM2_FIELD_P], sizeof(double) * c.nv,
                             cudaMemcpyDeviceToDevice, c.stream));
  if (c.inst[0].cs.reassemble_every_step) PFEM2_TRY(assemble_matrices(c));
  int nouter = std::max(1, c.inst[0].cs.outer_corrections);
  for (int oc = 0; oc < nouter; ++oc) {
    PFEM2_TRY(launch_rhs_prediction(c));
    PFEM2_TRY(krylov_solve(c, 0));
    if (oc == nouter - 1) mark(c, 4);
    PFEM2_TRY(launch_rhs_pressure(c));
    if (oc == nouter - 1) mark(c, 5);
    PFEM2_TRY(krylov_solve(c, 1));
    if (oc == nouter - 1) mark(c, 6);
    PFEM2_TRY(launch_rhs_correction(c));
    PFEM2_TRY(krylov_solve(c, 2));
    PFEM2_TRY(launch_finish_fem(c));
  }
  mark(c, 7);
  return PFEM2_OK;
}

static pfem2_status step_launch(Ctx& c) {
  mark(c, 0);
  PFEM2_TRY(launch_advect(c, true));
  mark(c, 1);
  PFEM2_TRY(launch_rebin(c, true, true, true));
  mark(c, 2);
  PFEM2_TRY(launch_project(c, true));
  mark(c, 3);
  if (c.cfg.particles_only) {
    PFEM2_TRY(launch_restore_frozen(c));
    for (int k = 4; k < 8; ++k) mark(c, k);
    return PFEM2_OK;
  }
  PFEM2_TRY(fem_step_launch(c));
  return PFEM2_OK;
}

// folds the events of the last timed step into stage_ms
static pfem2_status collect_stage_times(Ctx& c) {
  if (!c.ev_pending) return PFEM2_OK;
  PFEM2_CUDA(cudaEventSynchronize(c.ev[7]));
  for (int k = 0; k < PFEM2_N_STAGES; ++k) {
    float ms = 0.f;
    PFEM2_CUDA(cudaEventElapsedTime(&ms, c.ev[k], c.ev[k + 1]));
    c.stage_ms[k] += ms;
  }
  c.ev_pending = false;
  return PFEM2_OK;
}

}  // namespace pfem2

using namespace pfem2;

struct pfem2_ctx {
  Ctx c;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long long graph_launches[2] = {0, 0};
  bool graph_failed = false;
};

#define CTX_CHECK(ctx)                              \
  do {                                              \
    if (!(ctx)) {                                   \
      set_error("null context");                    \
      return PFEM2_INVALID_ARG;                     \
    }                                               \
  } while (0)
#define SETUP_CHECK(ctx)                            \
  do {                                              \
    CTX_CHECK(ctx);                                 \
    if (!(ctx)->c.setup_done) {                     \
      set_error("pfem2_setup has not run");         \
      return PFEM2_BAD_STATE;                       \
    }                                               \
  } while (0)
// a context whose device-side wait timed out refuses further stepping
#define LIVE_CHECK(ctx)                                                          \
  do {                                                                           \
    if ((ctx)->c.failed) {                                                       \
      set_error("a device-side wait of this context timed out: destroy it");   \
      return PFEM2_BAD_STATE;                                                    \
    }                                                                            \
  } while (0)
#define SEED_CHECK(ctx)                             \
  do {                                              \
    SETUP_CHECK(ctx);                               \
    LIVE_CHECK(ctx);                                \
    if (!(ctx)->c.seeded) {                         \
      set_error("no particles (seed first)");       \
      return PFEM2_BAD_STATE;                       \
    }                                               \
  } while (0)

extern "C" {

const char* pfem2_last_error(void) { return g_last_error.c_str(); }
int32_t pfem2_abi_version(void) { return PFEM2_ABI_VERSION; }

pfem2_status pfem2_create(const pfem2_config* cfg, pfem2_ctx** out) {
  if (!cfg || !out) { set_error("null argument"); return PFEM2_INVALID_ARG; }
  if (cfg->dim != 2 && cfg->dim != 3) { set_error("dim must be 2 or 3"); return PFEM2_INVALID_ARG; }
  if (cfg->movement_steps < 1 || cfg->max_particles_per_cell_part < 1) {
    set_error("movement_steps and max_particles_per_cell_part must be >= 1");
    return PFEM2_INVALID_ARG;
  }
  if (cfg->movement_steps > 65535) {
    set_error("movement_steps must be <= 65535");
    return PFEM2_INVALID_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device");
    return PFEM2_NO_DEVICE;
  }
  if (cfg->device < 0 || cfg->device >= ndev) { set_error("bad device ordinal"); return PFEM2_INVALID_ARG; }
  pfem2_ctx* x = new (std::nothrow) pfem2_ctx();
  if (!x) { set_error("out of host memory"); return PFEM2_INVALID_ARG; }
  Ctx& c = x->c;
  c.cfg = *cfg;
  c.dim = cfg->dim;
  if (cfg->precision == PFEM2_PREC_MIXED) {
    const int m = cfg->fp32_stages ? cfg->fp32_stages : PFEM2_FP32_DEFAULT;
    c.pmixed = (m & PFEM2_FP32_PARTICLES) != 0;
    c.amixed = (m & PFEM2_FP32_ASSEMBLY) != 0;
    c.prmixed = (m & PFEM2_FP32_PRESSURE_RHS) != 0;
    c.kmixed = (m & PFEM2_FP32_KRYLOV) != 0;
  }
  if (cfg->precision != PFEM2_PREC_FP64 && cfg->precision != PFEM2_PREC_MIXED) {
    set_error("precision must be PFEM2_PREC_FP64 or PFEM2_PREC_MIXED");
    return PFEM2_INVALID_ARG;
  }
  if (cfg->fp32_stages < 0 || cfg->fp32_stages > 15) {
    set_error("fp32_stages: a mask of PFEM2_FP32_* bits");
    return PFEM2_INVALID_ARG;
  }
  c.device = cfg->device;
  PFEM2_CUDA(cudaSetDevice(c.device));
  cudaDeviceProp prop;
  PFEM2_CUDA(cudaGetDeviceProperties(&prop, c.device));
  c.num_sms = prop.multiProcessorCount;
  c.device_name = prop.name;
  c.moving = cfg->moving_mesh != 0;
  if (const char* v = getenv("PFEM2_ADVECT_SPLIT_MIN")) c.adv_split_min = atoll(v);
  if (const char* v = getenv("PFEM2_MG_WIDE_MIN")) c.mg_wide_min = atoll(v);
  if (const char* v = getenv("PFEM2_MG_SPLIT_MIN")) c.mg_split_min = atoll(v);
  if (const char* v = getenv("PFEM2_SPIN_LIMIT")) c.spin_limit = (unsigned)std::min(atoll(v), (long long)c.spin_limit);
  PFEM2_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
  for (int k = 0; k < 8; ++k) PFEM2_CUDA(cudaEventCreate(&c.ev[k]));
  *out = x;
  return PFEM2_OK;
}

pfem2_status pfem2_destroy(pfem2_ctx* x) {
  if (!x) return PFEM2_OK;
  Ctx& c = x->c;
  cudaSetDevice(c.device);
  cudaStreamSynchronize(c.stream);
  for (int k = 0; k < 2; ++k)
    if (x->graph[k]) cudaGraphExecDestroy(x->graph[k]);
  krylov_free(c);
  ale_free(c);
  // device memory is released with the context's allocations; free the big ones
  void* ptrs[] = {c.cell_geo, c.X, c.cv, c.fb, c.cell_inst, c.vert_inst, c.v2c_ptr, c.v2c_cell, c.v2c_loc, c.v2c_dir,
                  c.ring_ptr, c.ring_cell, c.sl_ptr, c.sl_len, c.sl_col, c.inc_slot, c.zero_flag, c.wall_dv,
                  c.wall_cells, c.ring_rev, c.dest_mask, c.d_inst,
                  c.sys_scalars, c.d_sysinfo, c.Vr, c.dVr, c.partial, c.rebin_tiles, c.d_np, c.d_counters,
                  c.far_keys, c.barrier, c.d_err, c.d_err_sticky, c.newcell};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c.pmixed && c.v2c_dir_r) cudaFree(c.v2c_dir_r);
  for (int k = 0; k < kNumSys; ++k) {
    cudaFree(c.A64[k]); cudaFree(c.A32[k]); cudaFree(c.dinv64[k]); cudaFree(c.dinv32[k]);
  }
  for (int f = 0; f < 4; ++f) { cudaFree(c.isdir[f]); cudaFree(c.dirval[f]); cudaFree(c.shift[f]); }
  for (int f = 0; f < PFEM2_N_FIELDS; ++f) cudaFree(c.F[f]);
  for (int k = 0; k < 3; ++k) { cudaFree(c.corr[k]); cudaFree(c.rhs[k]); }
  for (int b = 0; b < 2; ++b) {
    cudaFree(c.pcell[b]); cudaFree(c.pxi[b]); cudaFree(c.pu[b]); cudaFree(c.cell_start[b]);
  }
  for (int k = 0; k < 8; ++k) cudaEventDestroy(c.ev[k]);
  for (const Ctx::LoadFaces& e : c.load_faces) cudaFree(e.d);
  cudaFree(c.loads_dev);
  cudaFreeHost(c.loads_host);
  cudaStreamDestroy(c.stream);
  delete x;
  return PFEM2_OK;
}

pfem2_status pfem2_add_instance(pfem2_ctx* x, const pfem2_mesh_view* mesh, const pfem2_case* cs, int32_t* inst_out) {
  CTX_CHECK(x);
  Ctx& c = x->c;
  if (c.setup_done) { set_error("instances must be added before pfem2_setup"); return PFEM2_BAD_STATE; }
  if (!mesh || !cs || !mesh->vertices || !mesh->cells || !mesh->face_boundary_id || mesh->n_cells <= 0 ||
      mesh->n_vertices <= 0) {
    set_error("invalid mesh view");
    return PFEM2_INVALID_ARG;
  }
  if (!(cs->dt > 0) || !(cs->rho > 0) || !(cs->mu >= 0)) { set_error("invalid case parameters"); return PFEM2_INVALID_ARG; }
  for (int f = 0; f < 4; ++f)
    if (cs->n_dirichlet[f] < 0 || cs->n_dirichlet[f] > PFEM2_MAX_BC) { set_error("bad n_dirichlet"); return PFEM2_INVALID_ARG; }
  const int dim = c.dim, NV = 1 << dim, NF = 2 * dim;
  HostInst in;
  in.nv = mesh->n_vertices;
  in.nc = mesh->n_cells;
  in.cs = *cs;
  in.X.assign(mesh->vertices, mesh->vertices + (size_t)in.nv * dim);
  in.cells.assign(mesh->cells, mesh->cells + (size_t)in.nc * NV);
  in.fb.assign(mesh->face_boundary_id, mesh->face_boundary_id + (size_t)in.nc * NF);
  c.inst.push_back(std::move(in));
  if (inst_out) *inst_out = (int32_t)c.inst.size() - 1;
  return PFEM2_OK;
}

pfem2_status pfem2_setup(pfem2_ctx* x) {
  CTX_CHECK(x);
  Ctx& c = x->c;
  if (c.setup_done) { set_error("pfem2_setup called twice"); return PFEM2_BAD_STATE; }
  if (c.inst.empty()) { set_error("no instances"); return PFEM2_BAD_STATE; }
  PFEM2_CUDA(cudaSetDevice(c.device));
  return do_setup(c);
}

pfem2_status pfem2_seed(pfem2_ctx* x, int32_t instance, const uint32_t q[3], uint64_t seed, double jitter) {
  SETUP_CHECK(x);
  LIVE_CHECK(x);
  Ctx& c = x->c;
  if (!q || q[0] < 1 || q[1] < 1 || (c.dim == 3 && q[2] < 1)) { set_error("bad q"); return PFEM2_INVALID_ARG; }
  int nb = (q[0] + 1) * (q[1] + 1) * (c.dim == 3 ? q[2] + 1 : 1);
  if (nb > 256) { set_error("q too large: at most 256 sub-cell buckets per cell"); return PFEM2_INVALID_ARG; }
  if (instance >= (int)c.inst.size()) { set_error("bad instance"); return PFEM2_INVALID_ARG; }
  PFEM2_CUDA(cudaSetDevice(c.device));
  for (size_t i = 0; i < c.inst.size(); ++i)
    if (instance < 0 || (int)i == instance) {
      for (int d = 0; d < 3; ++d) c.inst[i].q[d] = (d < c.dim) ? q[d] : 1;
      for (int d = 0; d < 3; ++d) {
        c.h_inst[i].q[d] = (int)c.inst[i].q[d];
        c.h_inst[i].h[d] = 1.0 / c.h_inst[i].q[d];
        c.h_inst[i].qm[d] = ((1ull << 32) + c.h_inst[i].q[d] - 1) / c.h_inst[i].q[d];
      }
    }
  for (auto& in : c.inst)
    if (in.q[0] == 0) { set_error("every instance needs particles: seed all instances"); return PFEM2_BAD_STATE; }
  PFEM2_CUDA(cudaMemcpy(c.d_inst, c.h_inst.data(), sizeof(DevInst) * c.h_inst.size(), cudaMemcpyHostToDevice));
  size_t total = 0;
  for (auto& in : c.inst) total += (size_t)in.nc * in.q[0] * in.q[1] * in.q[2];
  PFEM2_TRY(alloc_particles(c, total));
  c.cur = 0;
  PFEM2_TRY(launch_seed(c, instance, q, seed, jitter));
  c.seeded = true;
  c.stats.n_particles = (int)total;
  x->graph_failed = false;
  for (int k = 0; k < 2; ++k)
    if (x->graph[k]) { cudaGraphExecDestroy(x->graph[k]); x->graph[k] = nullptr; }
  return PFEM2_OK;
}

pfem2_status pfem2_correct(pfem2_ctx* x) {
  SEED_CHECK(x);
  PFEM2_TRY(launch_correct(x->c));
  PFEM2_CUDA(cudaStreamSynchronize(x->c.stream));
  PFEM2_CUDA(cudaGetLastError());
  return PFEM2_OK;
}

pfem2_status pfem2_advect(pfem2_ctx* x) {
  SEED_CHECK(x);
  PFEM2_TRY(launch_advect(x->c, false));
  PFEM2_TRY(launch_rebin(x->c, false, false, true));
  PFEM2_CUDA(cudaGetLastError());
  return check_counters(x->c, true);
}

pfem2_status pfem2_check_empty(pfem2_ctx* x) {
  SEED_CHECK(x);
  PFEM2_CUDA(cudaMemsetAsync(x->c.d_counters, 0, sizeof(int) * CNT_N_STATS, x->c.stream));
  PFEM2_TRY(launch_rebin(x->c, true, false, false));
  PFEM2_CUDA(cudaGetLastError());
  return check_counters(x->c, true);
}

pfem2_status pfem2_move(pfem2_ctx* x) {
  SEED_CHECK(x);
  PFEM2_TRY(launch_advect(x->c, false));
  PFEM2_TRY(launch_rebin(x->c, true, false, true));
  PFEM2_CUDA(cudaGetLastError());
  return check_counters(x->c, true);
}

pfem2_status pfem2_project(pfem2_ctx* x) {
  SEED_CHECK(x);
  PFEM2_TRY(launch_project(x->c, false));
  PFEM2_CUDA(cudaStreamSynchronize(x->c.stream));
  PFEM2_CUDA(cudaGetLastError());
  return PFEM2_OK;
}

pfem2_status pfem2_fem_step(pfem2_ctx* x) {
  SETUP_CHECK(x);
  LIVE_CHECK(x);
  if (x->c.cfg.particles_only) {
    set_error("pfem2_fem_step: the context was created with particles_only");
    return PFEM2_BAD_STATE;
  }
  PFEM2_TRY(fem_step_launch(x->c));
  PFEM2_CUDA(cudaStreamSynchronize(x->c.stream));
  PFEM2_CUDA(cudaGetLastError());
  return krylov_read_stats(x->c);
}

static pfem2_status run_step(pfem2_ctx* x) {
  Ctx& c = x->c;
  const int par = c.cur;
  if (c.cfg.use_graph && !x->graph_failed) {
    if (!x->graph[par]) {
      cudaGraph_t g;
      cudaError_t e = cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return cuda_status(e, "cudaStreamBeginCapture");
      long long l0 = c.launches;
      pfem2_status s = step_launch(c);
      e = cudaStreamEndCapture(c.stream, &g);
      c.cur = par;  // capture does not execute: restore the parity
      x->graph_launches[par] = c.launches - l0;
      c.launches = l0;
      if (s != PFEM2_OK || e != cudaSuccess) {
        cudaGetLastError();
        x->graph_failed = true;
        if (g) cudaGraphDestroy(g);
      } else {
        e = cudaGraphInstantiate(&x->graph[par], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
          cudaGetLastError();
          x->graph[par] = nullptr;
          x->graph_failed = true;
        }
      }
    }
    if (x->graph[par]) {
      PFEM2_CUDA(cudaGraphLaunch(x->graph[par], c.stream));
      c.cur = 1 - par;
      c.launches += x->graph_launches[par];
      return PFEM2_OK;
    }
  }
  return step_launch(c);
}

pfem2_status pfem2_step(pfem2_ctx* x) {
  SEED_CHECK(x);
  Ctx& c = x->c;
  if (c.timing) PFEM2_TRY(collect_stage_times(c));
  PFEM2_TRY(run_step(x));
  c.ev_pending = c.timing;
  c.time += c.inst[0].cs.dt;
  c.timestep += 1;
  PFEM2_CUDA(cudaGetLastError());
  return PFEM2_OK;
}

// the loads of instance i (5 sums, then the two probe pressures) into
// loads_dev[7 i ...], asynchronously on the context's stream
static pfem2_status enqueue_loads(Ctx& c, int i, int patch) {
  double* d = c.loads_dev + 7 * i;
  PFEM2_TRY(launch_loads(c, i, patch, d));
  const pfem2_case& cs = c.inst[i].cs;
  const double* P = c.F[PFEM2_FIELD_P] + c.inst[i].v_off;
  PFEM2_CUDA(cudaMemsetAsync(d + 5, 0, 2 * sizeof(double), c.stream));
  if (cs.probe_a >= 0) PFEM2_CUDA(cudaMemcpyAsync(d + 5, P + cs.probe_a, 8, cudaMemcpyDeviceToDevice, c.stream));
  if (cs.probe_b >= 0) PFEM2_CUDA(cudaMemcpyAsync(d + 6, P + cs.probe_b, 8, cudaMemcpyDeviceToDevice, c.stream));
  return PFEM2_OK;
}

// the 5 published load values of instance i from its 7 raw values
// (2D: drag and lift coefficients split into viscous and pressure parts and
// the probe pressure difference p(a) - p(b), TurekBenchmark/pfem2particle.cpp:
// 945-956; 3D: the pressure force and the pressure at the probe, the mean
// over the listed probe vertices, tubePoiseuille3D/pfem2particle.cpp:720-731)
static void finish_loads(const Ctx& c, int i, const double* raw, double* out) {
  const pfem2_case& cs = c.inst[i].cs;
  if (c.dim == 2) {
    const double s = cs.rho * cs.load_umean * cs.load_umean * cs.load_diam;
    for (int k = 0; k < 4; ++k) out[k] = s != 0 ? 2.0 * raw[k] / s : 0.0;
    out[4] = (cs.probe_a >= 0 ? raw[5] : 0.0) - (cs.probe_b >= 0 ? raw[6] : 0.0);
  } else {
    for (int k = 0; k < 3; ++k) out[k] = raw[k];
    out[3] = 0.0;
    const int np = (cs.probe_a >= 0) + (cs.probe_b >= 0);
    out[4] = np ? ((cs.probe_a >= 0 ? raw[5] : 0.0) + (cs.probe_b >= 0 ? raw[6] : 0.0)) / np : 0.0;
  }
}

pfem2_status pfem2_step_and_read(pfem2_ctx* x, double* loads_out, const int32_t* fields, int32_t n_fields,
                                 double* host_fields) {
  SEED_CHECK(x);
  Ctx& c = x->c;
  const int ni = (int)c.inst.size();
  if (host_fields && fields)
    for (int f = 0; f < n_fields; ++f)
      if (fields[f] < 0 || fields[f] >= PFEM2_N_FIELDS) { set_error("bad field"); return PFEM2_INVALID_ARG; }
  PFEM2_TRY(pfem2_step(x));
  if (loads_out) {
    for (int i = 0; i < ni; ++i) PFEM2_TRY(enqueue_loads(c, i, c.inst[i].cs.load_patch_id));
    PFEM2_CUDA(cudaMemcpyAsync(c.loads_host, c.loads_dev, sizeof(double) * 7 * ni, cudaMemcpyDeviceToHost, c.stream));
  }
  if (host_fields && fields) {
    size_t off = 0;
    for (int i = 0; i < ni; ++i)
      for (int f = 0; f < n_fields; ++f) {
        PFEM2_CUDA(cudaMemcpyAsync(host_fields + off, c.F[fields[f]] + c.inst[i].v_off, sizeof(double) * c.inst[i].nv,
                                   cudaMemcpyDeviceToHost, c.stream));
        off += c.inst[i].nv;
      }
  }
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  for (int i = 0; i < ni && loads_out; ++i) finish_loads(c, i, c.loads_host + 7 * i, loads_out + 5 * i);
  return check_counters(c, false);
}

pfem2_status pfem2_calculate_vorticity(pfem2_ctx* x) {
  SETUP_CHECK(x);
  Ctx& c = x->c;
  if (c.dim != 2) {
    set_error("calculate_vorticity: the vorticity is computed for 2D meshes only");
    return PFEM2_INVALID_ARG;
  }
  PFEM2_TRY(launch_vorticity(c));
  PFEM2_CUDA(cudaGetLastError());
  return PFEM2_OK;
}

pfem2_status pfem2_loads(pfem2_ctx* x, int32_t instance, int32_t patch_id, double out[5]) {
  SETUP_CHECK(x);
  Ctx& c = x->c;
  if (instance < 0 || instance >= (int)c.inst.size() || !out) { set_error("bad argument"); return PFEM2_INVALID_ARG; }
  PFEM2_TRY(enqueue_loads(c, instance, patch_id));
  double* h = c.loads_host + 7 * instance;
  PFEM2_CUDA(cudaMemcpyAsync(h, c.loads_dev + 7 * instance, 7 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  finish_loads(c, instance, h, out);
  return PFEM2_OK;
}

pfem2_status pfem2_get_field(pfem2_ctx* x, int32_t instance, int32_t field, double* host) {
  SETUP_CHECK(x);
  Ctx& c = x->c;
  if (instance < 0 || instance >= (int)c.inst.size() || field < 0 || field >= PFEM2_N_FIELDS || !host) {
    set_error("bad argument");
    return PFEM2_INVALID_ARG;
  }
  PFEM2_CUDA(cudaMemcpyAsync(host, c.F[field] + c.inst[instance].v_off, sizeof(double) * c.inst[instance].nv,
                             cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  return PFEM2_OK;
}

pfem2_status pfem2_set_field(pfem2_ctx* x, int32_t instance, int32_t field, const double* host) {
  SETUP_CHECK(x);
  Ctx& c = x->c;
  if (instance < 0 || instance >= (int)c.inst.size() || field < 0 || field >= PFEM2_N_FIELDS || !host) {
    set_error("bad argument");
    return PFEM2_INVALID_ARG;
  }
  for (int k = 0; k < c.inst[instance].nv; ++k)
    if (!std::isfinite(host[k])) {
      set_error("set_field: a value is not finite");
      return PFEM2_INVALID_ARG;
    }
  PFEM2_CUDA(cudaMemcpyAsync(c.F[field] + c.inst[instance].v_off, host, sizeof(double) * c.inst[instance].nv,
                             cudaMemcpyHostToDevice, c.stream));
  PFEM2_TRY(launch_sync_real_fields(c));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  return PFEM2_OK;
}

pfem2_status pfem2_get_vertices(pfem2_ctx* x, int32_t instance, double* host) {
  SETUP_CHECK(x);
  Ctx& c = x->c;
  if (instance < 0 || instance >= (int)c.inst.size() || !host) { set_error("bad argument"); return PFEM2_INVALID_ARG; }
  PFEM2_CUDA(cudaMemcpyAsync(host, c.X + (size_t)c.inst[instance].v_off * c.dim,
                             sizeof(double) * c.dim * c.inst[instance].nv, cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  return PFEM2_OK;
}

pfem2_status pfem2_particle_count(pfem2_ctx* x, int32_t instance, int32_t* n) {
  SEED_CHECK(x);
  if (!n || instance < 0 || instance >= (int)x->c.inst.size()) { set_error("bad argument"); return PFEM2_INVALID_ARG; }
  int nn = 0;
  PFEM2_TRY(read_particles(x->c, instance, nullptr, nullptr, nullptr, &nn));
  *n = nn;
  return PFEM2_OK;
}

pfem2_status pfem2_get_particles(pfem2_ctx* x, int32_t instance, int32_t* cell, double* xi, double* u) {
  SEED_CHECK(x);
  if (!cell || !xi || !u || instance < 0 || instance >= (int)x->c.inst.size()) { set_error("bad argument"); return PFEM2_INVALID_ARG; }
  int n = 0;
  return read_particles(x->c, instance, cell, xi, u, &n);
}

pfem2_status pfem2_set_particles(pfem2_ctx* x, const int32_t* counts, const int32_t* cell, const double* xi,
                                 const double* u) {
  SETUP_CHECK(x);
  LIVE_CHECK(x);
  Ctx& c = x->c;
  if (!counts || !cell || !xi || !u) { set_error("bad argument"); return PFEM2_INVALID_ARG; }
  size_t total = 0;
  for (size_t i = 0; i < c.inst.size(); ++i) total += counts[i];
  for (auto& in : c.inst)
    if (in.q[0] == 0) { set_error("seed (to set q) before set_particles"); return PFEM2_BAD_STATE; }
  PFEM2_TRY(alloc_particles(c, total));
  c.cur = 0;
  PFEM2_TRY(launch_set_particles(c, counts, cell, xi, u));
  c.seeded = true;
  for (int k = 0; k < 2; ++k)
    if (x->graph[k]) { cudaGraphExecDestroy(x->graph[k]); x->graph[k] = nullptr; }
  return PFEM2_OK;
}

pfem2_status pfem2_get_stats(pfem2_ctx* x, pfem2_stats* out) {
  SETUP_CHECK(x);
  if (!out) { set_error("bad argument"); return PFEM2_INVALID_ARG; }
  pfem2_status s1 = x->c.seeded ? check_counters(x->c, true) : PFEM2_OK;
  pfem2_status s2 = x->c.cfg.particles_only ? PFEM2_OK : krylov_read_stats(x->c);
  *out = x->c.stats;
  return s1 != PFEM2_OK ? s1 : s2;
}

pfem2_status pfem2_get_time(pfem2_ctx* x, double* t, int32_t* n) {
  CTX_CHECK(x);
  if (t) *t = x->c.time;
  if (n) *n = x->c.timestep;
  return PFEM2_OK;
}

pfem2_status pfem2_synchronize(pfem2_ctx* x) {
  CTX_CHECK(x);
  PFEM2_CUDA(cudaStreamSynchronize(x->c.stream));
  return PFEM2_OK;
}

pfem2_status pfem2_launch_count(pfem2_ctx* x, int64_t* n) {
  CTX_CHECK(x);
  if (n) *n = x->c.launches;
  return PFEM2_OK;
}

pfem2_status pfem2_stage_times(pfem2_ctx* x, double* ms, int32_t reset) {
  CTX_CHECK(x);
  PFEM2_TRY(collect_stage_times(x->c));
  if (ms) std::memcpy(ms, x->c.stage_ms, sizeof(double) * PFEM2_N_STAGES);
  if (reset) std::memset(x->c.stage_ms, 0, sizeof(x->c.stage_ms));
  return PFEM2_OK;
}

pfem2_status pfem2_solver_sizes(pfem2_ctx* x, int64_t* out) {
  CTX_CHECK(x);
  if (!out) {
    set_error("pfem2_solver_sizes: null output");
    return PFEM2_INVALID_ARG;
  }
  long long v[PFEM2_N_SOLVER_SIZES];
  krylov_sizes(x->c, v);
  for (int k = 0; k < PFEM2_N_SOLVER_SIZES; ++k) out[k] = v[k];
  return PFEM2_OK;
}

pfem2_status pfem2_enable_stage_timing(pfem2_ctx* x, int32_t on) {
  CTX_CHECK(x);
  PFEM2_TRY(collect_stage_times(x->c));
  if ((on != 0) != x->c.timing) {
    // the captured graphs contain (or lack) the event records: recapture
    for (int k = 0; k < 2; ++k)
      if (x->graph[k]) { cudaGraphExecDestroy(x->graph[k]); x->graph[k] = nullptr; }
  }
  x->c.timing = on != 0;
  return PFEM2_OK;
}

pfem2_status pfem2_get_stream(pfem2_ctx* x, void** stream) {
  CTX_CHECK(x);
  if (stream) *stream = (void*)x->c.stream;
  return PFEM2_OK;
}

pfem2_status pfem2_mesh_elasticity(pfem2_ctx* x, int32_t instance, const pfem2_elasticity* e,
                                   const double body_disp[3], int32_t* iterations, double* residual) {
  SETUP_CHECK(x);
  LIVE_CHECK(x);
  Ctx& c = x->c;
  if (!c.moving) { set_error("pfem2_mesh_elasticity: the context was not created with moving_mesh"); return PFEM2_BAD_STATE; }
  if (instance != 0 || !e || !body_disp) { set_error("pfem2_mesh_elasticity: bad argument"); return PFEM2_INVALID_ARG; }
  if (!(e->lambda >= 0.0) || !(e->mu > 0.0) || !(e->tol >= 0.0) || !(e->rtol >= 0.0) ||
      !(e->tol > 0.0 || e->rtol > 0.0)) {
    set_error("pfem2_mesh_elasticity: lambda >= 0, mu > 0 and a positive tolerance needed");
    return PFEM2_INVALID_ARG;
  }
  for (int d = 0; d < c.dim; ++d)
    if (!std::isfinite(body_disp[d])) { set_error("pfem2_mesh_elasticity: body_disp not finite"); return PFEM2_INVALID_ARG; }
  PFEM2_CUDA(cudaSetDevice(c.device));
  int it = 0;
  double res = 0.0;
  const pfem2_status st = ale_elasticity(c, *e, body_disp, &it, &res);
  if (iterations) *iterations = it;
  if (residual) *residual = res;
  return st;
}

pfem2_status pfem2_move_mesh(pfem2_ctx* x) {
  SETUP_CHECK(x);
  LIVE_CHECK(x);
  Ctx& c = x->c;
  if (!c.moving) { set_error("pfem2_move_mesh: the context was not created with moving_mesh"); return PFEM2_BAD_STATE; }
  PFEM2_CUDA(cudaSetDevice(c.device));
  PFEM2_TRY(ale_move_mesh(c));
  // the graphs hold kernels of the old particle capacity only: geometry is
  // read from device memory, so they stay valid
  return c.seeded ? check_counters(c, true) : PFEM2_OK;
}

pfem2_status pfem2_set_tuning(pfem2_ctx* x, const pfem2_tuning* t) {
  CTX_CHECK(x);
  if (!t) { set_error("pfem2_set_tuning: null argument"); return PFEM2_INVALID_ARG; }
  if (x->c.setup_done) { set_error("pfem2_set_tuning: call it before pfem2_setup"); return PFEM2_BAD_STATE; }
  PFEM2_TRY(check_tuning(*t));
  x->c.tune_req = *t;
  return PFEM2_OK;
}

pfem2_status pfem2_get_tuning(pfem2_ctx* x, pfem2_tuning* t) {
  CTX_CHECK(x);
  if (!t) { set_error("pfem2_get_tuning: null argument"); return PFEM2_INVALID_ARG; }
  const Ctx& c = x->c;
  *t = c.setup_done ? c.tune : c.tune_req;
  if (c.setup_done && !t->advect_split) t->advect_split = (long long)c.pcap >= c.adv_split_min ? 2 : 1;
  return PFEM2_OK;
}

pfem2_status pfem2_tuning_key(pfem2_ctx* x, char* buf, int32_t len) {
  CTX_CHECK(x);
  if (!buf || len <= 0) { set_error("pfem2_tuning_key: no buffer"); return PFEM2_INVALID_ARG; }
  if (x->c.inst.empty()) { set_error("pfem2_tuning_key: no instances"); return PFEM2_BAD_STATE; }
  const std::string k = tuning_key(x->c);
  if ((int)k.size() >= len) { set_error("pfem2_tuning_key: buffer too small"); return PFEM2_INVALID_ARG; }
  std::memcpy(buf, k.c_str(), k.size() + 1);
  return PFEM2_OK;
}

}  // extern "C"
