// particles.cu -- particle kernels of the PFEM2 step (sm_100a).
//
// Layout: particles are SoA and sorted by cell (cell_start offsets), with
// reference coordinates xi[d][cap] and carried velocity u[d][cap] in the
// arithmetic type R (float for the mixed path, double for the plain path).
//
// Kernels and the reference routines they replace:
//   k_seed          seed_particles / seed_particles_into_cell
//                   (TurekBenchmark/pfem2particle.cpp:701-721,774-790)
//   k_correct       correct_particles_velocities (:792-811)
//   k_advect_q,     move_particles sub-steps (:813-848) + point location
//   k_advect_one
//                   sort_particles_into_subdomains_and_cells (:276-507),
//                   find_closest_vertex_of_cell (:142-166),
//                   compare_particle_association (:268-274)
//   k_rebin         the re-sort by cell plus check_cell_for_empty_parts
//                   (:723-772), with the projection partials fused in
//   k_project_*     distribute_particle_velocities_to_grid (:858-918)
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "common.cuh"
#include "ctx.h"

namespace pfem2 {

constexpr int kRebinWarps = 8;
constexpr int kMaxBuckets = 256;
// resident rebin blocks per SM the registers are capped for: the kernel is
// bound by dependent loads, so resident warps pay more than registers; in 2D
// FP32 six blocks (48 warps) measured 17% faster than the four that 64
// registers allowed, in 3D FP32 four blocks 36% faster than uncapped; with
// FP64 particles five blocks in 2D (0.186 -> 0.110 ms on the 52k-cell
// channel against two uncapped, 96 registers) and three in 3D (3.15 -> 1.61
// ms on the 442k-cell pipe against one, 181 registers)
template <int DIM, typename R>
struct RebinMinBlocks {
  static constexpr int value = sizeof(R) == 4 ? (DIM == 2 ? 6 : 4) : (DIM == 2 ? 5 : 3);
};

// ------------------------------------------------------------------ seed
template <int DIM, typename R>
__global__ void k_seed(int c0, int c1, int q0, int q1, int q2, int pbase, uint64_t seed, double jitter,
                       const double* __restrict__ X, const int* __restrict__ cv, const double* __restrict__ V0,
                       const double* __restrict__ V1, const double* __restrict__ V2, int* __restrict__ cell,
                       R* __restrict__ xi, R* __restrict__ u, size_t cap, int* __restrict__ cell_start) {
  constexpr int NV = Dims<DIM>::NV;
  const int Q = q0 * q1 * q2;
  const double h[3] = {1.0 / q0, 1.0 / q1, 1.0 / q2};
  const double* V[3] = {V0, V1, V2};
  for (int c = c0 + blockIdx.x * blockDim.x + threadIdx.x; c < c1; c += gridDim.x * blockDim.x) {
    const size_t pc = (size_t)pbase + (size_t)(c - c0) * Q;
    cell_start[c] = (int)pc;
    for (int t = 0; t < Q; ++t) {
      int idx[3] = {t / (q1 * q2), (t / q2) % q1, t % q2};
      uint64_t ord = (uint64_t)(c - c0) * Q + t;
      double x[3];
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        x[d] = (idx[d] + 1.0 / 2) * h[d];
        if (jitter != 0.0) x[d] += jitter * (2.0 * uniform01(seed, ord, d) - 1.0);
      }
      double N[NV];
      shape_values<DIM, double>(x, N);
      double uu[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        int g = __ldg(cv + (size_t)c * NV + v);
#pragma unroll
        for (int d = 0; d < DIM; ++d) uu[d] = uu[d] + N[v] * V[d][g];
      }
      size_t p = pc + t;
      cell[p] = c;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        xi[d * cap + p] = R(x[d]);
        u[d * cap + p] = R(uu[d]);
      }
    }
  }
}

template <int DIM, typename R>
static pfem2_status seed_impl(Ctx& c, uint64_t seed, double jitter) {
  int b = c.cur;
  size_t total = 0;
  for (auto& in : c.inst) total += (size_t)in.nc * in.q[0] * in.q[1] * (DIM == 3 ? in.q[2] : 1);
  if (total > (size_t)c.pcap) {
    set_error("seed: particle capacity exceeded");
    return PFEM2_PARTICLE_OVERFLOW;
  }
  size_t pbase = 0;
  for (auto& in : c.inst) {
    int q2 = DIM == 3 ? (int)in.q[2] : 1;
    int grid = grid_for(c, in.nc, 128, 16);
    k_seed<DIM, R><<<grid, 128, 0, c.stream>>>(in.c_off, in.c_off + in.nc, in.q[0], in.q[1], q2, (int)pbase, seed,
                                               jitter, c.X, c.cv, c.F[PFEM2_FIELD_VX], c.F[PFEM2_FIELD_VY],
                                               c.F[PFEM2_FIELD_VZ], c.pcell[b], (R*)c.pxi[b], (R*)c.pu[b],
                                               (size_t)c.pcap, c.cell_start[b]);
    c.launches++;
    pbase += (size_t)in.nc * in.q[0] * in.q[1] * q2;
  }
  int tot = (int)total;
  PFEM2_CUDA(cudaMemcpyAsync(c.cell_start[b] + c.nc, &tot, sizeof(int), cudaMemcpyHostToDevice, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(c.d_np + b, &tot, sizeof(int), cudaMemcpyHostToDevice, c.stream));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  PFEM2_CUDA(cudaGetLastError());
  return PFEM2_OK;
}

pfem2_status launch_seed(Ctx& c, int instance, const uint32_t q[3], uint64_t seed, double jitter) {
  (void)instance;
  if (c.dim == 2) return c.pmixed ? seed_impl<2, float>(c, seed, jitter) : seed_impl<2, double>(c, seed, jitter);
  return c.pmixed ? seed_impl<3, float>(c, seed, jitter) : seed_impl<3, double>(c, seed, jitter);
}

// -------------------------------------------------------- real mirrors
template <int DIM, typename R>
__global__ void k_sync_real(int nv, const double* __restrict__ V0, const double* __restrict__ V1,
                            const double* __restrict__ V2, const double* __restrict__ O0,
                            const double* __restrict__ O1, const double* __restrict__ O2, R* __restrict__ Vr,
                            R* __restrict__ dVr) {
  const double* V[3] = {V0, V1, V2};
  const double* O[3] = {O0, O1, O2};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      double v = V[d][i];
      Vr[(size_t)d * nv + i] = R(v);
      dVr[(size_t)d * nv + i] = R(v - O[d][i]);
    }
  }
}

template <int DIM, typename R>
static pfem2_status sync_real_impl(Ctx& c) {
  k_sync_real<DIM, R><<<grid_for(c, c.nv, 256), 256, 0, c.stream>>>(
      c.nv, c.F[PFEM2_FIELD_VX], c.F[PFEM2_FIELD_VY], c.F[PFEM2_FIELD_VZ], c.F[PFEM2_FIELD_OLD_VX],
      c.F[PFEM2_FIELD_OLD_VY], c.F[PFEM2_FIELD_OLD_VZ], (R*)c.Vr, (R*)c.dVr);
  c.launches++;
  return PFEM2_OK;
}

pfem2_status launch_sync_real_fields(Ctx& c) {
  if (c.dim == 2) return c.pmixed ? sync_real_impl<2, float>(c) : sync_real_impl<2, double>(c);
  return c.pmixed ? sync_real_impl<3, float>(c) : sync_real_impl<3, double>(c);
}

// --------------------------------------------------------------- correct
template <int DIM, typename R>
__global__ void __launch_bounds__(256) k_correct(const int* __restrict__ cell, const R* __restrict__ xi,
                                                 R* __restrict__ u, size_t cap, const int* __restrict__ d_np,
                                                 const int* __restrict__ cv, const R* __restrict__ dV, int nv) {
  constexpr int NV = Dims<DIM>::NV;
  const int n = min(*d_np, (int)cap);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int c = cell[p];
    R x[DIM], up[DIM], N[NV];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      x[d] = xi[d * cap + p];
      up[d] = u[d * cap + p];
    }
    shape_values<DIM, R>(x, N);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      int g = __ldg(cv + (size_t)c * NV + v);
#pragma unroll
      for (int d = 0; d < DIM; ++d) up[d] = up[d] + N[v] * __ldg(dV + (size_t)d * nv + g);
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) u[d * cap + p] = up[d];
  }
}

template <int DIM, typename R>
static pfem2_status correct_impl(Ctx& c) {
  int b = c.cur;
  k_correct<DIM, R><<<grid_for(c, c.pcap, 256, 8), 256, 0, c.stream>>>(
      c.pcell[b], (const R*)c.pxi[b], (R*)c.pu[b], (size_t)c.pcap, c.d_np + b, c.cv, (const R*)c.dVr, c.nv);
  c.launches++;
  return PFEM2_OK;
}

pfem2_status launch_correct(Ctx& c) {
  if (c.dim == 2) return c.pmixed ? correct_impl<2, float>(c) : correct_impl<2, double>(c);
  return c.pmixed ? correct_impl<3, float>(c) : correct_impl<3, double>(c);
}

// ---------------------------------------------------------------- advect
// One thread per particle; all PARTICLES_MOVEMENT_STEPS sub-steps run in
// registers (the nodal field is fixed during move_particles). After each
// sub-step the particle is located like the reference does: current cell
// first, then the patch of the "closest" vertex in alignment order; a
// particle found nowhere is deleted (newcell = -1).
// resident 256-thread blocks per SM the advection kernel is compiled for:
// it is latency-bound, so the FP32 2D variant trades its few extra
// registers for four blocks (32 warps) per SM, and the FP64 3D variant
// (240 registers uncapped, one block) runs two at 128 registers in spite of
// its spills (2.72 -> 2.40 ms on the 442k-cell pipe; three: 4.0 ms); the
// FP64 2D variant measured slower with three than with two
template <int DIM, typename R>
struct AdvectMinBlocks {
  static constexpr int value = DIM == 2 ? (sizeof(R) == 4 ? 4 : 2) : 2;
};


constexpr int kAdvLeft = -2;  // advect_steps<.., false>: the particle left its cell

// patches of at most this many cells are searched without the sort's
// local-memory arrays
constexpr int kSmallPatch = 8;

// The reference's search for a point xn (cell-local frame of cell c, whose
// record is G / L / x0) that left cell c (sort_particles_into_subdomains_and_
// cells, TurekBenchmark/pfem2particle.cpp:276-507): the vertex of c best
// aligned with the direction uf from the old position xo
// (find_closest_vertex_of_cell, :142-166), then that vertex's cells ordered
// by the alignment of their centre directions with vertex -> point
// (compare_particle_association, :268-274), the first that contains the
// point. On success c, G, L, x0 and the reference coordinates x are those of
// the new cell; false when no cell of the patch contains the point.
template <int DIM, typename R>
__device__ __forceinline__ bool locate_from(int& c, CellGeo<DIM, R>& G, LocalCell<DIM, R>& L, double* x0,
                                            const R* xo, const R* xn, const R* uf, R* x, const int* gvx,
                                            const CellGeo<DIM, R>* __restrict__ geo,
                                            const int* __restrict__ v2c_ptr, const int* __restrict__ v2c_cell,
                                            const R* __restrict__ v2c_dir) {
  constexpr int NV = Dims<DIM>::NV;
  R x2[DIM];
  {
    // closest vertex of the old cell seen along the velocity
    R un = R(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) un += uf[d] * uf[d];
    un = sqrt(un);
    R best = R(0);
    int bv = 0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      R t[DIM], tn = R(0), dot = R(0);
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        t[d] = L.D[v][d] - xo[d];
        tn += t[d] * t[d];
      }
      tn = sqrt(tn);
#pragma unroll
      for (int d = 0; d < DIM; ++d) dot += (uf[d] / un) * (t[d] / tn);
      if (v == 0) best = dot;
      else if (dot > best) { best = dot; bv = v; }
    }
    const int gv = gvx[bv];
    R vp[DIM], vpn = R(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      vp[d] = xn[d] - L.D[bv][d];
      vpn += vp[d] * vp[d];
    }
    vpn = sqrt(vpn);
#pragma unroll
    for (int d = 0; d < DIM; ++d) vp[d] /= vpn;
    const int k0 = __ldg(v2c_ptr + gv);
    int nk = __ldg(v2c_ptr + gv + 1) - k0;
    if (nk > kMaxPatch) nk = kMaxPatch;
    bool found = false;
    // the point in patch cell i (i in v2c order): on success the new cell
    auto try_cell = [&](int i) {
      const int cc = __ldg(v2c_cell + k0 + i);
      const CellGeo<DIM, R> Gc = geo[cc];
      LocalCell<DIM, R> Lc;
      double xc[DIM];
      geo_to_local<DIM, R>(Gc, Lc, xc);
      R t[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) t[d] = xn[d] + R(x0[d] - xc[d]);
      if (geo_inverse<DIM, R>(Gc, Lc, t, x2) && inside_unit<DIM, R>(x2)) {
        found = true;
        c = cc;
        G = Gc;
        L = Lc;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          x0[d] = xc[d];
          x[d] = x2[d];
        }
      }
    };
    auto align = [&](int i) {
      R sdot = R(0);
#pragma unroll
      for (int d = 0; d < DIM; ++d) sdot += __ldg(v2c_dir + (size_t)(k0 + i) * DIM + d) * vp[d];
      return sdot;
    };
    if (nk <= kSmallPatch) {
      // small patches: the cells are tried in order by repeated selection of
      // the best aligned remaining one (the lowest index among equal
      // alignments), which is the order of the stable sort below without
      // its local-memory arrays; the alignments are recomputed per round
      // from cached loads, and usually the first cell tried holds the point
      unsigned left = (1u << nk) - 1u;
      while (left && !found) {
        int bi = -1;
        R bk = R(0);
        for (int i = 0; i < nk; ++i) {
          if (!((left >> i) & 1u)) continue;
          const R k = align(i);
          if (bi < 0 || k > bk) {
            bi = i;
            bk = k;
          }
        }
        left &= ~(1u << bi);
        try_cell(bi);
      }
      return found;
    }
    R key[kMaxPatch];
    int perm[kMaxPatch];
    for (int i = 0; i < nk; ++i) {
      const R sdot = align(i);
      key[i] = sdot;
      // stable insertion by descending alignment (std::sort is an
      // insertion sort, hence stable, for patches of <= 16 cells)
      int j = i - 1;
      while (j >= 0 && sdot > key[perm[j]]) {
        perm[j + 1] = perm[j];
        --j;
      }
      perm[j + 1] = i;
    }
    for (int i = 0; i < nk && !found; ++i) try_cell(perm[i]);
    return found;
  }
}

// Sub-steps s0 .. S-1 of the S forward-Euler sub-steps of one particle with
// the Q1-interpolated mesh velocity (move_particles,
// TurekBenchmark/pfem2particle.cpp:813-856), starting in cell c0 at
// reference coordinates x (updated). After a sub-step
// the point is first tried in the current cell; if it left, FULL runs the
// reference's search (sort_particles_into_subdomains_and_cells: the vertex
// of the old cell best aligned with the velocity, then that vertex's cells
// ordered by alignment with the directions to their centres, :276-507) and
// returns the new cell, or -1 when no cell of the patch contains the point
// (the particle is deleted); without FULL it returns kAdvLeft at the first
// sub-step that leaves the cell, with x still at the start of that
// sub-step and its index in s_left. Otherwise it returns the cell.
template <int DIM, typename R, bool FULL>
__device__ __forceinline__ int advect_steps(int c0, R* x, R dts, int s0, int& s_left, int S,
                                            const CellGeo<DIM, R>* __restrict__ geo,
                                            const int* __restrict__ cv, const R* __restrict__ Vr, int nv,
                                            const int* __restrict__ v2c_ptr, const int* __restrict__ v2c_cell,
                                            const R* __restrict__ v2c_dir) {
  constexpr int NV = Dims<DIM>::NV;
  int c = c0;
  // vertex ids and velocities of the current cell, reloaded only when the
  // particle changes cell
  int gvx[NV];
  R vv[NV][DIM], N[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) gvx[v] = __ldg(cv + (size_t)c * NV + v);
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int d = 0; d < DIM; ++d) vv[v][d] = __ldg(Vr + (size_t)d * nv + gvx[v]);
  CellGeo<DIM, R> G = geo[c];
  LocalCell<DIM, R> L;
  double x0[DIM];
  geo_to_local<DIM, R>(G, L, x0);
  for (int s = s0; s < S; ++s) {
    shape_values<DIM, R>(x, N);
    R uf[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) uf[d] = R(0);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) uf[d] = uf[d] + N[v] * vv[v][d];
    }
    R xo[DIM], xn[DIM], x2[DIM];
    local_map<DIM, R>(L, x, xo);
#pragma unroll
    for (int d = 0; d < DIM; ++d) xn[d] = xo[d] + uf[d] * dts;
    if (geo_inverse<DIM, R>(G, L, xn, x2) && inside_unit<DIM, R>(x2)) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) x[d] = x2[d];
      continue;
    }
    if (!FULL) {
      s_left = s;
      return kAdvLeft;
    }
    if (!locate_from<DIM, R>(c, G, L, x0, xo, xn, uf, x, gvx, geo, v2c_ptr, v2c_cell, v2c_dir)) return -1;
#pragma unroll
    for (int v = 0; v < NV; ++v) gvx[v] = __ldg(cv + (size_t)c * NV + v);
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int d = 0; d < DIM; ++d) vv[v][d] = __ldg(Vr + (size_t)d * nv + gvx[v]);
  }
  return c;
}

// deletion count and far movers of one advected particle (c: its new cell,
// -1 when deleted)
__device__ __forceinline__ void advect_record(int p, int c0, int c, const int* __restrict__ ring_ptr,
                                              const int* __restrict__ ring_cell,
                                              unsigned long long* __restrict__ far_keys, int far_cap,
                                              int* __restrict__ counters, unsigned* __restrict__ dest_mask) {
  if (c < 0) {
    atomicAdd(counters + CNT_DELETED, 1);
  } else if (c != c0) {
    // a particle that left the 1-ring of its old cell goes to the far list;
    // one that stays in it marks its destination (bit = ring position) in
    // the old cell's mask, so that the re-sort scans only segments that send
    // particles to a cell
    bool near = false;
    const int r0 = __ldg(ring_ptr + c0);
    for (int rr = r0; rr < __ldg(ring_ptr + c0 + 1); ++rr)
      if (__ldg(ring_cell + rr) == c) {
        near = true;
        atomicOr(dest_mask + c0, rr - r0 < 32 ? 1u << (rr - r0) : 0xffffffffu);
        break;
      }
    if (!near) {
      int slot = atomicAdd(counters + CNT_FAR, 1);
      if (slot < far_cap) far_keys[slot] = ((unsigned long long)(unsigned)c << 32) | (unsigned)p;
      else atomicExch(counters + CNT_FAR_OVERFLOW, 1);
    }
  }
}

// Advection in one pass (selectable with advect_split = 1 or below
// PFEM2_ADVECT_SPLIT_MIN slots): correction, every sub-step with the full
// point location in line. Same arithmetic as the two-phase form.
template <int DIM, typename R, bool FUSE>
__global__ void __launch_bounds__(256, AdvectMinBlocks<DIM, R>::value) k_advect_one(
    const int* __restrict__ cell, R* __restrict__ xi, R* __restrict__ u, int* __restrict__ newcell, size_t cap,
    const int* __restrict__ d_np, const CellGeo<DIM, R>* __restrict__ geo, const int* __restrict__ cv,
    const R* __restrict__ Vr, const R* __restrict__ dVr, int nv, int S, const DevInst* __restrict__ inst,
    const int* __restrict__ cell_inst, const int* __restrict__ v2c_ptr, const int* __restrict__ v2c_cell,
    const R* __restrict__ v2c_dir, const int* __restrict__ ring_ptr, const int* __restrict__ ring_cell,
    unsigned long long* __restrict__ far_keys, int far_cap, int* __restrict__ counters, unsigned* __restrict__ dest_mask) {
  constexpr int NV = Dims<DIM>::NV;
  const int n = min(*d_np, (int)cap);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int c0 = cell[p];
    R x[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) x[d] = xi[d * cap + p];
    if (FUSE) {
      R N[NV], up[DIM];
      shape_values<DIM, R>(x, N);
#pragma unroll
      for (int d = 0; d < DIM; ++d) up[d] = u[d * cap + p];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const int g = __ldg(cv + (size_t)c0 * NV + v);
#pragma unroll
        for (int d = 0; d < DIM; ++d) up[d] = up[d] + N[v] * __ldg(dVr + (size_t)d * nv + g);
      }
#pragma unroll
      for (int d = 0; d < DIM; ++d) u[d * cap + p] = up[d];
    }
    const R dts = R(inst[__ldg(cell_inst + c0)].dt_sub);
    int s_left = 0;
    int c = advect_steps<DIM, R, true>(c0, x, dts, 0, s_left, S, geo, cv, Vr, nv, v2c_ptr, v2c_cell, v2c_dir);
    if (c < 0) c = -1;
    advect_record(p, c0, c, ring_ptr, ring_cell, far_keys, far_cap, counters, dest_mask);
    newcell[p] = c;
#pragma unroll
    for (int d = 0; d < DIM; ++d) xi[d * cap + p] = x[d];
  }
}

// Advection in two phases per warp (large particle sets): a warp walks its
// 32-particle slices of the block's contiguous chunk; every particle is
// corrected (FUSE) and takes the lean sub-steps while it stays in its cell,
// and one that leaves is appended to the warp's queue in shared memory with
// its state (slot, old cell, the sub-step it left in, its reference
// coordinates at the start of that sub-step). Whenever the queue holds 32
// particles the warp resumes them with the full point location, so that the
// divergent patch search runs on full warps, the leavers' state never goes
// back to memory and the warps stay independent of each other (no block
// barrier). The arithmetic is that of k_advect_one (bitwise equal results).
constexpr int kAdvThreads = 256;

template <int DIM, typename R, bool FUSE>
__global__ void __launch_bounds__(kAdvThreads, AdvectMinBlocks<DIM, R>::value) k_advect_q(
    const int* __restrict__ cell, R* __restrict__ xi, R* __restrict__ u, int* __restrict__ newcell, size_t cap,
    const int* __restrict__ d_np, const CellGeo<DIM, R>* __restrict__ geo, const int* __restrict__ cv,
    const R* __restrict__ Vr, const R* __restrict__ dVr, int nv, int S, const DevInst* __restrict__ inst,
    const int* __restrict__ cell_inst, const int* __restrict__ v2c_ptr, const int* __restrict__ v2c_cell,
    const R* __restrict__ v2c_dir, const int* __restrict__ ring_ptr, const int* __restrict__ ring_cell,
    unsigned long long* __restrict__ far_keys, int far_cap, int* __restrict__ counters, unsigned* __restrict__ dest_mask) {
  constexpr int NV = Dims<DIM>::NV;
  constexpr int NW = kAdvThreads / 32;
  constexpr int QN = 64;  // below 32 left over + 32 appended
  __shared__ int q_p[NW][QN], q_c[NW][QN];
  __shared__ R q_x[NW][DIM][QN];
  __shared__ unsigned short q_s[NW][QN];  // sub-step index (movement_steps <= 65535)
  const int n = min(*d_np, (int)cap);
  const int chunk = (n + gridDim.x - 1) / gridDim.x;
  const int lo = min(n, (int)blockIdx.x * chunk), hi = min(n, lo + chunk);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int nq = 0;  // the warp's queued particles (uniform over the warp)
  for (int base = lo + warp * 32;; base += kAdvThreads) {
    const bool more = base < hi;  // uniform over the warp
    if (more) {
      const int p = base + lane;
      bool leave = false;
      int s_left = 0, c0 = 0;
      R x[DIM];
      if (p < hi) {
        c0 = cell[p];
#pragma unroll
        for (int d = 0; d < DIM; ++d) x[d] = xi[d * cap + p];
        if (FUSE) {
          R N[NV], up[DIM];
          shape_values<DIM, R>(x, N);
#pragma unroll
          for (int d = 0; d < DIM; ++d) up[d] = u[d * cap + p];
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            const int g = __ldg(cv + (size_t)c0 * NV + v);
#pragma unroll
            for (int d = 0; d < DIM; ++d) up[d] = up[d] + N[v] * __ldg(dVr + (size_t)d * nv + g);
          }
#pragma unroll
          for (int d = 0; d < DIM; ++d) u[d * cap + p] = up[d];
        }
        const R dts = R(inst[__ldg(cell_inst + c0)].dt_sub);
        const int c = advect_steps<DIM, R, false>(c0, x, dts, 0, s_left, S, geo, cv, Vr, nv, nullptr, nullptr, nullptr);
        if (c == kAdvLeft) {
          leave = true;
        } else {
          newcell[p] = c;
#pragma unroll
          for (int d = 0; d < DIM; ++d) xi[d * cap + p] = x[d];
        }
      }
      const unsigned m = __ballot_sync(PFEM2_FULL_MASK, leave);
      if (leave) {
        const int k = nq + __popc(m & lanemask_lt());
        q_p[warp][k] = p;
        q_c[warp][k] = c0;
        q_s[warp][k] = (unsigned short)s_left;
#pragma unroll
        for (int d = 0; d < DIM; ++d) q_x[warp][d][k] = x[d];
      }
      nq += __popc(m);
    }
    __syncwarp();
    // resume 32 queued particles at a time (after the last slice: all),
    // from the top of the queue; the order does not change any result
    while (nq >= 32 || (!more && nq > 0)) {
      const int k = nq - 32 + lane;
      if (k >= 0) {
        const int p = q_p[warp][k], c0 = q_c[warp][k];
        R x[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) x[d] = q_x[warp][d][k];
        const R dts = R(inst[__ldg(cell_inst + c0)].dt_sub);
        int s_left = 0;
        int c = advect_steps<DIM, R, true>(c0, x, dts, (int)q_s[warp][k], s_left, S, geo, cv, Vr, nv, v2c_ptr,
                                           v2c_cell, v2c_dir);
        if (c < 0) c = -1;
        advect_record(p, c0, c, ring_ptr, ring_cell, far_keys, far_cap, counters, dest_mask);
        newcell[p] = c;
#pragma unroll
        for (int d = 0; d < DIM; ++d) xi[d * cap + p] = x[d];
      }
      nq = nq > 32 ? nq - 32 : 0;
      __syncwarp();  // the resumed entries are read before the next slice appends over them
    }
    if (!more) break;
  }
}

__global__ void k_far_sort(unsigned long long* keys, const int* __restrict__ counters, int cap);

// ------------------------------------------------------------ moving mesh
// physical position of every particle (FP64) from its cell record, before
// the mesh moves
template <int DIM, typename R>
__global__ void k_particle_positions(const int* __restrict__ cell, const R* __restrict__ xi, size_t cap,
                                     const int* __restrict__ d_np, const CellGeo<DIM, R>* __restrict__ geo,
                                     double* __restrict__ out) {
  const int n = min(*d_np, (int)cap);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const CellGeo<DIM, R> G = geo[cell[p]];
    LocalCell<DIM, R> L;
    double x0[DIM];
    geo_to_local<DIM, R>(G, L, x0);
    R x[DIM], xl[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) x[d] = xi[d * cap + p];
    local_map<DIM, R>(L, x, xl);
#pragma unroll
    for (int d = 0; d < DIM; ++d) out[d * cap + p] = x0[d] + (double)xl[d];
  }
}

// sort_particles_into_subdomains_and_cells after transform_grid: every
// particle keeps its physical position xphys and is located in the moved
// mesh: its cell first, else the reference's vertex-patch search from its
// cell along the direction it moved relative to the mesh (from where its
// old reference coordinates now map to); the new cell (-1: deleted) goes
// to newcell with the moves recorded for the re-sort like the advection's
template <int DIM, typename R>
__global__ void __launch_bounds__(256) k_relocate(
    const int* __restrict__ cell, R* __restrict__ xi, int* __restrict__ newcell, size_t cap,
    const int* __restrict__ d_np, const CellGeo<DIM, R>* __restrict__ geo, const int* __restrict__ cv,
    const int* __restrict__ v2c_ptr, const int* __restrict__ v2c_cell, const R* __restrict__ v2c_dir,
    const double* __restrict__ xphys, const int* __restrict__ ring_ptr, const int* __restrict__ ring_cell,
    unsigned long long* __restrict__ far_keys, int far_cap, int* __restrict__ counters,
    unsigned* __restrict__ dest_mask) {
  constexpr int NV = Dims<DIM>::NV;
  const int n = min(*d_np, (int)cap);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int c0 = cell[p];
    int c = c0;
    CellGeo<DIM, R> G = geo[c0];
    LocalCell<DIM, R> L;
    double x0[DIM];
    geo_to_local<DIM, R>(G, L, x0);
    R x[DIM], xo[DIM], xn[DIM], uf[DIM], x2[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) x[d] = xi[d * cap + p];
    local_map<DIM, R>(L, x, xo);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      xn[d] = R(xphys[d * cap + p] - x0[d]);
      uf[d] = xn[d] - xo[d];
    }
    if (geo_inverse<DIM, R>(G, L, xn, x2) && inside_unit<DIM, R>(x2)) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) x[d] = x2[d];
    } else {
      int gvx[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) gvx[v] = __ldg(cv + (size_t)c0 * NV + v);
      if (!locate_from<DIM, R>(c, G, L, x0, xo, xn, uf, x, gvx, geo, v2c_ptr, v2c_cell, v2c_dir)) c = -1;
    }
    advect_record(p, c0, c, ring_ptr, ring_cell, far_keys, far_cap, counters, dest_mask);
    newcell[p] = c;
    if (c >= 0)
#pragma unroll
      for (int d = 0; d < DIM; ++d) xi[d * cap + p] = x[d];
  }
}

// per-cell records of the particle kernels rebuilt from the vertices on the
// device (the same arithmetic as at setup); *flag = 1 if a cell has a
// non-positive Jacobian at its centre
template <int DIM, typename R>
__global__ void k_cell_geo(int nc, const double* __restrict__ X, const int* __restrict__ cv,
                           CellGeo<DIM, R>* __restrict__ geo, int* __restrict__ flag) {
  constexpr int NV = Dims<DIM>::NV;
  for (int ce = blockIdx.x * blockDim.x + threadIdx.x; ce < nc; ce += gridDim.x * blockDim.x) {
    CellGeo<DIM, R> g;
    double D[NV][DIM];
    const int g0 = cv[(size_t)ce * NV];
#pragma unroll
    for (int a = 0; a < DIM; ++a) g.x0[a] = X[(size_t)g0 * DIM + a];
    double scale = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        D[v][a] = X[(size_t)cv[(size_t)ce * NV + v] * DIM + a] - g.x0[a];
        scale = fmax(scale, fabs(D[v][a]));
        if (v > 0) g.D[v - 1][a] = (R)D[v][a];
      }
    double J[DIM * DIM];
#pragma unroll
    for (int k = 0; k < DIM * DIM; ++k) J[k] = 0.0;
    const double w0 = DIM == 2 ? 0.5 : 0.25;
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int b = 0; b < DIM; ++b) {
        const double w = ((v >> b) & 1) ? w0 : -w0;
#pragma unroll
        for (int a = 0; a < DIM; ++a) J[a * DIM + b] += D[v][a] * w;
      }
    double Ji[DIM * DIM];
    const double det = det_inv<DIM, double>(J, Ji);
    if (!(det > 0.0)) atomicExch(flag, 1);
#pragma unroll
    for (int k = 0; k < DIM * DIM; ++k) g.Ji[k] = (R)Ji[k];
    bool aff = true;
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < DIM; ++b)
          if ((v >> b) & 1) s += D[1 << b][a];
        if (fabs(D[v][a] - s) > 1e-13 * scale) aff = false;
      }
    g.affine = aff ? 1 : 0;
    geo[ce] = g;
  }
}

template <int DIM, typename R>
static pfem2_status positions_impl(Ctx& c, double* out) {
  const int b = c.cur;
  k_particle_positions<DIM, R><<<grid_for(c, c.pcap, 256, 8), 256, 0, c.stream>>>(
      c.pcell[b], (const R*)c.pxi[b], (size_t)c.pcap, c.d_np + b, (const CellGeo<DIM, R>*)c.cell_geo, out);
  c.launches++;
  return PFEM2_OK;
}

pfem2_status launch_particle_positions(Ctx& c, double* out) {
  if (c.dim == 2) return c.pmixed ? positions_impl<2, float>(c, out) : positions_impl<2, double>(c, out);
  return c.pmixed ? positions_impl<3, float>(c, out) : positions_impl<3, double>(c, out);
}

template <int DIM, typename R>
static pfem2_status relocate_impl(Ctx& c, const double* xphys) {
  const int b = c.cur;
  PFEM2_CUDA(cudaMemsetAsync(c.d_counters, 0, sizeof(int) * CNT_N_STATS, c.stream));
  PFEM2_CUDA(cudaMemsetAsync(c.dest_mask, 0, sizeof(unsigned) * c.nc, c.stream));
  k_relocate<DIM, R><<<grid_for(c, c.pcap, 256, 8), 256, 0, c.stream>>>(
      c.pcell[b], (R*)c.pxi[b], c.newcell, (size_t)c.pcap, c.d_np + b, (const CellGeo<DIM, R>*)c.cell_geo, c.cv,
      c.v2c_ptr, c.v2c_cell, (const R*)c.v2c_dir_r, xphys, c.ring_ptr, c.ring_cell, c.far_keys, c.far_cap,
      c.d_counters, c.dest_mask);
  k_far_sort<<<1, 1024, sizeof(unsigned long long) * c.far_cap, c.stream>>>(c.far_keys, c.d_counters, c.far_cap);
  c.launches += 2;
  return PFEM2_OK;
}

pfem2_status launch_relocate(Ctx& c, const double* xphys) {
  const pfem2_status s = c.dim == 2 ? (c.pmixed ? relocate_impl<2, float>(c, xphys) : relocate_impl<2, double>(c, xphys))
                                    : (c.pmixed ? relocate_impl<3, float>(c, xphys) : relocate_impl<3, double>(c, xphys));
  if (s != PFEM2_OK) return s;
  // the re-sort into the moved cells with check_empty_cells
  return launch_rebin(c, true, false, true);
}

pfem2_status launch_cell_geo(Ctx& c, int* flag) {
  const int grid = grid_for(c, c.nc, 128, 8);
  if (c.dim == 2) {
    if (c.pmixed) k_cell_geo<2, float><<<grid, 128, 0, c.stream>>>(c.nc, c.X, c.cv, (CellGeo<2, float>*)c.cell_geo, flag);
    else k_cell_geo<2, double><<<grid, 128, 0, c.stream>>>(c.nc, c.X, c.cv, (CellGeo<2, double>*)c.cell_geo, flag);
  } else {
    if (c.pmixed) k_cell_geo<3, float><<<grid, 128, 0, c.stream>>>(c.nc, c.X, c.cv, (CellGeo<3, float>*)c.cell_geo, flag);
    else k_cell_geo<3, double><<<grid, 128, 0, c.stream>>>(c.nc, c.X, c.cv, (CellGeo<3, double>*)c.cell_geo, flag);
  }
  c.launches++;
  PFEM2_CUDA(cudaGetLastError());
  return PFEM2_OK;
}

// single-CTA bitonic sort of the (cell, particle) keys of the far movers
__global__ void k_far_sort(unsigned long long* keys, const int* __restrict__ counters, int cap) {
  extern __shared__ unsigned long long sk[];
  int n = counters[CNT_FAR];
  if (n > cap) n = cap;
  if (n <= 1) return;
  int m = 1;
  while (m < n) m <<= 1;
  for (int i = threadIdx.x; i < m; i += blockDim.x) sk[i] = i < n ? keys[i] : ~0ull;
  __syncthreads();
  for (int k = 2; k <= m; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        int l = i ^ j;
        if (l > i) {
          bool up = (i & k) == 0;
          unsigned long long a = sk[i], b = sk[l];
          if ((a > b) == up) { sk[i] = b; sk[l] = a; }
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < n; i += blockDim.x) keys[i] = sk[i];
}

// the far-mover sort's shared memory beyond the 48 KB default
pfem2_status far_sort_setup(Ctx& c) {
  PFEM2_CUDA(cudaFuncSetAttribute((const void*)k_far_sort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(unsigned long long) * c.far_cap)));
  return PFEM2_OK;
}

template <int DIM, typename R>
static pfem2_status advect_impl(Ctx& c, bool fuse) {
  int b = c.cur;
  int S = c.cfg.movement_steps;
  const bool split = c.tune.advect_split ? c.tune.advect_split == 2 : (long long)c.pcap >= c.adv_split_min;
  if (!split) {
    const int grid = grid_for(c, c.pcap, 256, c.tune.advect_blocks_per_sm);
    if (fuse)
      k_advect_one<DIM, R, true><<<grid, 256, 0, c.stream>>>(
          c.pcell[b], (R*)c.pxi[b], (R*)c.pu[b], c.newcell, (size_t)c.pcap, c.d_np + b,
          (const CellGeo<DIM, R>*)c.cell_geo, c.cv, (const R*)c.Vr, (const R*)c.dVr, c.nv, S, c.d_inst, c.cell_inst,
          c.v2c_ptr, c.v2c_cell, (const R*)c.v2c_dir_r, c.ring_ptr, c.ring_cell, c.far_keys, c.far_cap, c.d_counters,
          c.dest_mask);
    else
      k_advect_one<DIM, R, false><<<grid, 256, 0, c.stream>>>(
          c.pcell[b], (R*)c.pxi[b], (R*)c.pu[b], c.newcell, (size_t)c.pcap, c.d_np + b,
          (const CellGeo<DIM, R>*)c.cell_geo, c.cv, (const R*)c.Vr, (const R*)c.dVr, c.nv, S, c.d_inst, c.cell_inst,
          c.v2c_ptr, c.v2c_cell, (const R*)c.v2c_dir_r, c.ring_ptr, c.ring_cell, c.far_keys, c.far_cap, c.d_counters,
          c.dest_mask);
    c.launches++;
  } else {
    // the queue kernel's blocks walk contiguous chunks
    const int grid = grid_for(c, c.pcap, kAdvThreads, c.tune.advect_blocks_per_sm);
    if (fuse)
      k_advect_q<DIM, R, true><<<grid, kAdvThreads, 0, c.stream>>>(
          c.pcell[b], (R*)c.pxi[b], (R*)c.pu[b], c.newcell, (size_t)c.pcap, c.d_np + b,
          (const CellGeo<DIM, R>*)c.cell_geo, c.cv, (const R*)c.Vr, (const R*)c.dVr, c.nv, S, c.d_inst, c.cell_inst,
          c.v2c_ptr, c.v2c_cell, (const R*)c.v2c_dir_r, c.ring_ptr, c.ring_cell, c.far_keys, c.far_cap, c.d_counters,
          c.dest_mask);
    else
      k_advect_q<DIM, R, false><<<grid, kAdvThreads, 0, c.stream>>>(
          c.pcell[b], (R*)c.pxi[b], (R*)c.pu[b], c.newcell, (size_t)c.pcap, c.d_np + b,
          (const CellGeo<DIM, R>*)c.cell_geo, c.cv, (const R*)c.Vr, (const R*)c.dVr, c.nv, S, c.d_inst, c.cell_inst,
          c.v2c_ptr, c.v2c_cell, (const R*)c.v2c_dir_r, c.ring_ptr, c.ring_cell, c.far_keys, c.far_cap, c.d_counters,
          c.dest_mask);
    c.launches++;
  }
  k_far_sort<<<1, 1024, sizeof(unsigned long long) * c.far_cap, c.stream>>>(c.far_keys, c.d_counters, c.far_cap);
  c.launches++;
  return PFEM2_OK;
}

pfem2_status launch_advect(Ctx& c, bool fuse) {
  PFEM2_CUDA(cudaMemsetAsync(c.d_counters, 0, sizeof(int) * CNT_N_STATS, c.stream));
  PFEM2_CUDA(cudaMemsetAsync(c.dest_mask, 0, sizeof(unsigned) * c.nc, c.stream));
  if (c.dim == 2) return c.pmixed ? advect_impl<2, float>(c, fuse) : advect_impl<2, double>(c, fuse);
  return c.pmixed ? advect_impl<3, float>(c, fuse) : advect_impl<3, double>(c, fuse);
}

// ----------------------------------------------------------------- rebin
// One warp per target cell. Pass 0 counts, pass 1 writes. The incoming
// particles of cell c are gathered from the old segments of the cells
// sharing a vertex with c (ascending cell id, segment order), so the
// result is a stable sort by cell of the old storage order; particles that
// left that 1-ring come from the sorted far list and are merged by index.
// With CHECK the per-sub-cell counts are walked in that order: a particle
// whose bucket already holds MAX_PARTICLES_PER_CELL_PART is removed, and
// every empty sub-cell receives one particle at its centre, appended in
// (i,j,k) order with the interpolated nodal velocity.
template <int DIM, typename R>
struct ProjAcc {
  R a[Dims<DIM>::NV][DIM + 1];
};

template <int DIM, typename R>
__device__ __forceinline__ void proj_add(ProjAcc<DIM, R>& acc, const R* x, const R* uu) {
  R N[Dims<DIM>::NV];
  shape_values<DIM, R>(x, N);
#pragma unroll
  for (int v = 0; v < Dims<DIM>::NV; ++v) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) acc.a[v][d] += N[v] * uu[d];
    acc.a[v][DIM] += N[v];
  }
}

// Sums N values (N a power of two, at most 32) over a warp with N - 1
// exchanges instead of N * 5: at each halving step a lane keeps one half of
// its values, sends the other half to its partner and adds what it receives.
// Afterwards the lane holds the warp total of value warp_sum_many_index<N>.
template <int N, typename T>
__device__ __forceinline__ T warp_sum_many(T (&v)[N], int lane) {
#pragma unroll
  for (int h = N / 2, o = 16; h >= 1; h >>= 1, o >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < h; ++i) {
      const T send = up ? v[i] : v[i + h];
      const T keep = up ? v[i + h] : v[i];
      v[i] = keep + __shfl_xor_sync(PFEM2_FULL_MASK, send, o);
    }
  }
  T r = v[0];
#pragma unroll
  for (int o = 16 / N; o > 0; o >>= 1) r += __shfl_xor_sync(PFEM2_FULL_MASK, r, o);
  return r;
}

template <int N>
__device__ __forceinline__ int warp_sum_many_index(int lane) {
  int idx = 0;
#pragma unroll
  for (int h = N / 2, o = 16; h >= 1; h >>= 1, o >>= 1)
    if (lane & o) idx += h;
  return idx;
}

template <int DIM, typename R>
__device__ __forceinline__ void proj_store(ProjAcc<DIM, R>& acc, R* __restrict__ partial, int c, int lane) {
  constexpr int K = Dims<DIM>::NV * (DIM + 1);
  constexpr int N = K <= 16 ? 16 : 32;
  static_assert(K <= N, "projection partials exceed a warp");
  R v[N];
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = i < K ? acc.a[i / (DIM + 1)][i % (DIM + 1)] : R(0);
  const R tot = warp_sum_many<N, R>(v, lane);
  const int idx = warp_sum_many_index<N>(lane);
  // every value is held by 32 / N lanes; the first of them stores it
  if ((lane & (32 / N - 1)) == 0 && idx < K) partial[(size_t)c * K + idx] = tot;
}

// sub-cell index of check_cell_for_empty_parts: unsigned(xi / h) with
// h = 1.0 / q, which is q for xi == 1 (a bucket of its own, as in the
// reference); clamped to [0, q]. xi * q has the same integer part unless it
// lies within rounding of an integer, and only there the quotient is formed.
// For FP32 coordinates xi * q is exact in FP64, so that happens only when
// it is an integer; for FP64 coordinates a relative 1e-12 decides.
template <typename R>
__device__ __forceinline__ int sub_bucket_fp64(R xr, double h, int q) {
  const double xi = (double)xr;
  double t = xi * (double)q;
  if (sizeof(R) == 4) {
    if (t == rint(t)) t = xi / h;
  } else if (fabs(t - rint(t)) <= 1e-12 * fmax(1.0, fabs(t))) {
    t = xi / h;
  }
  if (!(t >= 0.0)) t = 0.0;
  if (t > (double)q) t = (double)q;
  return (int)(unsigned)t;
}

template <typename R>
__device__ __forceinline__ int sub_bucket(R xr, double h, int q) {
  return sub_bucket_fp64<R>(xr, h, q);
}

// FP32 coordinates: for 0 < xi < 1, xi = m 2^-s with the 24-bit significand
// m and s = 150 - (biased exponent) >= 24, so xi q = (m q) 2^-s exactly in
// 64-bit integers (q < 2^16): its integer part is the bucket unless xi q
// is itself an integer, where the quotient xi / h decides (the FP64 form,
// as for 0, 1 and anything outside (0, 1)). Same results as the FP64 form,
// with integer instructions only.
template <>
__device__ __forceinline__ int sub_bucket<float>(float xr, double h, int q) {
  const unsigned b = __float_as_uint(xr);
  if (b - 1u < 0x3f7fffffu) {  // 0 < xi < 1 (positive, below the bits of 1.0f)
    const int e = (int)(b >> 23);
    if (e == 0) return 0;  // subnormal: 0 < xi q < 1
    const int sh = 150 - e;
    if (sh < 64) {
      const unsigned long long prod = (unsigned long long)((b & 0x7fffffu) | 0x800000u) * (unsigned)q;
      if (prod & ((1ull << sh) - 1ull)) return (int)(prod >> sh);
    } else {
      return 0;  // xi < 2^-40: 0 < xi q < 1
    }
  }
  return sub_bucket_fp64<float>(xr, h, q);
}

// t / q for t, q < 2^16 with qm = ceil(2^32 / q)
__device__ __forceinline__ int div_small(int t, unsigned long long qm) {
  return (int)(((unsigned long long)(unsigned)t * qm) >> 32);
}

// (i, j, k) of sub-cell t in (i, j, k) order with extents (q0, q1, q2)
__device__ __forceinline__ void sub_cell_ijk(int t, int q1, int q2, const unsigned long long* qm, int id[3]) {
  const int u = div_small(t, qm[2]);  // t / q2
  id[2] = t - u * q2;
  id[0] = div_small(u, qm[1]);        // t / (q1 q2)
  id[1] = u - id[0] * q1;
}

__device__ __forceinline__ int far_lower_bound(const unsigned long long* keys, int n, unsigned long long k) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (keys[mid] < k) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// status words of the single-pass scan over tiles of kRebinWarps cells:
// bits 62-63 = 1 (tile aggregate known) or 2 (inclusive prefix known), the
// low bits the value
constexpr unsigned long long kTileAgg = 1ull << 62, kTilePre = 2ull << 62, kTileVal = (1ull << 62) - 1;

// One pass: a block takes tiles of kRebinWarps consecutive target cells in
// ticket order (an atomic counter, so a block waits only on tiles taken by
// blocks already running), a warp per cell gathers and checks its incoming
// particles into shared memory, the block publishes the tile's particle
// count and finds its output offset by looking back over the previous
// tiles' published counts (decoupled look-back; waits bounded, a timeout is
// flagged in CNT_SCAN_TIMEOUT), then every warp writes its cell's particles,
// its new_start entry and its projection partials.
template <int DIM, typename R, bool CHECK, bool PROJ>
__global__ void __launch_bounds__(kRebinWarps * 32, RebinMinBlocks<DIM, R>::value) k_rebin(
    const int* __restrict__ old_start, const int* __restrict__ newcell, const R* __restrict__ oxi,
    const R* __restrict__ ou, size_t cap, int* __restrict__ ncell, R* __restrict__ nxi, R* __restrict__ nu,
    int* __restrict__ new_start, int* __restrict__ np_out, int nc, const int* __restrict__ ring_ptr,
    const int* __restrict__ ring_cell, const int* __restrict__ ring_rev,
    const unsigned* __restrict__ dest_mask, const unsigned long long* __restrict__ far_keys, int far_cap,
    const DevInst* __restrict__ inst, const int* __restrict__ cell_inst, const int* __restrict__ cv,
    const R* __restrict__ Vr, int nv, R* __restrict__ partial, int list_cap, int* __restrict__ counters,
    unsigned long long* __restrict__ tiles, unsigned spin_limit) {
  constexpr int NV = Dims<DIM>::NV;
  extern __shared__ int smem[];
  __shared__ int s_tile, s_base;
  __shared__ int s_cnt[kRebinWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* list = smem + warp * (list_cap + kMaxBuckets);
  int* bcnt = list + list_cap;
  const unsigned lt = lanemask_lt();
  int nfar = counters[CNT_FAR];
  if (nfar > far_cap) nfar = far_cap;
  const int ntiles = (nc + kRebinWarps - 1) / kRebinWarps;
  unsigned long long* status = tiles + 1;
  for (;;) {
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(tiles, 1ull);
    __syncthreads();
    const int t = s_tile;
    if (t >= ntiles) break;
    const int c = t * kRebinWarps + warp;
    int ntot = 0;
    if (c < nc) {
    // gather the incoming particles of c in (ring cell, segment) order: the
    // ring's segment bounds are loaded across lanes, segments of neighbours
    // that sent no particle to c (their destination masks) are dropped, then
    // the first 32 new-cell ids of 8 remaining segments at a time, so the
    // loads overlap
    int n_in = 0;
    const int r0 = __ldg(ring_ptr + c), nr = __ldg(ring_ptr + c + 1) - r0;
    for (int kb = 0; kb < nr; kb += 32) {
      int sb = 0, se = 0;
      if (kb + lane < nr) {
        const int s = __ldg(ring_cell + r0 + kb + lane);
        sb = min(old_start[s], (int)cap);
        se = min(old_start[s + 1], (int)cap);
        if (s != c) {
          const int rv = __ldg(ring_rev + r0 + kb + lane);
          const unsigned m = dest_mask[s];
          const bool sends = rv < 32 ? ((m >> rv) & 1u) != 0u : m != 0u;
          if (!sends) se = sb;
        }
      }
      unsigned act = __ballot_sync(PFEM2_FULL_MASK, se > sb);
      while (act) {
        int idx[8], v[8], bs[8], es[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          idx[j] = act ? __ffs(act) - 1 : -1;
          act &= act ? act - 1u : 0u;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int src = idx[j] < 0 ? 0 : idx[j];
          bs[j] = __shfl_sync(PFEM2_FULL_MASK, sb, src);
          es[j] = __shfl_sync(PFEM2_FULL_MASK, se, src);
          const int p = bs[j] + lane;
          v[j] = (idx[j] >= 0 && p < es[j]) ? newcell[p] : -1;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if (idx[j] < 0) break;
          {
            const int p = bs[j] + lane;
            const bool pred = v[j] == c;
            const unsigned m = __ballot_sync(PFEM2_FULL_MASK, pred);
            const int pos = n_in + __popc(m & lt);
            if (pred && pos < list_cap) list[pos] = p;
            n_in += __popc(m);
          }
          for (int base = bs[j] + 32; base < es[j]; base += 32) {  // segments longer than a warp
            const int p = base + lane;
            const bool pred = p < es[j] && newcell[p] == c;
            const unsigned m = __ballot_sync(PFEM2_FULL_MASK, pred);
            const int pos = n_in + __popc(m & lt);
            if (pred && pos < list_cap) list[pos] = p;
            n_in += __popc(m);
          }
        }
      }
    }
    if (nfar > 0) {
      const int lo = far_lower_bound(far_keys, nfar, (unsigned long long)(unsigned)c << 32);
      const int hi = far_lower_bound(far_keys, nfar, (unsigned long long)(unsigned)(c + 1) << 32);
      __syncwarp();
      if (hi > lo && lane == 0) {
        int m = n_in < list_cap ? n_in : list_cap;
        for (int k = lo; k < hi; ++k) {
          const int p = (int)(far_keys[k] & 0xffffffffu);
          if (p < 0 || p >= (int)cap) continue;
          int j = m - 1;
          while (j >= 0 && list[j] > p) {
            if (j + 1 < list_cap) list[j + 1] = list[j];
            --j;
          }
          if (j + 1 < list_cap) list[j + 1] = p;
          if (m < list_cap) ++m;
        }
      }
      n_in += hi - lo;
      __syncwarp();
    }
    if (n_in > list_cap) {
      if (lane == 0) atomicExch(counters + CNT_LIST_OVERFLOW, 1);
      n_in = list_cap;
    }
    const DevInst& I = inst[__ldg(cell_inst + c)];
    const int q0 = I.q[0], q1 = I.q[1], q2 = DIM == 3 ? I.q[2] : 1;
    const int nb1 = q1 + 1, nb2 = q2 + 1;
    const double h0 = I.h[0], h1 = I.h[1], h2 = I.h[2];
    int n_keep = n_in, n_new = 0;
    if (CHECK) {
      const int nb = (q0 + 1) * nb1 * nb2;
      for (int k = lane; k < nb; k += 32) bcnt[k] = 0;
      __syncwarp();
      n_keep = 0;
      for (int base = 0; base < n_in; base += 32) {
        const int i = base + lane;
        const bool active = i < n_in;
        const int p = active ? list[i] : -1;
        int bi = -1;
        if (active) {
          const int b0 = sub_bucket<R>(oxi[p], h0, q0);
          const int b1 = sub_bucket<R>(oxi[cap + p], h1, q1);
          const int b2 = DIM == 3 ? sub_bucket<R>(oxi[2 * cap + p], h2, q2) : 0;
          bi = (b0 * nb1 + b1) * nb2 + b2;
        }
        const unsigned peers = __match_any_sync(PFEM2_FULL_MASK, bi);
        bool keep = false;
        int prev = 0;
        if (active) prev = bcnt[bi];
        __syncwarp();
        if (active) {
          keep = prev + __popc(peers & lt) + 1 <= I.max_per_part;
          if ((peers & lt) == 0) bcnt[bi] = prev + __popc(peers);
        }
        const unsigned km = __ballot_sync(PFEM2_FULL_MASK, keep);
        const int kpos = n_keep + __popc(km & lt);
        __syncwarp();
        if (keep) list[kpos] = p;
        n_keep += __popc(km);
        __syncwarp();
      }
      // empty sub-cells -> new particles, (i,j,k) order
      const int Q = q0 * q1 * q2;
      for (int base = 0; base < Q; base += 32) {
        const int t = base + lane;
        bool e = false;
        if (t < Q) {
          int ijk[3];
          sub_cell_ijk(t, q1, q2, I.qm, ijk);
          const int i0 = ijk[0], i1 = ijk[1], i2 = ijk[2];
          e = bcnt[(i0 * nb1 + i1) * nb2 + i2] == 0;
        }
        const unsigned em = __ballot_sync(PFEM2_FULL_MASK, e);
        const int pos = n_keep + n_new + __popc(em & lt);
        if (e && pos < list_cap) list[pos] = -1 - t;
        n_new += __popc(em);
      }
      if (n_keep + n_new > list_cap) {
        if (lane == 0) atomicExch(counters + CNT_LIST_OVERFLOW, 1);
        n_new = list_cap - n_keep;
      }
      __syncwarp();
    }
      ntot = n_keep + n_new;
      if (CHECK && lane == 0) {
        if (n_in - n_keep) atomicAdd(counters + CNT_REMOVED, n_in - n_keep);
        if (n_new) atomicAdd(counters + CNT_RESEEDED, n_new);
      }
    }
    if (lane == 0) s_cnt[warp] = ntot;
    __syncthreads();
    if (warp == 0) {
      unsigned long long agg = 0;
      for (int w = 0; w < kRebinWarps; ++w) agg += (unsigned)s_cnt[w];
      unsigned long long excl = 0;
      if (t == 0) {
        if (lane == 0) atomicExch(status, kTilePre | agg);
      } else {
        if (lane == 0) atomicExch(status + t, kTileAgg | agg);
        // look back over windows of 32 predecessors (lane k reads tile
        // j - k): the window ends at the nearest tile with a published
        // prefix; the tiles before it must have published their aggregates
        int j = t - 1;
        unsigned spins = 0;
        for (;;) {
          const int k = j - lane;
          const unsigned long long wd =
              k >= 0 ? *(volatile const unsigned long long*)(status + k) : kTilePre;  // before tile 0: prefix 0
          const unsigned pre = __ballot_sync(PFEM2_FULL_MASK, (wd >> 62) == 2);
          const unsigned wait = __ballot_sync(PFEM2_FULL_MASK, (wd >> 62) == 0);
          const int lp = pre ? __ffs(pre) - 1 : 31;
          const unsigned upto = lp == 31 ? PFEM2_FULL_MASK : (2u << lp) - 1u;
          if (wait & upto) {
            if (++spins > spin_limit) {
              if (lane == 0) atomicExch(counters + CNT_SCAN_TIMEOUT, 1);
              break;
            }
            __nanosleep(32);
            continue;
          }
          excl += warp_sum((unsigned long long)(lane <= lp ? (wd & kTileVal) : 0ull));
          if (pre) break;
          j -= 32;
        }
        if (lane == 0) atomicExch(status + t, kTilePre | ((excl + agg) & kTileVal));
      }
      if (lane == 0) s_base = (int)excl;
    }
    __syncthreads();
    if (c < nc) {
      int out = s_base;
      for (int w = 0; w < warp; ++w) out += s_cnt[w];
      if (lane == 0) {
        new_start[c] = out;
        if (c == nc - 1) {
          new_start[nc] = out + ntot;
          *np_out = out + ntot;
        }
      }
      const DevInst& I = inst[__ldg(cell_inst + c)];
      const int q1 = I.q[1], q2 = DIM == 3 ? I.q[2] : 1;
      const double h0 = I.h[0], h1 = I.h[1], h2 = I.h[2];
      ProjAcc<DIM, R> acc;
      if (PROJ) {
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int k = 0; k <= DIM; ++k) acc.a[v][k] = R(0);
      }
      for (int j = lane; j < ntot; j += 32) {
        const int code = list[j];
        R x[DIM], uu[DIM];
        if (code >= 0) {
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            x[d] = oxi[d * cap + code];
            uu[d] = ou[d * cap + code];
          }
        } else {
          const int t = -1 - code;
          int id[3];
          sub_cell_ijk(t, q1, q2, I.qm, id);
          const double hh[3] = {h0, h1, h2};
#pragma unroll
          for (int d = 0; d < DIM; ++d) x[d] = R((id[d] + 1.0 / 2) * hh[d]);
          R N[NV];
          shape_values<DIM, R>(x, N);
#pragma unroll
          for (int d = 0; d < DIM; ++d) uu[d] = R(0);
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            const int g = __ldg(cv + (size_t)c * NV + v);
#pragma unroll
            for (int d = 0; d < DIM; ++d) uu[d] = uu[d] + N[v] * Vr[(size_t)d * nv + g];
          }
        }
        const size_t o = (size_t)out + j;
        if (o < cap) {
          ncell[o] = c;
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            nxi[d * cap + o] = x[d];
            nu[d * cap + o] = uu[d];
          }
        }
        if (PROJ) proj_add<DIM, R>(acc, x, uu);
      }
      if (PROJ) proj_store<DIM, R>(acc, partial, c, lane);
    }
    __syncwarp();
    __syncthreads();
  }
}

template <int DIM, typename R, bool CHECK, bool PROJ>
static void rebin_launch(Ctx& c, const int* newcell) {
  const int o = c.cur, nb = 1 - c.cur;
  const size_t smem = (size_t)kRebinWarps * (c.list_cap + kMaxBuckets) * sizeof(int);
  const int ntiles = (c.nc + kRebinWarps - 1) / kRebinWarps;
  const int grid = grid_for(c, (long long)c.nc * 32, kRebinWarps * 32, c.tune.rebin_blocks_per_sm);
  cudaMemsetAsync(c.rebin_tiles, 0, sizeof(unsigned long long) * ((size_t)ntiles + 1), c.stream);
  k_rebin<DIM, R, CHECK, PROJ><<<grid, kRebinWarps * 32, smem, c.stream>>>(
      c.cell_start[o], newcell, (const R*)c.pxi[o], (const R*)c.pu[o], (size_t)c.pcap, c.pcell[nb], (R*)c.pxi[nb],
      (R*)c.pu[nb], c.cell_start[nb], c.d_np + nb, c.nc, c.ring_ptr, c.ring_cell, c.ring_rev, c.dest_mask, c.far_keys,
      c.far_cap, c.d_inst,
      c.cell_inst, c.cv, (const R*)c.Vr, c.nv, (R*)c.partial, c.list_cap, c.d_counters, c.rebin_tiles,
      c.spin_limit >> 2);
  c.launches += 1;
  c.cur = nb;
}

template <int DIM, typename R>
static pfem2_status rebin_impl(Ctx& c, bool check, bool proj, bool from_advect) {
  const int* nc_arr = from_advect ? c.newcell : c.pcell[c.cur];
  const size_t smem = (size_t)kRebinWarps * (c.list_cap + kMaxBuckets) * sizeof(int);
  auto set_attr = [&](const void* f) { cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); };
  if (check && proj) {
    set_attr((const void*)k_rebin<DIM, R, true, true>);
    rebin_launch<DIM, R, true, true>(c, nc_arr);
  } else if (check) {
    set_attr((const void*)k_rebin<DIM, R, true, false>);
    rebin_launch<DIM, R, true, false>(c, nc_arr);
  } else if (proj) {
    set_attr((const void*)k_rebin<DIM, R, false, true>);
    rebin_launch<DIM, R, false, true>(c, nc_arr);
  } else {
    set_attr((const void*)k_rebin<DIM, R, false, false>);
    rebin_launch<DIM, R, false, false>(c, nc_arr);
  }
  return PFEM2_OK;
}

pfem2_status launch_rebin(Ctx& c, bool check, bool proj, bool from_advect) {
  if (!from_advect) {
    // no movers: make sure the far list is empty
    PFEM2_CUDA(cudaMemsetAsync(c.d_counters + CNT_FAR, 0, sizeof(int), c.stream));
  }
  if (c.dim == 2) return c.pmixed ? rebin_impl<2, float>(c, check, proj, from_advect) : rebin_impl<2, double>(c, check, proj, from_advect);
  return c.pmixed ? rebin_impl<3, float>(c, check, proj, from_advect) : rebin_impl<3, double>(c, check, proj, from_advect);
}

// --------------------------------------------------------------- project
template <int DIM, typename R>
__global__ void __launch_bounds__(256) k_project_cells(const int* __restrict__ cell_start, const R* __restrict__ xi,
                                                       const R* __restrict__ u, size_t cap, int nc,
                                                       R* __restrict__ partial) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int c = blockIdx.x * wpb + warp; c < nc; c += gridDim.x * wpb) {
    const int b = min(cell_start[c], (int)cap), n = min(cell_start[c + 1], (int)cap) - b;
    ProjAcc<DIM, R> acc;
#pragma unroll
    for (int v = 0; v < Dims<DIM>::NV; ++v)
#pragma unroll
      for (int k = 0; k <= DIM; ++k) acc.a[v][k] = R(0);
    for (int j = lane; j < n; j += 32) {
      R x[DIM], uu[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        x[d] = xi[d * cap + b + j];
        uu[d] = u[d * cap + b + j];
      }
      proj_add<DIM, R>(acc, x, uu);
    }
    proj_store<DIM, R>(acc, partial, c, lane);
  }
}

// node gather: u_n = sum_k N u / sum_k N over the cells around node n, in
// ascending cell order (deterministic, no float atomics)
template <int DIM, typename R>
__global__ void __launch_bounds__(256) k_project_nodes(int nv, const int* __restrict__ v2c_ptr,
                                                       const int* __restrict__ v2c_cell,
                                                       const unsigned char* __restrict__ v2c_loc,
                                                       const R* __restrict__ partial,
                                                       const unsigned char* __restrict__ zero_flag,
                                                       double* __restrict__ V0, double* __restrict__ V1,
                                                       double* __restrict__ V2, double* __restrict__ W,
                                                       R* __restrict__ Vr, int* __restrict__ counters,
                                                       double* __restrict__ wall_dv) {
  constexpr int K = Dims<DIM>::NV * (DIM + 1);
  double* V[3] = {V0, V1, V2};
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    R s[DIM + 1];
#pragma unroll
    for (int k = 0; k <= DIM; ++k) s[k] = R(0);
    const int k1 = v2c_ptr[v + 1];
    for (int k = v2c_ptr[v]; k < k1; ++k) {
      const R* pp = partial + (size_t)v2c_cell[k] * K + v2c_loc[k] * (DIM + 1);
#pragma unroll
      for (int q = 0; q <= DIM; ++q) s[q] += pp[q];
    }
    const R w = s[DIM];
    const bool z = zero_flag[v] != 0;
    if (w == R(0) && k1 > v2c_ptr[v]) atomicAdd(counters + CNT_ZERO_WEIGHT, 1);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      R val = (w != R(0)) ? s[d] / w : R(0);
      if (z) {
        if (wall_dv) wall_dv[(size_t)d * nv + v] = (double)val;  // for the wall push-back
        val = R(0);
      }
      V[d][v] = (double)val;
      Vr[(size_t)d * nv + v] = val;
    }
    W[v] = (double)w;
  }
}

// Wall push-back after the projection (nacaAirfoil/pfem2particle.cpp:
// 919-952): a warp per cell touching a zero-flag vertex; every particle of
// the cell loses N_v(xi_p) times the projected velocity of each such vertex v
// whose velocity has a component above 1e-5 in magnitude (vertices in
// ascending local order, FP64 products).
template <int DIM, typename R>
__global__ void __launch_bounds__(256) k_wall_pushback(int ncells, const int* __restrict__ cells,
                                                       const int* __restrict__ cell_start, const int* __restrict__ cv,
                                                       const unsigned char* __restrict__ zero_flag,
                                                       const double* __restrict__ dv, int nv,
                                                       const R* __restrict__ xi, R* __restrict__ u, size_t cap) {
  constexpr int NV = Dims<DIM>::NV;
  const int lane = threadIdx.x & 31;
  for (int wc = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5); wc < ncells;
       wc += (int)((gridDim.x * (size_t)blockDim.x) >> 5)) {
    const int c = cells[wc];
    double d[NV][DIM];
    bool on[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const int g = __ldg(cv + (size_t)c * NV + v);
      on[v] = false;
#pragma unroll
      for (int a = 0; a < DIM; ++a) d[v][a] = 0.0;
      if (zero_flag[g]) {
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          d[v][a] = dv[(size_t)a * nv + g];
          on[v] |= fabs(d[v][a]) > 1e-5;
        }
      }
    }
    const int p1 = cell_start[c + 1];
    for (int p = cell_start[c] + lane; p < p1; p += 32) {
      double x[DIM], N[NV];
#pragma unroll
      for (int a = 0; a < DIM; ++a) x[a] = (double)xi[(size_t)a * cap + p];
      shape_values<DIM, double>(x, N);
      double uu[DIM];
#pragma unroll
      for (int a = 0; a < DIM; ++a) uu[a] = (double)u[(size_t)a * cap + p];
#pragma unroll
      for (int v = 0; v < NV; ++v)
        if (on[v])
#pragma unroll
          for (int a = 0; a < DIM; ++a) uu[a] -= N[v] * d[v][a];
#pragma unroll
      for (int a = 0; a < DIM; ++a) u[(size_t)a * cap + p] = R(uu[a]);
    }
  }
}

template <int DIM, typename R>
static pfem2_status project_impl(Ctx& c, bool partials_ready) {
  const int b = c.cur;
  if (!partials_ready) {
    k_project_cells<DIM, R><<<grid_for(c, (long long)c.nc * 32, 256, 8), 256, 0, c.stream>>>(
        c.cell_start[b], (const R*)c.pxi[b], (const R*)c.pu[b], (size_t)c.pcap, c.nc, (R*)c.partial);
    c.launches++;
  }
  k_project_nodes<DIM, R><<<grid_for(c, c.nv, 256, 8), 256, 0, c.stream>>>(
      c.nv, c.v2c_ptr, c.v2c_cell, c.v2c_loc, (const R*)c.partial, c.zero_flag, c.F[PFEM2_FIELD_VX],
      c.F[PFEM2_FIELD_VY], c.dim == 3 ? c.F[PFEM2_FIELD_VZ] : c.F[PFEM2_FIELD_VZ], c.F[PFEM2_FIELD_NODE_WEIGHT],
      (R*)c.Vr, c.d_counters, c.wall_dv);
  c.launches++;
  if (c.n_wall_cells > 0) {
    k_wall_pushback<DIM, R><<<grid_for(c, (long long)c.n_wall_cells * 32, 256, 8), 256, 0, c.stream>>>(
        c.n_wall_cells, c.wall_cells, c.cell_start[b], c.cv, c.zero_flag, c.wall_dv, c.nv, (const R*)c.pxi[b],
        (R*)c.pu[b], (size_t)c.pcap);
    c.launches++;
  }
  return PFEM2_OK;
}

pfem2_status launch_project(Ctx& c, bool partials_ready) {
  if (c.dim == 2) return c.pmixed ? project_impl<2, float>(c, partials_ready) : project_impl<2, double>(c, partials_ready);
  return c.pmixed ? project_impl<3, float>(c, partials_ready) : project_impl<3, double>(c, partials_ready);
}

// -------------------------------------------------- particle state access
template <int DIM, typename R>
__global__ void k_pack_out(const int* __restrict__ cell, const R* __restrict__ xi, const R* __restrict__ u,
                           size_t cap, int p0, int n, int c_off, int* __restrict__ ocell, double* __restrict__ oxi,
                           double* __restrict__ ou) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const size_t p = (size_t)p0 + j;
    ocell[j] = cell[p] - c_off;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      oxi[(size_t)j * DIM + d] = (double)xi[d * cap + p];
      ou[(size_t)j * DIM + d] = (double)u[d * cap + p];
    }
  }
}

template <int DIM, typename R>
static pfem2_status read_impl(Ctx& c, int instance, int* cell, double* xi, double* u, int* n_out) {
  const int b = c.cur;
  const HostInst& in = c.inst[instance];
  int se[2];
  PFEM2_CUDA(cudaMemcpyAsync(&se[0], c.cell_start[b] + in.c_off, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(&se[1], c.cell_start[b] + in.c_off + in.nc, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  const int n = se[1] - se[0];
  *n_out = n;
  if (!cell) return PFEM2_OK;
  if (n == 0) return PFEM2_OK;
  int* dc;
  double *dx, *du;
  PFEM2_CUDA(cudaMallocAsync(&dc, sizeof(int) * n, c.stream));
  PFEM2_CUDA(cudaMallocAsync(&dx, sizeof(double) * n * DIM, c.stream));
  PFEM2_CUDA(cudaMallocAsync(&du, sizeof(double) * n * DIM, c.stream));
  k_pack_out<DIM, R><<<grid_for(c, n, 256), 256, 0, c.stream>>>(c.pcell[b], (const R*)c.pxi[b], (const R*)c.pu[b],
                                                               (size_t)c.pcap, se[0], n, in.c_off, dc, dx, du);
  c.launches++;
  PFEM2_CUDA(cudaMemcpyAsync(cell, dc, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(xi, dx, sizeof(double) * n * DIM, cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(u, du, sizeof(double) * n * DIM, cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaFreeAsync(dc, c.stream));
  PFEM2_CUDA(cudaFreeAsync(dx, c.stream));
  PFEM2_CUDA(cudaFreeAsync(du, c.stream));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  return PFEM2_OK;
}

pfem2_status read_particles(Ctx& c, int instance, int* cell, double* xi, double* u, int* n) {
  if (c.dim == 2) return c.pmixed ? read_impl<2, float>(c, instance, cell, xi, u, n) : read_impl<2, double>(c, instance, cell, xi, u, n);
  return c.pmixed ? read_impl<3, float>(c, instance, cell, xi, u, n) : read_impl<3, double>(c, instance, cell, xi, u, n);
}

// unsorted particles in, stable sort by cell through the rebin machinery:
// the particles are first placed one per "virtual old segment" (all in the
// segment of their own cell, in input order) and then rebinned without check.
template <int DIM, typename R>
__global__ void k_unpack_in(int n, const int* __restrict__ pos, const int* __restrict__ icell,
                            const double* __restrict__ ixi, const double* __restrict__ iu, int* __restrict__ cell,
                            R* __restrict__ xi, R* __restrict__ u, size_t cap) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const size_t p = pos[j];
    cell[p] = icell[j];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      xi[d * cap + p] = R(ixi[(size_t)j * DIM + d]);
      u[d * cap + p] = R(iu[(size_t)j * DIM + d]);
    }
  }
}

template <int DIM, typename R>
static pfem2_status set_impl(Ctx& c, const int* counts, const int* cell, const double* xi, const double* u) {
  // host-side stable placement by cell (a state-loading utility, not the step)
  size_t n = 0;
  for (size_t i = 0; i < c.inst.size(); ++i) n += counts[i];
  if (n > (size_t)c.pcap) {
    set_error("set_particles: capacity exceeded");
    return PFEM2_PARTICLE_OVERFLOW;
  }
  std::vector<int> gcell(n), cnt(c.nc + 1, 0), pos(n);
  size_t k = 0;
  for (size_t i = 0; i < c.inst.size(); ++i)
    for (int j = 0; j < counts[i]; ++j, ++k) {
      int lc = cell[k];
      if (lc < 0 || lc >= c.inst[i].nc) {
        set_error("set_particles: cell out of range");
        return PFEM2_INVALID_ARG;
      }
      for (int d = 0; d < DIM; ++d)
        if (!std::isfinite(xi[k * DIM + d]) || !std::isfinite(u[k * DIM + d])) {
          set_error("set_particles: a coordinate or velocity is not finite");
          return PFEM2_INVALID_ARG;
        }
      gcell[k] = lc + c.inst[i].c_off;
      cnt[gcell[k] + 1]++;
    }
  for (int i = 0; i < c.nc; ++i) cnt[i + 1] += cnt[i];
  std::vector<int> start(cnt.begin(), cnt.end());
  for (size_t j = 0; j < n; ++j) pos[j] = cnt[gcell[j]]++;
  const int b = c.cur;
  int *dpos, *dcell;
  double *dxi, *du;
  size_t nn = n ? n : 1;
  PFEM2_CUDA(cudaMalloc(&dpos, sizeof(int) * nn));
  PFEM2_CUDA(cudaMalloc(&dcell, sizeof(int) * nn));
  PFEM2_CUDA(cudaMalloc(&dxi, sizeof(double) * nn * DIM));
  PFEM2_CUDA(cudaMalloc(&du, sizeof(double) * nn * DIM));
  PFEM2_CUDA(cudaMemcpy(dpos, pos.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  PFEM2_CUDA(cudaMemcpy(dcell, gcell.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  PFEM2_CUDA(cudaMemcpy(dxi, xi, sizeof(double) * n * DIM, cudaMemcpyHostToDevice));
  PFEM2_CUDA(cudaMemcpy(du, u, sizeof(double) * n * DIM, cudaMemcpyHostToDevice));
  if (n) {
    k_unpack_in<DIM, R><<<grid_for(c, n, 256), 256, 0, c.stream>>>((int)n, dpos, dcell, dxi, du, c.pcell[b],
                                                                 (R*)c.pxi[b], (R*)c.pu[b], (size_t)c.pcap);
    c.launches++;
  }
  PFEM2_CUDA(cudaMemcpyAsync(c.cell_start[b], start.data(), sizeof(int) * (c.nc + 1), cudaMemcpyHostToDevice, c.stream));
  int nint = (int)n;
  PFEM2_CUDA(cudaMemcpyAsync(c.d_np + b, &nint, sizeof(int), cudaMemcpyHostToDevice, c.stream));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  cudaFree(dpos); cudaFree(dcell); cudaFree(dxi); cudaFree(du);
  PFEM2_CUDA(cudaGetLastError());
  return PFEM2_OK;
}

pfem2_status launch_set_particles(Ctx& c, const int* counts, const int* cell, const double* xi, const double* u) {
  if (c.dim == 2) return c.pmixed ? set_impl<2, float>(c, counts, cell, xi, u) : set_impl<2, double>(c, counts, cell, xi, u);
  return c.pmixed ? set_impl<3, float>(c, counts, cell, xi, u) : set_impl<3, double>(c, counts, cell, xi, u);
}

}  // namespace pfem2
