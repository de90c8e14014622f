// krylov.cu -- batched, persistent preconditioned CG with FP64 reliable
// updates on the SELL-32 pattern (sm_100a).
//
// One cooperative launch solves every system of a solve phase (components x
// instances) to the reference's stopping rule: the absolute 2-norm of the
// unpreconditioned residual b - A x <= tol within max_iter iterations
// (deal.II SolverControl(max_iter, tol), cylinder2D/cylinder2D.cc:736-779).
// The reference runs BiCGStab with Jacobi (velocity) / SSOR (pressure); the
// prediction, mass and Poisson matrices here are symmetric positive definite
// after the symmetric Dirichlet elimination, so CG reaches the same solution.
//
// Each CG iteration is two phases separated by a bounded grid barrier:
//   A  p' = z + beta p ; q = A (z + beta p)     (p double buffered)  | (p', q)
//   B  e += alpha p' ; r -= alpha q ; z = M^-1 r                    | (r, z), (r, r), sum r
// Every block that owns tiles of a system computes that system's scalars
// itself, from the per-tile partial sums of the previous phase, in a fixed
// order: no block publishes scalars and no phase waits for a finalizer.
//
// Preconditioners: Jacobi for the prediction and mass systems; for the
// pressure Poisson system an additive two-level preconditioner
//   M^-1 = B^-1 + Z E^-1 Z^T,
// B = the 32x32 diagonal blocks of A (one SELL slice = one warp, inverted at
// setup, applied with warp shuffles), Z = indicator vectors of the tiles of
// the system (contiguous runs of slices), E = Z^T A Z (inverted at setup,
// FP32 copy in shared memory). The coarse part needs the tile sums of r,
// which are partials of phase B anyway, so it is applied on the fly in
// phase A (z_i = (B^-1 r)_i + y_tile(i), y = E^-1 Z^T r) and costs no
// extra barrier.
//
// The iterate is split x + e: e accumulates in the inner type R (FP32 for
// the mixed path, FP64 for the plain path); once the recurrence residual
// has dropped below max(eta * res, tol / 2) a reliable update runs in FP64
// (phase A: r64 = b - A64 (x + e); phase B: x += e, e = 0, r = r64) and CG
// restarts from the true residual. A system is done when the FP64 residual
// is <= tol.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "ctx.h"

namespace pfem2 {

constexpr int kSolveThreads = 384;  // 12 warps
constexpr int kWarps = kSolveThreads / 32;
constexpr int kMaxLocalSys = 16;

// system states (A states act in even iterations, B states in odd ones)
enum { S_OUT_A = 0, S_OUT_B = 1, S_A = 2, S_B = 3, S_DONE = 4 };
// actions
enum { ACT_NONE = 0, ACT_OUT_A = 1, ACT_OUT_B = 2, ACT_OUT_DONE = 3, ACT_A = 4, ACT_B = 5 };

template <typename R> struct SolveArgs {
  int ncomp, ninst, nsys, ntiles, nv;
  const Tile* tiles;
  const int* sys_t0;     // [nsys+1] first tile of each system
  const int* blk_t0;     // [grid+1] first tile of each block
  const int* sl_ptr;
  const int* sl_len;
  const int* sl_col;
  const double* A64[3];
  const R* Ain[3];
  const R* dinv[3];
  // two-level data (pressure phase)
  const R* Binv;         // [nslices][32 cols][32 rows]
  const float* Einv;     // per system D_s x D_s (symmetric), at sys_eoff[s]
  const int* sys_eoff;
  const int* sys_D;      // coarse size = tiles of the system
  const int* sys_sl0;    // first slice of the system
  const int* sys_sps;    // slices per tile (= per coarse subdomain)
  int dmax;              // max D over systems (smem stride)
  int binv_smem;         // 1: this block's B^-1 slices are staged in shared memory
  double* x[3];
  const double* b[3];
  const unsigned char* isd[3];
  const double* g[3];    // Dirichlet values preset in x (nullptr -> 0)
  const double* tol_i;   // per instance
  const int* maxit_i;    // per instance
  // workspace per component slot, nv entries each
  R *e, *r, *z, *p, *q;  // p: 2 buffers; z = B^-1 r (two-level) or D^-1 r
  double* r64;
  double* part;          // [2][ntiles][3], by iteration parity
  int* active;
  int* out_it;           // [nsys] iterations
  double* out_res;       // [nsys] final residual norm
  int* out_outer;        // [nsys] FP64 residual evaluations
  double eta;
  int iter_cap;
  GridBarrier gb;
  unsigned long long* prof;  // optional: ns spent per sub-phase by block 0 (PFEM2_SOLVER_PROFILE)
};

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct LocalSys {
  int sys, state, it, outer, par, first, owner, maxit, act;
  int D, sl0, sps;
  double tol, intol, res, rz_prev, alpha, beta, rzc;
  double sum[2];
};

// z = B^-1 r on one SELL slice: lane i holds r_i, returns z_i
template <typename R>
__device__ __forceinline__ R block_jacobi32(const R* __restrict__ Binv, int slice, R ri, int lane) {
  const R* B = Binv + (size_t)slice * 1024;
  R acc = R(0);
#pragma unroll 8
  for (int j = 0; j < 32; ++j) acc += B[j * 32 + lane] * __shfl_sync(PFEM2_FULL_MASK, ri, j);
  return acc;
}

template <typename R, bool TWO>
__global__ void __launch_bounds__(kSolveThreads) k_krylov(SolveArgs<R> a) {
  extern __shared__ unsigned char dyn_smem[];
  __shared__ LocalSys ls[kMaxLocalSys];
  __shared__ double red[kWarps][2];
  __shared__ int s_nls, s_sys0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t nv = (size_t)a.nv;
  const int t_lo = a.blk_t0[blockIdx.x], t_hi = a.blk_t0[blockIdx.x + 1];
  unsigned bar_gen = 0;
  // two-level shared memory: per local system E^-1 (dmax^2 floats), y and Z^T r (dmax doubles each)
  float* sE = reinterpret_cast<float*>(dyn_smem);
  const int nE = a.dmax * a.dmax;

  // ---- local systems of this block
  if (threadIdx.x == 0) {
    int n = 0, s0 = -1;
    if (t_hi > t_lo) {
      s0 = a.tiles[t_lo].sys;
      n = a.tiles[t_hi - 1].sys - s0 + 1;
    }
    if (n > kMaxLocalSys) n = kMaxLocalSys;  // the host guarantees n <= kMaxLocalSys
    s_nls = n;
    s_sys0 = s0;
    for (int k = 0; k < n; ++k) {
      LocalSys& L = ls[k];
      const int s = s0 + k, inst = s % a.ninst;
      L.sys = s;
      L.state = S_OUT_A;
      L.it = L.outer = L.par = 0;
      L.first = 1;
      L.owner = a.sys_t0[s] >= t_lo && a.sys_t0[s] < t_hi;
      L.maxit = a.maxit_i[inst];
      L.tol = a.tol_i[inst];
      L.intol = 0.5 * L.tol;
      L.res = L.rz_prev = L.alpha = L.beta = L.rzc = 0.0;
      L.act = ACT_NONE;
      if (TWO) {
        L.D = a.sys_D[s];
        L.sl0 = a.sys_sl0[s];
        L.sps = a.sys_sps[s];
      } else {
        L.D = 0; L.sl0 = 0; L.sps = 1;
      }
    }
  }
  __syncthreads();
  const int nls = s_nls, sys0 = s_sys0;
  float* sEk[kMaxLocalSys];
  double* sYk[kMaxLocalSys];
  double* sSk[kMaxLocalSys];
  const R* Bsrc = a.Binv;  // B^-1 of slice s at Bsrc + (s - bsl0) * 1024
  int bsl0 = 0;
  if (TWO) {
    double* ybase = reinterpret_cast<double*>(sE + (size_t)nls * nE + ((nls * nE) & 1));
    for (int k = 0; k < nls; ++k) {
      sEk[k] = sE + (size_t)k * nE;
      sYk[k] = ybase + (size_t)k * 3 * a.dmax;
      sSk[k] = sYk[k] + 2 * a.dmax;
      const float* src = a.Einv + a.sys_eoff[ls[k].sys];
      const int n2 = ls[k].D * ls[k].D;
      for (int i = threadIdx.x; i < n2; i += kSolveThreads) sEk[k][i] = src[i];
    }
    if (a.binv_smem && t_hi > t_lo) {
      R* sB = reinterpret_cast<R*>(ybase + (size_t)nls * 3 * a.dmax);
      bsl0 = a.tiles[t_lo].s0;
      const int nsl = a.tiles[t_hi - 1].s1 - bsl0;
      const R* g = a.Binv + (size_t)bsl0 * 1024;
      for (int i = threadIdx.x; i < nsl * 1024; i += kSolveThreads) sB[i] = g[i];
      Bsrc = sB;
    }
  }

  // ---- init: Dirichlet values preset in x, e = 0, p = 0
  for (int t = t_lo; t < t_hi; ++t) {
    const Tile T = a.tiles[t];
    const int k = T.comp;
    for (int sl = T.s0 + warp; sl < T.s1; sl += kWarps) {
      const int row = sl * 32 + lane;
      if (a.isd[k][row]) a.x[k][row] = a.g[k] ? a.g[k][row] : 0.0;
      a.e[k * nv + row] = R(0);
      a.p[(2 * k) * nv + row] = R(0);
      a.p[(2 * k + 1) * nv + row] = R(0);
    }
  }
  bool stop = false;
  if (!grid_sync(a.gb, bar_gen)) return;

  const bool prof = a.prof != nullptr && blockIdx.x == 0 && threadIdx.x == 0;
  unsigned long long tp[6] = {0, 0, 0, 0, 0, 0}, tlast = prof ? gtimer() : 0;
#define PFEM2_PROF(k)                       \
  if (prof) {                               \
    const unsigned long long tn = gtimer(); \
    tp[k] += tn - tlast;                    \
    tlast = tn;                             \
  }
  for (int iter = 0;; ++iter) {
    if (stop) break;  // published by the last barrier: every system is done
    if (iter >= a.iter_cap) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(a.gb.err, 2);
      break;
    }
    const bool phaseA = (iter & 1) == 0;
    const double* prev = a.part + (size_t)((iter + 1) & 1) * a.ntiles * 3;
    PFEM2_PROF(5);
    // ---- Z^T r of the systems about to run phase A (warps 1..), loaded while
    // warp 0 sums the scalar partials
    if (TWO && phaseA && warp > 0) {
      for (int k = 0; k < nls; ++k) {
        if (ls[k].state != S_A) continue;
        const int D = ls[k].D, t0 = a.sys_t0[ls[k].sys];
        float* sf = reinterpret_cast<float*>(sYk[k] + a.dmax);
        for (int d = threadIdx.x - 32; d < D; d += kSolveThreads - 32) {
          const double v = __ldcg(prev + (size_t)(t0 + d) * 3 + 2);
          sSk[k][d] = v;
          sf[d] = (float)v;
        }
      }
    }
    // ---- sums of the previous phase's partials (warp 0, fixed order)
    if (warp == 0) {
      for (int k = 0; k < nls; ++k) {
        const int st = ls[k].state;
        if (st == S_DONE || st == S_OUT_A) continue;
        const int t0 = a.sys_t0[ls[k].sys], t1 = a.sys_t0[ls[k].sys + 1];
        double s0 = 0.0, s1 = 0.0;
#pragma unroll 4
        for (int t = t0 + lane; t < t1; t += 32) {
          s0 += __ldcg(prev + (size_t)t * 3);
          s1 += __ldcg(prev + (size_t)t * 3 + 1);
        }
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        if (lane == 0) {
          ls[k].sum[0] = s0;
          ls[k].sum[1] = s1;
        }
      }
    }
    __syncthreads();
    PFEM2_PROF(0);
    // ---- coarse correction y = E^-1 Z^T r for systems about to run phase A
    if (TWO && phaseA) {
      for (int k = 0; k < nls; ++k) {
        if (ls[k].state != S_A) continue;
        const int D = ls[k].D, t0 = a.sys_t0[ls[k].sys];
        const float* sf = reinterpret_cast<const float*>(sYk[k] + a.dmax);  // FP32 copy of Z^T r
        (void)t0;
        for (int j = threadIdx.x; j < D; j += kSolveThreads) {
          // y_j = sum_d E^-1[d][j] s_d (E^-1 symmetric: column reads are conflict free)
          const float* Ej = sEk[k] + j;
          float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
          int d = 0;
          for (; d + 3 < D; d += 4) {
            a0 = fmaf(Ej[(d + 0) * D], sf[d + 0], a0);
            a1 = fmaf(Ej[(d + 1) * D], sf[d + 1], a1);
            a2 = fmaf(Ej[(d + 2) * D], sf[d + 2], a2);
            a3 = fmaf(Ej[(d + 3) * D], sf[d + 3], a3);
          }
          for (; d < D; ++d) a0 = fmaf(Ej[d * D], sf[d], a0);
          sYk[k][j] = (double)((a0 + a1) + (a2 + a3));
        }
        __syncthreads();
        if (warp == 0) {
          double c = 0.0;
          for (int d = lane; d < D; d += 32) c += sSk[k][d] * sYk[k][d];
          c = warp_sum(c);
          if (lane == 0) ls[k].rzc = c;
        }
      }
    }
    __syncthreads();
    PFEM2_PROF(1);
    // ---- decisions (thread 0; identical in every block owning the system)
    if (threadIdx.x == 0) {
      for (int k = 0; k < nls; ++k) {
        LocalSys& L = ls[k];
        int act = ACT_NONE;
        if (phaseA) {
          if (L.state == S_OUT_A) {
            act = ACT_OUT_A;
            L.state = S_OUT_B;
          } else if (L.state == S_A) {
            const double rz = L.sum[0] + (TWO ? L.rzc : 0.0), rr = sqrt(L.sum[1]);
            if (rr <= L.intol || L.it >= L.maxit || !(rr == rr)) {
              act = ACT_OUT_A;  // reliable update in FP64
              L.state = S_OUT_B;
            } else {
              L.beta = L.first ? 0.0 : (L.rz_prev != 0.0 ? rz / L.rz_prev : 0.0);
              L.rz_prev = rz;
              L.first = 0;
              act = ACT_A;
              L.state = S_B;
            }
          }
        } else {
          if (L.state == S_OUT_B) {
            L.res = sqrt(L.sum[0]);
            L.outer += 1;
            if (L.res <= L.tol || L.it >= L.maxit || !(L.res == L.res)) {
              act = ACT_OUT_DONE;
              L.state = S_DONE;
            } else {
              L.intol = fmax(a.eta * L.res, 0.5 * L.tol);
              L.first = 1;  // CG restarts from the true residual
              act = ACT_OUT_B;
              L.state = S_A;
            }
          } else if (L.state == S_B) {
            L.alpha = L.sum[0] != 0.0 ? L.rz_prev / L.sum[0] : 0.0;
            L.it += 1;
            act = ACT_B;
            L.state = S_A;
          }
        }
        L.act = act;
      }
    }
    __syncthreads();
    PFEM2_PROF(2);
    // ---- work on the own tiles
    for (int t = t_lo; t < t_hi; ++t) {
      const Tile T = a.tiles[t];
      const int k = T.comp;
      const int lk = T.sys - sys0;
      const LocalSys& L = ls[lk];
      const int act = L.act;
      if (act == ACT_NONE) continue;
      double v0 = 0.0, v1 = 0.0, v2 = 0.0;
      const R* dinv = a.dinv[k];
      R* e = a.e + k * nv;
      R* r = a.r + k * nv;
      R* z = a.z + k * nv;
      R* q = a.q + k * nv;
      double* r64 = a.r64 + k * nv;
      if (act == ACT_OUT_A) {
        const double* A = a.A64[k];
        const double* xk = a.x[k];
        for (int sl = T.s0 + warp; sl < T.s1; sl += kWarps) {
          const int row = sl * 32 + lane;
          const int base = a.sl_ptr[sl], len = a.sl_len[sl];
          double acc = 0.0;
          for (int j = 0; j < len; ++j) {
            const int ei = base + j * 32 + lane;
            const int col = __ldg(a.sl_col + ei);
            acc += A[ei] * (__ldcg(xk + col) + (double)__ldcg(e + col));
          }
          const double rr = a.b[k][row] - acc;
          r64[row] = rr;
          v0 += rr * rr;
        }
      } else if (act == ACT_OUT_B || act == ACT_OUT_DONE) {
        for (int sl = T.s0 + warp; sl < T.s1; sl += kWarps) {
          const int row = sl * 32 + lane;
          a.x[k][row] += (double)e[row];
          e[row] = R(0);
          if (act == ACT_OUT_B) {
            const R rr = R(r64[row]);
            const R zz = TWO ? block_jacobi32<R>(Bsrc, sl - bsl0, rr, lane) : rr * dinv[row];
            r[row] = rr;
            z[row] = zz;
            v0 += (double)rr * (double)zz;
            v1 += (double)rr * (double)rr;
            v2 += (double)rr;
          }
        }
      } else if (act == ACT_A) {
        const R beta = R(L.beta);
        R* pn = a.p + (2 * k + L.par) * nv;
        const R* po = a.p + (2 * k + (L.par ^ 1)) * nv;
        const R* A = a.Ain[k];
        const double* y = TWO ? sYk[lk] : nullptr;
        for (int sl = T.s0 + warp; sl < T.s1; sl += kWarps) {
          const int row = sl * 32 + lane;
          const int base = a.sl_ptr[sl], len = a.sl_len[sl];
          R acc = R(0);
          for (int j = 0; j < len; ++j) {
            const int ei = base + j * 32 + lane;
            const int col = __ldg(a.sl_col + ei);
            R zc = __ldcg(z + col);
            if (TWO) zc += R(y[((col >> 5) - L.sl0) / L.sps]);
            acc += A[ei] * (zc + beta * __ldcg(po + col));
          }
          R zr = z[row];
          if (TWO) zr += R(y[(sl - L.sl0) / L.sps]);
          const R pp = zr + beta * po[row];
          pn[row] = pp;
          q[row] = acc;
          v0 += (double)pp * (double)acc;
        }
      } else if (act == ACT_B) {
        const R alpha = R(L.alpha);
        const R* pn = a.p + (2 * k + L.par) * nv;
        for (int sl = T.s0 + warp; sl < T.s1; sl += kWarps) {
          const int row = sl * 32 + lane;
          e[row] += alpha * pn[row];
          const R rr = r[row] - alpha * q[row];
          const R zz = TWO ? block_jacobi32<R>(Bsrc, sl - bsl0, rr, lane) : rr * dinv[row];
          r[row] = rr;
          z[row] = zz;
          v0 += (double)rr * (double)zz;
          v1 += (double)rr * (double)rr;
          v2 += (double)rr;
        }
      }
      // deterministic block reduction into this iteration's parity buffer
      v0 = warp_sum(v0);
      v1 = warp_sum(v1);
      v2 = warp_sum(v2);
      if (lane == 0) {
        red[warp][0] = v0;
        red[warp][1] = v1;
      }
      __shared__ double red2[kWarps];
      if (lane == 0) red2[warp] = v2;
      __syncthreads();
      if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int wv = 0; wv < kWarps; ++wv) {
          s0 += red[wv][0];
          s1 += red[wv][1];
          s2 += red2[wv];
        }
        double* dst = a.part + ((size_t)(iter & 1) * a.ntiles + t) * 3;
        dst[0] = s0;
        dst[1] = s1;
        dst[2] = s2;
      }
      __syncthreads();
    }
    PFEM2_PROF(3);
    // ---- bookkeeping
    if (threadIdx.x == 0) {
      for (int k = 0; k < nls; ++k) {
        LocalSys& L = ls[k];
        if (L.act == ACT_B) L.par ^= 1;
        if (L.act == ACT_OUT_DONE && L.owner) {
          a.out_it[L.sys] = L.it;
          a.out_res[L.sys] = L.res;
          a.out_outer[L.sys] = L.outer;
          atomicSub(a.active, 1);
        }
        L.act = ACT_NONE;
      }
    }
    PFEM2_PROF(3);
    if (!grid_sync(a.gb, bar_gen, a.active, &stop)) return;
    PFEM2_PROF(4);
  }
  if (prof)
    for (int k = 0; k < 6; ++k) atomicAdd(a.prof + k, tp[k]);
#undef PFEM2_PROF
}

// ------------------------------------------------------------------ host
struct KrylovWs {
  Tile* tiles[2];
  int* sys_t0[2];
  int* blk_t0[2];
  int ntiles[2], nsys[2], grid[2];
  std::vector<Tile> h_tiles0;
  std::vector<int> h_sys_t0_0;
  // two-level data of the pressure phase (phase 0)
  bool two_level = false;
  int dmax = 0, nls_max = 1;
  size_t smem_two = 0;
  int binv_smem = 0;
  void* Binv = nullptr;
  float* Einv = nullptr;
  int *sys_eoff = nullptr, *sys_D = nullptr, *sys_sl0 = nullptr, *sys_sps = nullptr;
  void *e = nullptr, *r = nullptr, *z = nullptr, *q = nullptr, *p = nullptr;
  double* r64 = nullptr;
  double* part = nullptr;
  int* active = nullptr;
  int* out_it[3];
  double* out_res[3];
  int* out_outer[3];
  unsigned long long* prof = nullptr;  // [3 solve kinds][6]
};

static int max_local_systems(const std::vector<Tile>& tiles, const std::vector<int>& bt0) {
  int worst = 0;
  for (size_t b = 0; b + 1 < bt0.size(); ++b)
    if (bt0[b + 1] > bt0[b]) worst = std::max(worst, tiles[bt0[b + 1] - 1].sys - tiles[bt0[b]].sys + 1);
  return worst;
}

template <typename R, bool TWO>
static int occupancy(size_t smem) {
  int occ = 0;
  // one process-wide upper bound, so contexts with different coarse sizes coexist
  if (TWO) cudaFuncSetAttribute((const void*)k_krylov<R, TWO>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_krylov<R, TWO>, kSolveThreads, smem) != cudaSuccess) return 0;
  return occ;
}

pfem2_status krylov_setup(Ctx& c) {
  KrylovWs* w = new KrylovWs();
  c.kws = w;
  const int dim = c.dim, ni = (int)c.inst.size();
  const size_t nv = c.nv;
  const size_t rs = c.mixed ? sizeof(float) : sizeof(double);
  const int bps = std::max(1, c.solve_blocks_per_sm);
  int maxtiles = 0, maxsys = 0;
  for (int ph = 0; ph < 2; ++ph) {
    const int ncomp = ph == 0 ? 1 : dim;
    std::vector<Tile> tiles;
    std::vector<int> st0(ncomp * ni + 1, 0);
    if (ph == 0) {
      // pressure: tiles = coarse subdomains; about one per block of the
      // persistent grid (balanced work), at most dcap per system
      // (a batch: subdomains of ~8 slices, at most dcap per system, so every
      // instance gets a coarse space of its own size)
      const int dcap = ni == 1 ? 160 : 96;
      const int nb = bps * c.num_sms;
      long long tot_sl = 0;
      for (int i = 0; i < ni; ++i) tot_sl += c.inst[i].nv_pad / kSlice;
      w->dmax = 1;
      for (int i = 0; i < ni; ++i) {
        st0[i] = (int)tiles.size();
        const int sl0 = c.inst[i].v_off / kSlice, nsl = c.inst[i].nv_pad / kSlice;
        const long long share = ni == 1 ? std::max<long long>(1, (long long)nb * nsl / tot_sl) : (nsl + 7) / 8;
        int D = (int)std::min<long long>(std::min<long long>(share, dcap), nsl);
        const int sps = (nsl + D - 1) / D;
        D = (nsl + sps - 1) / sps;
        for (int a = 0; a < nsl; a += sps) tiles.push_back(Tile{i, 0, sl0 + a, sl0 + std::min(nsl, a + sps)});
        w->dmax = std::max(w->dmax, D);
      }
      st0[ni] = (int)tiles.size();
    } else {
      const long long slices = (long long)c.nslices * ncomp;
      const long long target = 2LL * bps * c.num_sms;
      int ts = (int)std::max<long long>(8, (slices + target - 1) / target);
      if (c.tile_slices > 0) ts = c.tile_slices;
      for (int k = 0; k < ncomp; ++k)
        for (int i = 0; i < ni; ++i) {
          const int sidx = k * ni + i;
          st0[sidx] = (int)tiles.size();
          const int sl0 = c.inst[i].v_off / kSlice, sl1 = (c.inst[i].v_off + c.inst[i].nv_pad) / kSlice;
          for (int a = sl0; a < sl1; a += ts) tiles.push_back(Tile{sidx, k, a, std::min(sl1, a + ts)});
        }
      st0[ncomp * ni] = (int)tiles.size();
    }
    const int T = (int)tiles.size();
    int occ;
    size_t smem = 0;
    if (ph == 0) {
      // shared memory for the coarse inverses: sized after the chunking below,
      // first with one local system to bound the grid
      w->nls_max = 1;
      smem = (size_t)w->dmax * w->dmax * 4 + 8 + 3 * (size_t)w->dmax * 8;
      occ = c.mixed ? occupancy<float, true>(smem) : occupancy<double, true>(smem);
    } else {
      occ = c.mixed ? occupancy<float, false>(0) : occupancy<double, false>(0);
    }
    if (occ < 1) {
      set_error("krylov: the solver kernel cannot be resident");
      return PFEM2_CUDA_ERROR;
    }
    const int G = std::min(T, std::min(occ, bps) * c.num_sms);
    std::vector<int> bt0(G + 1);
    for (int b = 0; b <= G; ++b) bt0[b] = (int)((long long)T * b / G);
    const int nls = max_local_systems(tiles, bt0);
    if (nls > kMaxLocalSys) {
      set_error("krylov: more than 16 systems would share one block (instances too small for the batch)");
      return PFEM2_INVALID_ARG;
    }
    if (ph == 0) {
      w->nls_max = nls;
      w->smem_two = (size_t)nls * w->dmax * w->dmax * 4 + 8 + 3 * (size_t)nls * w->dmax * 8;
      int maxsl = 0;
      for (int b = 0; b < G; ++b)
        if (bt0[b + 1] > bt0[b]) maxsl = std::max(maxsl, tiles[bt0[b + 1] - 1].s1 - tiles[bt0[b]].s0);
      const size_t bj = (size_t)maxsl * 1024 * rs;
      if (w->smem_two + bj <= 220 * 1024) {
        w->smem_two += bj;
        w->binv_smem = 1;
      }
      if (w->smem_two > 220 * 1024) {
        set_error("krylov: coarse inverses of the pressure systems exceed shared memory");
        return PFEM2_INVALID_ARG;
      }
      const int occ2 = c.mixed ? occupancy<float, true>(w->smem_two) : occupancy<double, true>(w->smem_two);
      if (occ2 * c.num_sms < G) {
        set_error("krylov: the two-level solver grid cannot be resident");
        return PFEM2_CUDA_ERROR;
      }
      w->h_tiles0 = tiles;
      w->h_sys_t0_0 = st0;
    }
    w->ntiles[ph] = T;
    w->nsys[ph] = (int)st0.size() - 1;
    w->grid[ph] = G;
    PFEM2_CUDA(cudaMalloc(&w->tiles[ph], sizeof(Tile) * T));
    PFEM2_CUDA(cudaMemcpy(w->tiles[ph], tiles.data(), sizeof(Tile) * T, cudaMemcpyHostToDevice));
    PFEM2_CUDA(cudaMalloc(&w->sys_t0[ph], sizeof(int) * st0.size()));
    PFEM2_CUDA(cudaMemcpy(w->sys_t0[ph], st0.data(), sizeof(int) * st0.size(), cudaMemcpyHostToDevice));
    PFEM2_CUDA(cudaMalloc(&w->blk_t0[ph], sizeof(int) * bt0.size()));
    PFEM2_CUDA(cudaMemcpy(w->blk_t0[ph], bt0.data(), sizeof(int) * bt0.size(), cudaMemcpyHostToDevice));
    maxtiles = std::max(maxtiles, T);
    maxsys = std::max(maxsys, w->nsys[ph]);
  }
  void** vecs[] = {&w->e, &w->r, &w->z, &w->q};
  for (void** v : vecs) {
    PFEM2_CUDA(cudaMalloc(v, rs * nv * dim));
    PFEM2_CUDA(cudaMemset(*v, 0, rs * nv * dim));
  }
  PFEM2_CUDA(cudaMalloc(&w->p, rs * nv * dim * 2));
  PFEM2_CUDA(cudaMemset(w->p, 0, rs * nv * dim * 2));
  PFEM2_CUDA(cudaMalloc(&w->r64, sizeof(double) * nv * dim));
  PFEM2_CUDA(cudaMemset(w->r64, 0, sizeof(double) * nv * dim));
  PFEM2_CUDA(cudaMalloc(&w->part, sizeof(double) * 6 * maxtiles));
  PFEM2_CUDA(cudaMemset(w->part, 0, sizeof(double) * 6 * maxtiles));
  PFEM2_CUDA(cudaMalloc(&w->active, sizeof(int)));
  if (getenv("PFEM2_SOLVER_PROFILE")) {
    PFEM2_CUDA(cudaMalloc(&w->prof, sizeof(unsigned long long) * 18));
    PFEM2_CUDA(cudaMemset(w->prof, 0, sizeof(unsigned long long) * 18));
  }
  for (int k = 0; k < 3; ++k) {
    PFEM2_CUDA(cudaMalloc(&w->out_it[k], sizeof(int) * maxsys));
    PFEM2_CUDA(cudaMalloc(&w->out_res[k], sizeof(double) * maxsys));
    PFEM2_CUDA(cudaMalloc(&w->out_outer[k], sizeof(int) * maxsys));
    PFEM2_CUDA(cudaMemset(w->out_it[k], 0, sizeof(int) * maxsys));
    PFEM2_CUDA(cudaMemset(w->out_res[k], 0, sizeof(double) * maxsys));
    PFEM2_CUDA(cudaMemset(w->out_outer[k], 0, sizeof(int) * maxsys));
  }
  return PFEM2_OK;
}

// in-place inverse of an SPD matrix (Cholesky, then L^-T L^-1); false if not SPD
static bool spd_inverse(std::vector<double>& M, int n) {
  std::vector<double> L((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    double d = M[(size_t)j * n + j];
    for (int k = 0; k < j; ++k) d -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
    if (!(d > 0.0)) return false;
    d = std::sqrt(d);
    L[(size_t)j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double s = M[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) s -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
      L[(size_t)i * n + j] = s / d;
    }
  }
  // Linv (lower)
  std::vector<double> Li((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    Li[(size_t)j * n + j] = 1.0 / L[(size_t)j * n + j];
    for (int i = j + 1; i < n; ++i) {
      double s = 0.0;
      for (int k = j; k < i; ++k) s -= L[(size_t)i * n + k] * Li[(size_t)k * n + j];
      Li[(size_t)i * n + j] = s / L[(size_t)i * n + i];
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = 0.0;
      for (int k = i; k < n; ++k) s += Li[(size_t)k * n + i] * Li[(size_t)k * n + j];
      M[(size_t)i * n + j] = s;
      M[(size_t)j * n + i] = s;
    }
  return true;
}

// block-Jacobi inverses of the 32x32 slice blocks and the coarse inverses
// E^-1 = (Z^T A Z)^-1 of the pressure matrix (after Dirichlet elimination).
pfem2_status krylov_setup_precond(Ctx& c) {
  KrylovWs* w = (KrylovWs*)c.kws;
  const int ni = (int)c.inst.size();
  std::vector<double> A(c.nell);
  std::vector<int> col(c.nell), len(c.nslices);
  PFEM2_CUDA(cudaMemcpy(A.data(), c.A64[3], sizeof(double) * c.nell, cudaMemcpyDeviceToHost));
  PFEM2_CUDA(cudaMemcpy(col.data(), c.sl_col, sizeof(int) * c.nell, cudaMemcpyDeviceToHost));
  PFEM2_CUDA(cudaMemcpy(len.data(), c.sl_len, sizeof(int) * c.nslices, cudaMemcpyDeviceToHost));
  const std::vector<int>& sp = c.h_sl_ptr;
  // block Jacobi
  std::vector<double> B(1024);
  std::vector<double> bj64;
  std::vector<float> bj32;
  if (c.mixed) bj32.resize((size_t)c.nslices * 1024);
  else bj64.resize((size_t)c.nslices * 1024);
  for (int s = 0; s < c.nslices; ++s) {
    std::fill(B.begin(), B.end(), 0.0);
    for (int l = 0; l < 32; ++l)
      for (int j = 0; j < len[s]; ++j) {
        const int e = sp[s] + j * 32 + l;
        const int cc = col[e];
        if (cc / 32 == s) B[(size_t)l * 32 + (cc % 32)] += A[e];
      }
    if (!spd_inverse(B, 32)) {
      set_error("krylov: a diagonal block of the pressure matrix is not SPD");
      return PFEM2_MESH_ERROR;
    }
    for (int jj = 0; jj < 32; ++jj)
      for (int i = 0; i < 32; ++i) {
        const double v = B[(size_t)i * 32 + jj];
        if (c.mixed) bj32[(size_t)s * 1024 + jj * 32 + i] = (float)v;
        else bj64[(size_t)s * 1024 + jj * 32 + i] = v;
      }
  }
  const size_t bbytes = (size_t)c.nslices * 1024 * (c.mixed ? 4 : 8);
  PFEM2_CUDA(cudaMalloc(&w->Binv, bbytes));
  PFEM2_CUDA(cudaMemcpy(w->Binv, c.mixed ? (void*)bj32.data() : (void*)bj64.data(), bbytes, cudaMemcpyHostToDevice));
  // coarse inverses per system (tile = subdomain)
  const std::vector<Tile>& tiles = w->h_tiles0;
  const std::vector<int>& st0 = w->h_sys_t0_0;
  std::vector<int> eoff(ni), Dv(ni), sl0v(ni), spsv(ni);
  std::vector<float> Einv;
  std::vector<int> sub_of_slice(c.nslices, -1);
  for (int i = 0; i < ni; ++i) {
    const int t0 = st0[i], t1 = st0[i + 1], D = t1 - t0;
    Dv[i] = D;
    sl0v[i] = tiles[t0].s0;
    spsv[i] = tiles[t0].s1 - tiles[t0].s0;
    for (int t = t0; t < t1; ++t)
      for (int s = tiles[t].s0; s < tiles[t].s1; ++s) sub_of_slice[s] = t - t0;
    std::vector<double> E((size_t)D * D, 0.0);
    for (int t = t0; t < t1; ++t)
      for (int s = tiles[t].s0; s < tiles[t].s1; ++s)
        for (int l = 0; l < 32; ++l)
          for (int j = 0; j < len[s]; ++j) {
            const int e = sp[s] + j * 32 + l;
            E[(size_t)(t - t0) * D + sub_of_slice[col[e] / 32]] += A[e];
          }
    if (!spd_inverse(E, D)) {
      set_error("krylov: the coarse pressure matrix is not SPD");
      return PFEM2_MESH_ERROR;
    }
    eoff[i] = (int)Einv.size();
    for (double v : E) Einv.push_back((float)v);
  }
  PFEM2_CUDA(cudaMalloc(&w->Einv, sizeof(float) * Einv.size()));
  PFEM2_CUDA(cudaMemcpy(w->Einv, Einv.data(), sizeof(float) * Einv.size(), cudaMemcpyHostToDevice));
  int** dst[] = {&w->sys_eoff, &w->sys_D, &w->sys_sl0, &w->sys_sps};
  std::vector<int>* src[] = {&eoff, &Dv, &sl0v, &spsv};
  for (int k = 0; k < 4; ++k) {
    PFEM2_CUDA(cudaMalloc(dst[k], sizeof(int) * ni));
    PFEM2_CUDA(cudaMemcpy(*dst[k], src[k]->data(), sizeof(int) * ni, cudaMemcpyHostToDevice));
  }
  w->two_level = true;
  return PFEM2_OK;
}

__global__ void k_init_solve(int nsys, int* __restrict__ active, unsigned* __restrict__ barrier,
                             int* __restrict__ err) {
  if (threadIdx.x == 0) {
    *active = nsys;
    barrier[0] = 0;
    barrier[1] = 0;
    *err = 0;
  }
}

template <typename R>
static pfem2_status solve_impl(Ctx& c, int which) {
  KrylovWs* w = (KrylovWs*)c.kws;
  const int ph = which == 1 ? 0 : 1;
  const int ncomp = which == 1 ? 1 : c.dim;
  const int ni = (int)c.inst.size();
  const bool two = which == 1 && w->two_level && c.two_level;
  SolveArgs<R> a{};
  a.ncomp = ncomp;
  a.ninst = ni;
  a.nsys = w->nsys[ph];
  a.ntiles = w->ntiles[ph];
  a.nv = c.nv;
  a.tiles = w->tiles[ph];
  a.sys_t0 = w->sys_t0[ph];
  a.blk_t0 = w->blk_t0[ph];
  a.sl_ptr = c.sl_ptr;
  a.sl_len = c.sl_len;
  a.sl_col = c.sl_col;
  a.Binv = (const R*)w->Binv;
  a.Einv = w->Einv;
  a.sys_eoff = w->sys_eoff;
  a.sys_D = w->sys_D;
  a.sys_sl0 = w->sys_sl0;
  a.sys_sps = w->sys_sps;
  a.dmax = w->dmax;
  a.binv_smem = w->binv_smem;
  for (int k = 0; k < 3; ++k) {
    const int kk = k < ncomp ? k : 0;
    const int mtx = which == 0 ? kk : (which == 1 ? 3 : 4 + kk);
    a.A64[k] = c.A64[mtx];
    a.Ain[k] = c.mixed ? (const R*)c.A32[mtx] : (const R*)c.A64[mtx];
    a.dinv[k] = c.mixed ? (const R*)c.dinv32[mtx] : (const R*)c.dinv64[mtx];
    if (which == 0) {
      a.x[k] = c.F[PFEM2_FIELD_PRED_VX + kk];
      a.b[k] = c.rhs[kk];
      a.isd[k] = c.isdir[kk];
      a.g[k] = c.dirval[kk];
    } else if (which == 1) {
      a.x[k] = c.F[PFEM2_FIELD_P];
      a.b[k] = c.rhs[0];
      a.isd[k] = c.isdir[3];
      a.g[k] = c.dirval[3];
    } else {
      a.x[k] = c.corr[kk];
      a.b[k] = c.rhs[kk];
      a.isd[k] = c.isdir[kk];
      a.g[k] = nullptr;
    }
  }
  a.tol_i = (const double*)c.sys_scalars + (which == 1 ? ni : 0);
  a.maxit_i = c.d_sysinfo;
  a.e = (R*)w->e; a.r = (R*)w->r; a.z = (R*)w->z; a.q = (R*)w->q; a.p = (R*)w->p;
  a.r64 = w->r64;
  a.part = w->part;
  a.active = w->active;
  a.out_it = w->out_it[which];
  a.out_res = w->out_res[which];
  a.out_outer = w->out_outer[which];
  a.eta = c.mixed ? c.refine_eta : 0.0;
  int mx = 0;
  for (auto& in : c.inst) mx = std::max(mx, in.cs.max_iter > 0 ? in.cs.max_iter : 10000);
  a.iter_cap = 2 * mx + 64;
  a.gb.count = c.barrier;
  a.gb.gen = c.barrier + 1;
  a.gb.err = c.d_err;
  a.prof = w->prof ? w->prof + 6 * which : nullptr;
  k_init_solve<<<1, 32, 0, c.stream>>>(a.nsys, w->active, c.barrier, c.d_err);
  c.launches++;
  void* args[] = {&a};
  if (two)
    PFEM2_CUDA(cudaLaunchCooperativeKernel((const void*)k_krylov<R, true>, dim3(w->grid[ph]), dim3(kSolveThreads),
                                           args, w->smem_two, c.stream));
  else
    PFEM2_CUDA(cudaLaunchCooperativeKernel((const void*)k_krylov<R, false>, dim3(w->grid[ph]), dim3(kSolveThreads),
                                           args, 0, c.stream));
  c.launches++;
  return PFEM2_OK;
}

pfem2_status krylov_solve(Ctx& c, int which) {
  return c.mixed ? solve_impl<float>(c, which) : solve_impl<double>(c, which);
}

// per-system iteration counts / residuals into c.stats (max over
// instances); NOT_CONVERGED if a system ended above its tolerance
static pfem2_status read_stats_phase(Ctx& c, int which) {
  KrylovWs* w = (KrylovWs*)c.kws;
  const int ph = which == 1 ? 0 : 1;
  const int ns = w->nsys[ph];
  std::vector<int> it(ns), outer(ns);
  std::vector<double> res(ns);
  PFEM2_CUDA(cudaMemcpyAsync(it.data(), w->out_it[which], sizeof(int) * ns, cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(res.data(), w->out_res[which], sizeof(double) * ns, cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(outer.data(), w->out_outer[which], sizeof(int) * ns, cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  const int ni = (int)c.inst.size();
  const int ncomp = which == 1 ? 1 : c.dim;
  bool notconv = false;
  for (int k = 0; k < ncomp; ++k) {
    const int slot = which == 0 ? k : (which == 1 ? 3 : 4 + k);
    int mit = 0, mo = 0;
    double mres = 0.0;
    for (int i = 0; i < ni; ++i) {
      const int s = k * ni + i;
      mit = std::max(mit, it[s]);
      mo = std::max(mo, outer[s]);
      mres = std::max(mres, res[s]);
      const double tol = which == 1 ? c.inst[i].cs.p_tol : c.inst[i].cs.vel_tol;
      if (res[s] > tol) notconv = true;
    }
    c.stats.iters[slot] = mit;
    c.stats.residual[slot] = mres;
    if (which == 1) c.stats.refinements_p = mo;
  }
  return notconv ? PFEM2_NOT_CONVERGED : PFEM2_OK;
}

// sub-phase times of block 0 (ns): sums, coarse, decisions, work, barrier, loop
void krylov_profile(Ctx& c, unsigned long long* out18) {
  KrylovWs* w = (KrylovWs*)c.kws;
  if (!w || !w->prof) return;
  cudaMemcpy(out18, w->prof, sizeof(unsigned long long) * 18, cudaMemcpyDeviceToHost);
}

pfem2_status krylov_read_stats(Ctx& c) {
  pfem2_status worst = PFEM2_OK;
  for (int wch = 0; wch < 3; ++wch) {
    pfem2_status s = read_stats_phase(c, wch);
    if (s != PFEM2_OK && worst == PFEM2_OK) worst = s;
  }
  int err = 0;
  PFEM2_CUDA(cudaMemcpy(&err, c.d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err == 1) {
    set_error("krylov: a grid barrier wait timed out");
    return PFEM2_TIMEOUT;
  }
  if (err == 2) {
    set_error("krylov: iteration cap reached");
    return PFEM2_NOT_CONVERGED;
  }
  return worst;
}

}  // namespace pfem2
