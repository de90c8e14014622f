// krylov.cu -- batched, persistent preconditioned CG with FP64 reliable
// updates on the SELL-32 pattern (sm_100a).
//
// One cooperative launch solves every system of a solve phase (components x
// instances) to the reference's stopping rule: the absolute 2-norm of the
// unpreconditioned residual b - A x <= tol within max_iter iterations
// (deal.II SolverControl(max_iter, tol), cylinder2D/cylinder2D.cc:736-779).
// The reference runs BiCGStab with Jacobi (velocity) / SSOR or AMG
// (pressure); the prediction, mass and Poisson matrices here are symmetric
// positive definite after the symmetric Dirichlet elimination, so CG reaches
// the same solution.
//
// The work between two bounded grid barriers is a "phase". Every block that
// owns tiles of a system computes that system's scalars itself, from the
// per-tile partial sums of the previous phase, in a fixed order: no block
// publishes scalars and no phase waits for a finalizer.
//
// Jacobi-preconditioned systems (prediction, mass) take two phases per
// iteration:
//   A  p' = z + beta p ; q = A p'                 (p double buffered) | (p', q)
//   B  e += alpha p' ; r -= alpha q ; z = D^-1 r                     | (r, z), (r, r)
// The pressure systems are preconditioned with one multigrid V(1,1) cycle
// in additive form (amg.h) and take four:
//   B   e += alpha p' ; r' = r - alpha q (r double buffered) ;
//       b1 = R01 r' (level-1 rows of the block, r' formed on the fly)  | (r', r')
//   D   b2 = R12 b1 ; b3 = R13 b1
//   UZ  x3 = E^-1 b3, x2 = J2 b2 + Pt2 x3, x1 = J1 b1 + Pt1 x2 on the
//       block's own and halo coarse dofs (shared memory, redundant across
//       blocks), z = J0 r + Pt0 x1 on the own rows                  | (r, z)
//   A   p' = z + beta p ; q = A p'                                  | (p', q)
// so the coarse levels never need a barrier of their own.
//
// The iterate is split x + e: e accumulates in the inner type R (FP32 for
// the mixed path, FP64 for the plain path); once the recurrence residual
// has dropped below max(eta * res, tol / 2) a reliable update runs in FP64
// (r64 = b - A64 (x + e), then x += e, e = 0, r = r64) and CG restarts from
// the true residual. A system is done when the FP64 residual is <= tol.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <vector>

#include "amg.h"
#include "common.cuh"
#include "ctx.h"

namespace pfem2 {

constexpr int kSolveThreads = 384;  // 12 warps
constexpr int kWarps = kSolveThreads / 32;
constexpr int kMaxLocalSys = 16;

enum { S_OUT_A = 0, S_OUT_B = 1, S_A = 2, S_B = 3, S_DONE = 4, S_D = 5, S_UZ = 6 };
enum { ACT_NONE = 0, ACT_OUT_A = 1, ACT_OUT_B = 2, ACT_OUT_DONE = 3, ACT_A = 4, ACT_B = 5, ACT_D = 6, ACT_UZ = 7 };

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
  // multigrid (pressure phase), layout of MgHost
  const int *toff1, *toff2, *toff3;     // [ntiles+1]
  const int *lsys1, *lsys2, *lsys3;     // system of each level-l dof
  const int *r01_ptr, *r01_col, *r12_ptr, *r12_col, *r13_ptr, *r13_col;
  const R *r01_val, *r12_val, *r13_val;
  const R* j0;                          // [nell]
  const int *p0_ptr, *p0_len, *p0_col;  // SELL per slice, columns into the block's level-1 list
  const R* p0_val;
  const int *blk_s1, *s1_sys, *s1_jptr, *s1_jcol, *s1_pptr, *s1_pcol;
  const R *s1_jval, *s1_pval;
  const int *blk_s2, *s2_sys, *s2_jptr, *s2_jcol, *s2_pptr, *s2_pcol;
  const R *s2_jval, *s2_pval;
  const int *blk_s3, *s3_sys, *s3_eoff, *blk_e;
  const float* s3_E;
  const int *sys_D3, *sys_off3;
  int dmax, s1max, s2max, s3max;
  R *b1, *b2, *b3;
  double* x[3];
  const double* b[3];
  const unsigned char* isd[3];
  const double* g[3];    // Dirichlet values preset in x (nullptr -> 0)
  const double* tol_i;   // per instance
  const int* maxit_i;    // per instance
  // workspace per component slot, nv entries each; r and p: 2 buffers
  R *e, *r, *z, *p, *q;
  double* r64;
  double* part;          // [2][ntiles][3], by phase parity
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

__device__ __forceinline__ float fma_r(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_r(double a, double b, double c) { return fma(a, b, c); }

template <int GL, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = GL / 2; o > 0; o >>= 1) v += __shfl_xor_sync(PFEM2_FULL_MASK, v, o);
  return v;
}

struct LocalSys {
  int sys, state, it, outer, par, rpar, first, owner, maxit, act, chk;
  double tol, intol, res, rz_prev, alpha, beta;
  double sum[2];
};

template <typename R, bool MG>
__global__ void __launch_bounds__(kSolveThreads) k_krylov(SolveArgs<R> a) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ LocalSys ls[kMaxLocalSys];
  __shared__ double red[kWarps][2];
  __shared__ int s_nls, s_sys0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t nv = (size_t)a.nv;
  const int t_lo = a.blk_t0[blockIdx.x], t_hi = a.blk_t0[blockIdx.x + 1];
  unsigned bar_gen = 0;

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
      L.it = L.outer = L.par = L.rpar = L.chk = 0;
      L.first = 1;
      L.owner = a.sys_t0[s] >= t_lo && a.sys_t0[s] < t_hi;
      L.maxit = a.maxit_i[inst];
      L.tol = a.tol_i[inst];
      L.intol = 0.5 * L.tol;
      L.res = L.rz_prev = L.alpha = L.beta = 0.0;
      L.sum[0] = L.sum[1] = 0.0;
      L.act = ACT_NONE;
    }
  }
  __syncthreads();
  const int nls = s_nls, sys0 = s_sys0;
  // multigrid shared memory: x1 | x2 | x3 | b3 per local system (R), coarse-inverse rows (float)
  R* sx1 = reinterpret_cast<R*>(dyn_smem);
  R* sx2 = sx1 + a.s1max;
  R* sx3 = sx2 + a.s2max;
  R* sb3 = sx3 + a.s3max;
  float* sE = reinterpret_cast<float*>(sb3 + (size_t)nls * a.dmax);
  int s1_lo = 0, s1_hi = 0, s2_lo = 0, s2_hi = 0, s3_lo = 0, s3_hi = 0, o1lo = 0, o1hi = 0, o2lo = 0, o2hi = 0,
      o3lo = 0, o3hi = 0;
  if (MG) {
    s1_lo = a.blk_s1[blockIdx.x];
    s1_hi = a.blk_s1[blockIdx.x + 1];
    s2_lo = a.blk_s2[blockIdx.x];
    s2_hi = a.blk_s2[blockIdx.x + 1];
    s3_lo = a.blk_s3[blockIdx.x];
    s3_hi = a.blk_s3[blockIdx.x + 1];
    o1lo = a.toff1[t_lo];
    o1hi = a.toff1[t_hi];
    o2lo = a.toff2[t_lo];
    o2hi = a.toff2[t_hi];
    o3lo = a.toff3[t_lo];
    o3hi = a.toff3[t_hi];
    const int e0 = a.blk_e[blockIdx.x], ne = a.blk_e[blockIdx.x + 1] - e0;
    for (int i = threadIdx.x; i < ne; i += kSolveThreads) sE[i] = a.s3_E[e0 + i];
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
    // ---- sums of the previous phase's partials (warp 0, fixed order)
    if (warp == 0) {
      for (int k = 0; k < nls; ++k) {
        const int st = ls[k].state;
        if (st == S_DONE || st == S_OUT_A || st == S_UZ || (st == S_D && !ls[k].chk)) continue;
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
    // ---- decisions (thread 0; identical in every block owning the system)
    if (threadIdx.x == 0) {
      for (int k = 0; k < nls; ++k) {
        LocalSys& L = ls[k];
        int act = ACT_NONE;
        if (!MG) {
          if (phaseA) {
            if (L.state == S_OUT_A) {
              act = ACT_OUT_A;
              L.state = S_OUT_B;
            } else if (L.state == S_A) {
              const double rz = L.sum[0], rr = sqrt(L.sum[1]);
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
        } else {
          switch (L.state) {
            case S_OUT_A:
              act = ACT_OUT_A;
              L.state = S_OUT_B;
              break;
            case S_OUT_B:
              L.res = sqrt(L.sum[0]);
              L.outer += 1;
              if (L.res <= L.tol || L.it >= L.maxit || !(L.res == L.res)) {
                act = ACT_OUT_DONE;
                L.state = S_DONE;
              } else {
                L.intol = fmax(a.eta * L.res, 0.5 * L.tol);
                L.first = 1;  // CG restarts from the true residual
                L.chk = 0;
                act = ACT_OUT_B;
                L.state = S_D;
              }
              break;
            case S_D: {
              const double rr = sqrt(L.sum[0]);
              if (L.chk && (rr <= L.intol || L.it >= L.maxit || !(rr == rr))) {
                act = ACT_OUT_A;  // reliable update in FP64
                L.state = S_OUT_B;
              } else {
                act = ACT_D;
                L.state = S_UZ;
              }
              break;
            }
            case S_UZ:
              act = ACT_UZ;
              L.state = S_A;
              break;
            case S_A: {
              const double rz = L.sum[0];
              L.beta = L.first ? 0.0 : (L.rz_prev != 0.0 ? rz / L.rz_prev : 0.0);
              L.rz_prev = rz;
              L.first = 0;
              act = ACT_A;
              L.state = S_B;
              break;
            }
            case S_B:
              L.alpha = L.sum[0] != 0.0 ? L.rz_prev / L.sum[0] : 0.0;
              L.it += 1;
              L.chk = 1;
              act = ACT_B;
              L.state = S_D;
              break;
            default:
              break;
          }
        }
        L.act = act;
      }
    }
    __syncthreads();
    PFEM2_PROF(2);
    // ---- coarse-level work of the block (multigrid; pressure = component 0)
    if (MG) {
      bool any_b = false, any_d = false, any_uz = false;
      for (int k = 0; k < nls; ++k) {
        const int act = ls[k].act;
        any_b |= act == ACT_B || act == ACT_OUT_B;
        any_d |= act == ACT_D;
        any_uz |= act == ACT_UZ;
      }
      if (any_b) {
        // b1 = R01 r' on the own level-1 rows (8 lanes per row); after a
        // reliable update r' = r64, else r' = r - alpha q formed on the fly
        constexpr int GL = 8, NG = kSolveThreads / GL;
        const int sub = threadIdx.x % GL, grp = threadIdx.x / GL;
        for (int base = o1lo; base < o1hi; base += NG) {
          const int i = base + grp;
          R acc = R(0);
          int act = ACT_NONE;
          if (i < o1hi) {
            const LocalSys& L = ls[__ldg(a.lsys1 + i) - sys0];
            act = L.act;
            const int k1 = __ldg(a.r01_ptr + i + 1);
            if (act == ACT_B) {
              const R al = R(L.alpha);
              const R* rr = a.r + (size_t)L.rpar * nv;
#pragma unroll 4
              for (int k = __ldg(a.r01_ptr + i) + sub; k < k1; k += GL) {
                const int j = __ldg(a.r01_col + k);
                acc += __ldg(a.r01_val + k) * fma_r(-al, __ldcg(a.q + j), __ldcg(rr + j));
              }
            } else if (act == ACT_OUT_B) {
#pragma unroll 4
              for (int k = __ldg(a.r01_ptr + i) + sub; k < k1; k += GL)
                acc += __ldg(a.r01_val + k) * R(__ldcg(a.r64 + __ldg(a.r01_col + k)));
            }
          }
          acc = group_sum<GL>(acc);
          if (sub == 0 && (act == ACT_B || act == ACT_OUT_B)) a.b1[i] = acc;
        }
      }
      if (any_d) {
        // b2 = R12 b1, b3 = R13 b1 on the own level-2 / level-3 rows (warp per row)
        const int n2 = o2hi - o2lo, n3 = o3hi - o3lo;
        for (int w = warp; w < n2 + n3; w += kWarps) {
          const bool l2 = w < n2;
          const int i = l2 ? o2lo + w : o3lo + (w - n2);
          if (ls[__ldg((l2 ? a.lsys2 : a.lsys3) + i) - sys0].act != ACT_D) continue;
          const int* ptr = l2 ? a.r12_ptr : a.r13_ptr;
          const int* cl = l2 ? a.r12_col : a.r13_col;
          const R* vl = l2 ? a.r12_val : a.r13_val;
          R acc = R(0);
          const int k1 = __ldg(ptr + i + 1);
#pragma unroll 4
          for (int k = __ldg(ptr + i) + lane; k < k1; k += 32) acc += __ldg(vl + k) * __ldcg(a.b1 + __ldg(cl + k));
          acc = warp_sum(acc);
          if (lane == 0) (l2 ? a.b2 : a.b3)[i] = acc;
        }
      }
      if (any_uz) {
        // b3 of the local systems
        for (int k = 0; k < nls; ++k) {
          if (ls[k].act != ACT_UZ) continue;
          const int s = ls[k].sys, D = __ldg(a.sys_D3 + s), o = __ldg(a.sys_off3 + s);
          for (int d = threadIdx.x; d < D; d += kSolveThreads) sb3[k * a.dmax + d] = __ldcg(a.b3 + o + d);
        }
        __syncthreads();
        // x3 = E^-1 b3 on the block's level-3 list (warp per row, shared memory)
        for (int j = s3_lo + warp; j < s3_hi; j += kWarps) {
          const int s = __ldg(a.s3_sys + j), k = s - sys0;
          if (ls[k].act != ACT_UZ) continue;
          const int D = __ldg(a.sys_D3 + s);
          const float* E = sE + __ldg(a.s3_eoff + j);
          const R* bb = sb3 + k * a.dmax;
          R acc = R(0);
          for (int d = lane; d < D; d += 32) acc += R(E[d]) * bb[d];
          acc = warp_sum(acc);
          if (lane == 0) sx3[j - s3_lo] = acc;
        }
        __syncthreads();
        // x2 = J2 b2 + Pt2 x3 on the level-2 list (4 lanes per row)
        {
          constexpr int GL = 4, NG = kSolveThreads / GL;
          const int sub = threadIdx.x % GL, grp = threadIdx.x / GL;
          for (int base = s2_lo; base < s2_hi; base += NG) {
            const int j = base + grp;
            R acc = R(0);
            bool on = false;
            if (j < s2_hi && ls[__ldg(a.s2_sys + j) - sys0].act == ACT_UZ) {
              on = true;
              const int ja = __ldg(a.s2_jptr + j), jb = __ldg(a.s2_jptr + j + 1);
#pragma unroll 4
              for (int k = ja + sub; k < jb; k += GL) acc += __ldg(a.s2_jval + k) * __ldcg(a.b2 + __ldg(a.s2_jcol + k));
              const int pa = __ldg(a.s2_pptr + j), pb = __ldg(a.s2_pptr + j + 1);
              for (int k = pa + sub; k < pb; k += GL) acc += __ldg(a.s2_pval + k) * sx3[__ldg(a.s2_pcol + k)];
            }
            acc = group_sum<GL>(acc);
            if (on && sub == 0) sx2[j - s2_lo] = acc;
          }
        }
        __syncthreads();
        // x1 = J1 b1 + Pt1 x2 on the level-1 list (4 lanes per row)
        {
          constexpr int GL = 4, NG = kSolveThreads / GL;
          const int sub = threadIdx.x % GL, grp = threadIdx.x / GL;
          for (int base = s1_lo; base < s1_hi; base += NG) {
            const int j = base + grp;
            R acc = R(0);
            bool on = false;
            if (j < s1_hi && ls[__ldg(a.s1_sys + j) - sys0].act == ACT_UZ) {
              on = true;
              const int ja = __ldg(a.s1_jptr + j), jb = __ldg(a.s1_jptr + j + 1);
#pragma unroll 4
              for (int k = ja + sub; k < jb; k += GL) acc += __ldg(a.s1_jval + k) * __ldcg(a.b1 + __ldg(a.s1_jcol + k));
              const int pa = __ldg(a.s1_pptr + j), pb = __ldg(a.s1_pptr + j + 1);
              for (int k = pa + sub; k < pb; k += GL) acc += __ldg(a.s1_pval + k) * sx2[__ldg(a.s1_pcol + k)];
            }
            acc = group_sum<GL>(acc);
            if (on && sub == 0) sx1[j - s1_lo] = acc;
          }
        }
      }
      __syncthreads();
    }
    PFEM2_PROF(1);
    // ---- level-0 work on the own tiles
    for (int t = t_lo; t < t_hi; ++t) {
      const Tile T = a.tiles[t];
      const int k = T.comp;
      const int lk = T.sys - sys0;
      const LocalSys& L = ls[lk];
      const int act = L.act;
      if (act == ACT_NONE || act == ACT_D) continue;
      double v0 = 0.0, v1 = 0.0;
      const R* dinv = a.dinv[k];
      R* e = a.e + k * nv;
      R* r = a.r + (2 * k + L.rpar) * nv;
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
            r[row] = rr;
            if (!MG) {
              const R zz = rr * dinv[row];
              z[row] = zz;
              v0 += (double)rr * (double)zz;
              v1 += (double)rr * (double)rr;
            }
          }
        }
      } else if (act == ACT_A) {
        const R beta = R(L.beta);
        R* pn = a.p + (2 * k + L.par) * nv;
        const R* po = a.p + (2 * k + (L.par ^ 1)) * nv;
        const R* A = a.Ain[k];
        for (int sl = T.s0 + warp; sl < T.s1; sl += kWarps) {
          const int row = sl * 32 + lane;
          const int base = a.sl_ptr[sl], len = a.sl_len[sl];
          R acc = R(0);
          for (int j = 0; j < len; ++j) {
            const int ei = base + j * 32 + lane;
            const int col = __ldg(a.sl_col + ei);
            acc += A[ei] * fma_r(beta, __ldcg(po + col), __ldcg(z + col));
          }
          const R pp = fma_r(beta, po[row], z[row]);
          pn[row] = pp;
          q[row] = acc;
          v0 += (double)pp * (double)acc;
        }
      } else if (act == ACT_B) {
        const R alpha = R(L.alpha);
        const R* pn = a.p + (2 * k + L.par) * nv;
        R* rn = MG ? a.r + (2 * k + (L.rpar ^ 1)) * nv : r;
        for (int sl = T.s0 + warp; sl < T.s1; sl += kWarps) {
          const int row = sl * 32 + lane;
          e[row] += alpha * pn[row];
          const R rr = fma_r(-alpha, q[row], r[row]);
          rn[row] = rr;
          if (MG) {
            v0 += (double)rr * (double)rr;
          } else {
            const R zz = rr * dinv[row];
            z[row] = zz;
            v0 += (double)rr * (double)zz;
            v1 += (double)rr * (double)rr;
          }
        }
      } else if (MG && act == ACT_UZ) {
        // z = J0 r + Pt0 x1
        const R* J = a.j0;
        for (int sl = T.s0 + warp; sl < T.s1; sl += kWarps) {
          const int row = sl * 32 + lane;
          const int base = a.sl_ptr[sl], len = a.sl_len[sl];
          R acc = R(0);
          for (int j = 0; j < len; ++j) {
            const int ei = base + j * 32 + lane;
            acc += __ldg(J + ei) * __ldcg(r + __ldg(a.sl_col + ei));
          }
          const int pb = __ldg(a.p0_ptr + sl), pl = __ldg(a.p0_len + sl);
          for (int j = 0; j < pl; ++j) {
            const int ei = pb + j * 32 + lane;
            acc += __ldg(a.p0_val + ei) * sx1[__ldg(a.p0_col + ei)];
          }
          z[row] = acc;
          v0 += (double)__ldcg(r + row) * (double)acc;
        }
      }
      // deterministic block reduction into this phase's parity buffer
      v0 = warp_sum(v0);
      v1 = warp_sum(v1);
      if (lane == 0) {
        red[warp][0] = v0;
        red[warp][1] = v1;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int wv = 0; wv < kWarps; ++wv) {
          s0 += red[wv][0];
          s1 += red[wv][1];
        }
        double* dst = a.part + ((size_t)(iter & 1) * a.ntiles + t) * 3;
        dst[0] = s0;
        dst[1] = s1;
      }
      __syncthreads();
    }
    PFEM2_PROF(3);
    // ---- bookkeeping
    if (threadIdx.x == 0) {
      for (int k = 0; k < nls; ++k) {
        LocalSys& L = ls[k];
        if (L.act == ACT_B) {
          L.par ^= 1;
          if (MG) L.rpar ^= 1;
        }
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
  std::vector<int> h_sys_t0_0, h_blk_t0_0;
  // multigrid of the pressure phase (phase 0)
  bool mg = false;
  int nls0 = 1;
  size_t smem_mg = 0;
  int dmax = 1, s1max = 0, s2max = 0, s3max = 0;
  int n1 = 0, n2 = 0, n3 = 0;
  int *toff[4] = {}, *lsys[4] = {};
  int *r01_ptr = nullptr, *r01_col = nullptr, *r12_ptr = nullptr, *r12_col = nullptr, *r13_ptr = nullptr,
      *r13_col = nullptr;
  void *r01_val = nullptr, *r12_val = nullptr, *r13_val = nullptr, *j0 = nullptr;
  int *p0_ptr = nullptr, *p0_len = nullptr, *p0_col = nullptr;
  void* p0_val = nullptr;
  int *blk_s[3] = {}, *s_sys[3] = {}, *s_jptr[3] = {}, *s_jcol[3] = {}, *s_pptr[3] = {}, *s_pcol[3] = {};
  void *s_jval[3] = {}, *s_pval[3] = {};
  int *blk_s3 = nullptr, *s3_sys = nullptr, *s3_eoff = nullptr, *blk_e = nullptr;
  float* s3_E = nullptr;
  int *sys_D3 = nullptr, *sys_off3 = nullptr;
  void *b1 = nullptr, *b2 = nullptr, *b3 = nullptr;
  void *e = nullptr, *r = nullptr, *z = nullptr, *q = nullptr, *p = nullptr;
  double* r64 = nullptr;
  double* part = nullptr;
  int* active = nullptr;
  int* out_it[3];
  double* out_res[3];
  int* out_outer[3];
  unsigned long long* prof = nullptr;  // [3 solve kinds][6]
  std::vector<void*> allocs;            // every device allocation of the workspace
};

template <typename T>
static pfem2_status ws_alloc(KrylovWs* w, T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  PFEM2_CUDA(cudaMalloc((void**)p, sizeof(T) * n));
  PFEM2_CUDA(cudaMemset(*p, 0, sizeof(T) * n));
  w->allocs.push_back(*p);
  return PFEM2_OK;
}

template <typename T>
static pfem2_status ws_upload(KrylovWs* w, T** p, const std::vector<T>& v) {
  PFEM2_TRY(ws_alloc(w, p, v.size()));
  if (!v.empty()) PFEM2_CUDA(cudaMemcpy(*p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return PFEM2_OK;
}

// FP64 host values as the inner type R (float for the mixed path)
static pfem2_status ws_upload_r(KrylovWs* w, bool mixed, void** p, const std::vector<double>& v) {
  if (mixed) {
    std::vector<float> f(v.begin(), v.end());
    float* d;
    PFEM2_TRY(ws_upload(w, &d, f));
    *p = d;
  } else {
    double* d;
    PFEM2_TRY(ws_upload(w, &d, v));
    *p = d;
  }
  return PFEM2_OK;
}

static int max_local_systems(const std::vector<Tile>& tiles, const std::vector<int>& bt0) {
  int worst = 0;
  for (size_t b = 0; b + 1 < bt0.size(); ++b)
    if (bt0[b + 1] > bt0[b]) worst = std::max(worst, tiles[bt0[b + 1] - 1].sys - tiles[bt0[b]].sys + 1);
  return worst;
}

template <typename R, bool MG>
static int occupancy(size_t smem) {
  int occ = 0;
  // one process-wide upper bound, so contexts with different hierarchies coexist
  if (MG) cudaFuncSetAttribute((const void*)k_krylov<R, MG>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_krylov<R, MG>, kSolveThreads, smem) != cudaSuccess) return 0;
  return occ;
}

void krylov_free(Ctx& c) {
  KrylovWs* w = (KrylovWs*)c.kws;
  if (!w) return;
  for (void* p : w->allocs) cudaFree(p);
  delete w;
  c.kws = nullptr;
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
      // pressure: tiles = the aggregation domains of the multigrid; about
      // one per block of the persistent grid (balanced work), at most dcap
      // per system (a batch: tiles of ~8 slices, at most dcap per system,
      // so every instance gets a coarse space of its own size)
      const int dcap = ni == 1 ? 160 : 96;
      const int nb = bps * c.num_sms;
      long long tot_sl = 0;
      for (int i = 0; i < ni; ++i) tot_sl += c.inst[i].nv_pad / kSlice;
      for (int i = 0; i < ni; ++i) {
        st0[i] = (int)tiles.size();
        const int sl0 = c.inst[i].v_off / kSlice, nsl = c.inst[i].nv_pad / kSlice;
        const long long share = ni == 1 ? std::max<long long>(1, (long long)nb * nsl / tot_sl) : (nsl + 7) / 8;
        int D = (int)std::min<long long>(std::min<long long>(share, dcap), nsl);
        const int sps = (nsl + D - 1) / D;
        for (int a = 0; a < nsl; a += sps) tiles.push_back(Tile{i, 0, sl0 + a, sl0 + std::min(nsl, a + sps)});
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
    // the multigrid grid is sized before its shared memory is known (one
    // block per SM); krylov_setup_precond checks residency afterwards
    const int occ = ph == 0 ? 1 : (c.mixed ? occupancy<float, false>(0) : occupancy<double, false>(0));
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
      w->nls0 = nls;
      w->h_tiles0 = tiles;
      w->h_sys_t0_0 = st0;
      w->h_blk_t0_0 = bt0;
    }
    w->ntiles[ph] = T;
    w->nsys[ph] = (int)st0.size() - 1;
    w->grid[ph] = G;
    PFEM2_TRY(ws_upload(w, &w->tiles[ph], tiles));
    PFEM2_TRY(ws_upload(w, &w->sys_t0[ph], st0));
    PFEM2_TRY(ws_upload(w, &w->blk_t0[ph], bt0));
    maxtiles = std::max(maxtiles, T);
    maxsys = std::max(maxsys, w->nsys[ph]);
  }
  if (c.mixed) {
    float *e, *r, *z, *q, *p;
    PFEM2_TRY(ws_alloc(w, &e, nv * dim));
    PFEM2_TRY(ws_alloc(w, &r, 2 * nv * dim));
    PFEM2_TRY(ws_alloc(w, &z, nv * dim));
    PFEM2_TRY(ws_alloc(w, &q, nv * dim));
    PFEM2_TRY(ws_alloc(w, &p, 2 * nv * dim));
    w->e = e; w->r = r; w->z = z; w->q = q; w->p = p;
  } else {
    double *e, *r, *z, *q, *p;
    PFEM2_TRY(ws_alloc(w, &e, nv * dim));
    PFEM2_TRY(ws_alloc(w, &r, 2 * nv * dim));
    PFEM2_TRY(ws_alloc(w, &z, nv * dim));
    PFEM2_TRY(ws_alloc(w, &q, nv * dim));
    PFEM2_TRY(ws_alloc(w, &p, 2 * nv * dim));
    w->e = e; w->r = r; w->z = z; w->q = q; w->p = p;
  }
  (void)rs;
  PFEM2_TRY(ws_alloc(w, &w->r64, nv * dim));
  PFEM2_TRY(ws_alloc(w, &w->part, 6 * (size_t)maxtiles));
  PFEM2_TRY(ws_alloc(w, &w->active, 1));
  if (getenv("PFEM2_SOLVER_PROFILE")) PFEM2_TRY(ws_alloc(w, &w->prof, 18));
  for (int k = 0; k < 3; ++k) {
    PFEM2_TRY(ws_alloc(w, &w->out_it[k], maxsys));
    PFEM2_TRY(ws_alloc(w, &w->out_res[k], maxsys));
    PFEM2_TRY(ws_alloc(w, &w->out_outer[k], maxsys));
  }
  return PFEM2_OK;
}

// The multigrid hierarchy of the pressure matrix (after Dirichlet
// elimination), built on the host and uploaded in the kernel's layout.
pfem2_status krylov_setup_precond(Ctx& c) {
  KrylovWs* w = (KrylovWs*)c.kws;
  if (!c.two_level) return PFEM2_OK;
  std::vector<double> A(c.nell);
  std::vector<int> col(c.nell), len(c.nslices);
  PFEM2_CUDA(cudaMemcpy(A.data(), c.A64[3], sizeof(double) * c.nell, cudaMemcpyDeviceToHost));
  PFEM2_CUDA(cudaMemcpy(col.data(), c.sl_col, sizeof(int) * c.nell, cudaMemcpyDeviceToHost));
  PFEM2_CUDA(cudaMemcpy(len.data(), c.sl_len, sizeof(int) * c.nslices, cudaMemcpyDeviceToHost));
  MgHost H;
  PFEM2_TRY(mg_build(c, A, col, len, w->h_tiles0, w->h_sys_t0_0, w->h_blk_t0_0, H));
  const size_t rs = c.mixed ? sizeof(float) : sizeof(double);
  w->dmax = H.dmax;
  w->s1max = H.s1max;
  w->s2max = H.s2max;
  w->s3max = H.s3max;
  w->smem_mg = rs * ((size_t)H.s1max + H.s2max + H.s3max + (size_t)w->nls0 * H.dmax) + sizeof(float) * H.emax;
  if (w->smem_mg > 200 * 1024) {
    set_error("krylov: the pressure multigrid's per-block data exceed shared memory");
    return PFEM2_INVALID_ARG;
  }
  const int occ = c.mixed ? occupancy<float, true>(w->smem_mg) : occupancy<double, true>(w->smem_mg);
  if (occ * c.num_sms < w->grid[0]) {
    set_error("krylov: the multigrid solver grid cannot be resident");
    return PFEM2_CUDA_ERROR;
  }
  w->n1 = H.n[1];
  w->n2 = H.n[2];
  w->n3 = H.n[3];
  for (int l = 1; l < kMgLevels; ++l) {
    PFEM2_TRY(ws_upload(w, &w->toff[l], H.toff[l]));
    PFEM2_TRY(ws_upload(w, &w->lsys[l], H.lsys[l]));
  }
  PFEM2_TRY(ws_upload(w, &w->r01_ptr, H.r01_ptr));
  PFEM2_TRY(ws_upload(w, &w->r01_col, H.r01_col));
  PFEM2_TRY(ws_upload_r(w, c.mixed, &w->r01_val, H.r01_val));
  PFEM2_TRY(ws_upload(w, &w->r12_ptr, H.r12_ptr));
  PFEM2_TRY(ws_upload(w, &w->r12_col, H.r12_col));
  PFEM2_TRY(ws_upload_r(w, c.mixed, &w->r12_val, H.r12_val));
  PFEM2_TRY(ws_upload(w, &w->r13_ptr, H.r13_ptr));
  PFEM2_TRY(ws_upload(w, &w->r13_col, H.r13_col));
  PFEM2_TRY(ws_upload_r(w, c.mixed, &w->r13_val, H.r13_val));
  PFEM2_TRY(ws_upload_r(w, c.mixed, &w->j0, H.j0));
  PFEM2_TRY(ws_upload(w, &w->p0_ptr, H.p0_ptr));
  PFEM2_TRY(ws_upload(w, &w->p0_len, H.p0_len));
  PFEM2_TRY(ws_upload(w, &w->p0_col, H.p0_col));
  PFEM2_TRY(ws_upload_r(w, c.mixed, &w->p0_val, H.p0_val));
  for (int l = 1; l <= 2; ++l) {
    PFEM2_TRY(ws_upload(w, &w->blk_s[l], H.blk_s[l]));
    PFEM2_TRY(ws_upload(w, &w->s_sys[l], H.s_sys[l]));
    PFEM2_TRY(ws_upload(w, &w->s_jptr[l], H.s_jptr[l]));
    PFEM2_TRY(ws_upload(w, &w->s_jcol[l], H.s_jcol[l]));
    PFEM2_TRY(ws_upload_r(w, c.mixed, &w->s_jval[l], H.s_jval[l]));
    PFEM2_TRY(ws_upload(w, &w->s_pptr[l], H.s_pptr[l]));
    PFEM2_TRY(ws_upload(w, &w->s_pcol[l], H.s_pcol[l]));
    PFEM2_TRY(ws_upload_r(w, c.mixed, &w->s_pval[l], H.s_pval[l]));
  }
  PFEM2_TRY(ws_upload(w, &w->blk_s3, H.blk_s3));
  PFEM2_TRY(ws_upload(w, &w->s3_sys, H.s3_sys));
  PFEM2_TRY(ws_upload(w, &w->s3_eoff, H.s3_eoff));
  PFEM2_TRY(ws_upload(w, &w->blk_e, H.blk_e));
  PFEM2_TRY(ws_upload(w, &w->s3_E, H.s3_E));
  PFEM2_TRY(ws_upload(w, &w->sys_D3, H.sys_D3));
  PFEM2_TRY(ws_upload(w, &w->sys_off3, H.sys_off3));
  if (c.mixed) {
    float *b1, *b2, *b3;
    PFEM2_TRY(ws_alloc(w, &b1, H.n[1]));
    PFEM2_TRY(ws_alloc(w, &b2, H.n[2]));
    PFEM2_TRY(ws_alloc(w, &b3, H.n[3]));
    w->b1 = b1; w->b2 = b2; w->b3 = b3;
  } else {
    double *b1, *b2, *b3;
    PFEM2_TRY(ws_alloc(w, &b1, H.n[1]));
    PFEM2_TRY(ws_alloc(w, &b2, H.n[2]));
    PFEM2_TRY(ws_alloc(w, &b3, H.n[3]));
    w->b1 = b1; w->b2 = b2; w->b3 = b3;
  }
  w->mg = true;
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
  const bool mg = which == 1 && w->mg && c.two_level;
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
  if (mg) {
    a.toff1 = w->toff[1]; a.toff2 = w->toff[2]; a.toff3 = w->toff[3];
    a.lsys1 = w->lsys[1]; a.lsys2 = w->lsys[2]; a.lsys3 = w->lsys[3];
    a.r01_ptr = w->r01_ptr; a.r01_col = w->r01_col; a.r01_val = (const R*)w->r01_val;
    a.r12_ptr = w->r12_ptr; a.r12_col = w->r12_col; a.r12_val = (const R*)w->r12_val;
    a.r13_ptr = w->r13_ptr; a.r13_col = w->r13_col; a.r13_val = (const R*)w->r13_val;
    a.j0 = (const R*)w->j0;
    a.p0_ptr = w->p0_ptr; a.p0_len = w->p0_len; a.p0_col = w->p0_col; a.p0_val = (const R*)w->p0_val;
    a.blk_s1 = w->blk_s[1]; a.s1_sys = w->s_sys[1]; a.s1_jptr = w->s_jptr[1]; a.s1_jcol = w->s_jcol[1];
    a.s1_jval = (const R*)w->s_jval[1]; a.s1_pptr = w->s_pptr[1]; a.s1_pcol = w->s_pcol[1];
    a.s1_pval = (const R*)w->s_pval[1];
    a.blk_s2 = w->blk_s[2]; a.s2_sys = w->s_sys[2]; a.s2_jptr = w->s_jptr[2]; a.s2_jcol = w->s_jcol[2];
    a.s2_jval = (const R*)w->s_jval[2]; a.s2_pptr = w->s_pptr[2]; a.s2_pcol = w->s_pcol[2];
    a.s2_pval = (const R*)w->s_pval[2];
    a.blk_s3 = w->blk_s3; a.s3_sys = w->s3_sys; a.s3_eoff = w->s3_eoff; a.blk_e = w->blk_e; a.s3_E = w->s3_E;
    a.sys_D3 = w->sys_D3; a.sys_off3 = w->sys_off3;
    a.dmax = w->dmax; a.s1max = w->s1max; a.s2max = w->s2max; a.s3max = w->s3max;
    a.b1 = (R*)w->b1; a.b2 = (R*)w->b2; a.b3 = (R*)w->b3;
  }
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
  a.iter_cap = (mg ? 4 : 2) * mx + 256;
  a.gb.count = c.barrier;
  a.gb.gen = c.barrier + 1;
  a.gb.err = c.d_err;
  a.prof = w->prof ? w->prof + 6 * which : nullptr;
  k_init_solve<<<1, 32, 0, c.stream>>>(a.nsys, w->active, c.barrier, c.d_err);
  c.launches++;
  void* args[] = {&a};
  if (mg)
    PFEM2_CUDA(cudaLaunchCooperativeKernel((const void*)k_krylov<R, true>, dim3(w->grid[ph]), dim3(kSolveThreads),
                                           args, w->smem_mg, c.stream));
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
