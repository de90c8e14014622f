// krylov.cu -- batched, persistent preconditioned CG with FP64 iterative
// refinement on the SELL-32 pattern (sm_100a).
//
// One cooperative launch solves every system of a phase (components x
// instances) to the reference's stopping rule: the absolute 2-norm of the
// unpreconditioned residual b - A x <= tol, at most max_iter iterations
// (deal.II SolverControl, cylinder2D/cylinder2D.cc:736-779). The reference
// runs BiCGStab + Jacobi/SSOR; the velocity, mass and pressure matrices
// here are symmetric positive definite after symmetric Dirichlet
// elimination, so CG reaches the same fixed point with one SpMV per step.
//
// Per system a small state machine runs:
//   OUTER  r64 = b - A64 (x + e) in FP64, res = ||r64||; x += e, e = 0;
//          done when res <= tol, otherwise start an inner solve
//   INNER  Jacobi-PCG on A_in e = r in the inner type R (FP32 for the mixed
//          path, FP64 for the plain path), FP64 dot products; back to OUTER
//          once ||r_inner|| <= max(eta * res, tol / 2)
// Each iteration is two phases separated by a bounded grid barrier:
//   A  p' = z + beta p ; q = A (z + beta p)   (p double-buffered)   | pq
//   B  e += alpha p' ; r -= alpha q ; z = D^-1 r                    | rz, rr
// Tile partials are reduced by the last block to finish a system's tiles
// (threadfence + counter), in a fixed order, so results are deterministic.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "ctx.h"

namespace pfem2 {

constexpr int kSolveThreads = 256;  // 8 warps, one SELL slice each per tile

enum { ST_INNER = 0, ST_OUTER = 1, ST_DONE = 2 };
enum { SD_RHO = 0, SD_ALPHA, SD_BETA, SD_RES, SD_INTOL, SD_RR, SD_TOL, SD_N };
enum { SI_STATE = 0, SI_IT, SI_PAR, SI_DONEFLAG, SI_OUTER, SI_MAXIT, SI_N };

template <typename R> struct SolveArgs {
  int ncomp, ninst, nsys, ntiles, nv;
  const Tile* tiles;
  const int* sys_t0;  // [nsys+1] first tile of each system
  const int* sl_ptr;
  const int* sl_len;
  const int* sl_col;
  const double* A64[3];
  const R* Ain[3];
  const R* dinv[3];
  double* x[3];
  const double* b[3];
  const unsigned char* isd[3];
  const double* g[3];   // Dirichlet values to preset in x (nullptr -> 0)
  // workspace per component slot: nv entries each
  double* r64;
  R* e;
  R* r;
  R* z;
  R* p;   // 2*ncomp*nv
  R* q;
  double* part;  // [ntiles][2]
  int* cnt;      // [nsys] finished-tile counters
  double* sd;    // [nsys][SD_N]
  int* si;       // [nsys][SI_N]
  int* active;   // number of unfinished systems
  double eta;
  int iter_cap;  // hard bound on the global iteration count
  GridBarrier gb;
};

// deterministic block reduction of up to 2 doubles (fixed order)
template <int NK>
__device__ __forceinline__ void block_reduce_store(double (&v)[NK], double* out) {
  __shared__ double red[kSolveThreads / 32][2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NK; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NK; ++k) red[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      double s = 0.0;
      for (int w = 0; w < kSolveThreads / 32; ++w) s += red[w][k];
      out[k] = s;
    }
  }
  __syncthreads();
}

// sum of the partials of system s (whole block, fixed order)
__device__ __forceinline__ void system_sum(const double* part, int t0, int t1, int nk, double* res) {
  __shared__ double red[kSolveThreads][2];
  double a0 = 0.0, a1 = 0.0;
  for (int t = t0 + threadIdx.x; t < t1; t += kSolveThreads) {
    a0 += __ldcg(part + (size_t)t * 2);
    if (nk > 1) a1 += __ldcg(part + (size_t)t * 2 + 1);
  }
  red[threadIdx.x][0] = a0;
  red[threadIdx.x][1] = a1;
  __syncthreads();
  for (int s = kSolveThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[threadIdx.x][0] += red[threadIdx.x + s][0];
      red[threadIdx.x][1] += red[threadIdx.x + s][1];
    }
    __syncthreads();
  }
  res[0] = red[0][0];
  res[1] = red[0][1];
  __syncthreads();
}

// called by all threads of the block after it finished its tiles of system s
// in the current phase (ntouched of them); the last contributor finalizes.
template <typename R, int PHASE>
__device__ void contribute(const SolveArgs<R>& a, int s, int ntouched) {
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const int t0 = a.sys_t0[s], t1 = a.sys_t0[s + 1];
    int old = atomicAdd(a.cnt + s, ntouched);
    s_last = (old + ntouched == t1 - t0);
    if (s_last) {
      a.cnt[s] = 0;
      __threadfence();
    }
  }
  __syncthreads();
  if (!s_last) return;
  double sum[2];
  system_sum(a.part, a.sys_t0[s], a.sys_t0[s + 1], PHASE == 0 ? 1 : 2, sum);
  if (threadIdx.x == 0) {
    volatile double* sd = a.sd + (size_t)s * SD_N;
    volatile int* si = a.si + (size_t)s * SI_N;
    const int st = si[SI_STATE];
    if (PHASE == 0) {
      if (st == ST_OUTER) {
        const double res = sqrt(sum[0]);
        sd[SD_RES] = res;
        const bool conv = res <= sd[SD_TOL];
        const bool out_of_its = si[SI_IT] >= si[SI_MAXIT];
        si[SI_DONEFLAG] = (conv || out_of_its) ? 1 : 0;
        sd[SD_INTOL] = fmax(a.eta * res, 0.5 * sd[SD_TOL]);
        si[SI_OUTER] += 1;
      } else if (st == ST_INNER) {
        sd[SD_ALPHA] = sum[0] != 0.0 ? sd[SD_RHO] / sum[0] : 0.0;
      }
    } else {
      if (st == ST_OUTER) {
        if (si[SI_DONEFLAG]) {
          si[SI_STATE] = ST_DONE;
          atomicSub(a.active, 1);
        } else {
          sd[SD_RHO] = sum[0];
          sd[SD_RR] = sqrt(sum[1]);
          sd[SD_BETA] = 0.0;
          si[SI_STATE] = ST_INNER;
        }
      } else if (st == ST_INNER) {
        si[SI_IT] += 1;
        const double rr = sqrt(sum[1]);
        sd[SD_RR] = rr;
        if (rr <= sd[SD_INTOL] || si[SI_IT] >= si[SI_MAXIT] || !(rr == rr)) {
          si[SI_STATE] = ST_OUTER;
        } else {
          sd[SD_BETA] = sd[SD_RHO] != 0.0 ? sum[0] / sd[SD_RHO] : 0.0;
          sd[SD_RHO] = sum[0];
          si[SI_PAR] ^= 1;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
}

template <typename R>
__global__ void __launch_bounds__(kSolveThreads) k_krylov(SolveArgs<R> a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t nv = (size_t)a.nv;
  // ---- init: preset Dirichlet values, e = 0, p = 0
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
    const Tile T = a.tiles[t];
    const int k = T.comp;
    for (int sl = T.s0 + warp; sl < T.s1; sl += kSolveThreads / 32) {
      const int row = sl * 32 + lane;
      if (a.isd[k][row]) a.x[k][row] = a.g[k] ? a.g[k][row] : 0.0;
      a.e[k * nv + row] = R(0);
      a.p[(2 * k) * nv + row] = R(0);
      a.p[(2 * k + 1) * nv + row] = R(0);
    }
  }
  if (!grid_sync(a.gb)) return;
  for (int iter = 0;; ++iter) {
    if (*(volatile int*)a.active <= 0) break;
    if (iter >= a.iter_cap) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(a.gb.err, 2);
      break;
    }
    // ------------------------------------------------------------ phase A
    {
      int cur_s = -1, touched = 0;
      for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const Tile T = a.tiles[t];
        if (T.sys != cur_s) {
          if (cur_s >= 0) contribute<R, 0>(a, cur_s, touched);
          cur_s = T.sys;
          touched = 0;
        }
        ++touched;
        const int k = T.comp;
        const int st = __ldcg(a.si + (size_t)T.sys * SI_N + SI_STATE);
        double v[1] = {0.0};
        if (st == ST_OUTER) {
          const double* A = a.A64[k];
          const double* xk = a.x[k];
          const R* ek = a.e + k * nv;
          for (int sl = T.s0 + warp; sl < T.s1; sl += kSolveThreads / 32) {
            const int row = sl * 32 + lane;
            const int base = a.sl_ptr[sl], len = a.sl_len[sl];
            double s = 0.0;
            for (int j = 0; j < len; ++j) {
              const int ei = base + j * 32 + lane;
              const int col = __ldg(a.sl_col + ei);
              s += A[ei] * (__ldcg(xk + col) + (double)__ldcg(ek + col));
            }
            const double rr = a.b[k][row] - s;
            a.r64[k * nv + row] = rr;
            v[0] += rr * rr;
          }
        } else if (st == ST_INNER) {
          const double* sd = a.sd + (size_t)T.sys * SD_N;
          const R beta = R(__ldcg(sd + SD_BETA));
          const int par = __ldcg(a.si + (size_t)T.sys * SI_N + SI_PAR);
          const R* pold = a.p + (2 * k + (par ^ 1)) * nv;
          R* pnew = a.p + (2 * k + par) * nv;
          const R* zk = a.z + k * nv;
          const R* A = a.Ain[k];
          for (int sl = T.s0 + warp; sl < T.s1; sl += kSolveThreads / 32) {
            const int row = sl * 32 + lane;
            const int base = a.sl_ptr[sl], len = a.sl_len[sl];
            R s = R(0);
            if (beta != R(0)) {
              for (int j = 0; j < len; ++j) {
                const int ei = base + j * 32 + lane;
                const int col = __ldg(a.sl_col + ei);
                s += A[ei] * (__ldcg(zk + col) + beta * __ldcg(pold + col));
              }
            } else {
              for (int j = 0; j < len; ++j) {
                const int ei = base + j * 32 + lane;
                s += A[ei] * __ldcg(zk + __ldg(a.sl_col + ei));
              }
            }
            const R pn = beta != R(0) ? zk[row] + beta * pold[row] : zk[row];
            pnew[row] = pn;
            a.q[k * nv + row] = s;
            v[0] += (double)pn * (double)s;
          }
        }
        double outv[1];
        block_reduce_store<1>(v, outv);
        if (threadIdx.x == 0) a.part[(size_t)t * 2] = outv[0];
      }
      if (cur_s >= 0) contribute<R, 0>(a, cur_s, touched);
    }
    if (!grid_sync(a.gb)) return;
    // ------------------------------------------------------------ phase B
    {
      int cur_s = -1, touched = 0;
      for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const Tile T = a.tiles[t];
        if (T.sys != cur_s) {
          if (cur_s >= 0) contribute<R, 1>(a, cur_s, touched);
          cur_s = T.sys;
          touched = 0;
        }
        ++touched;
        const int k = T.comp;
        const int* si = a.si + (size_t)T.sys * SI_N;
        const double* sd = a.sd + (size_t)T.sys * SD_N;
        const int st = __ldcg(si + SI_STATE);
        double v[2] = {0.0, 0.0};
        if (st == ST_OUTER) {
          const bool done = __ldcg(si + SI_DONEFLAG) != 0;
          for (int sl = T.s0 + warp; sl < T.s1; sl += kSolveThreads / 32) {
            const int row = sl * 32 + lane;
            a.x[k][row] += (double)a.e[k * nv + row];
            a.e[k * nv + row] = R(0);
            if (!done) {
              const R rr = R(a.r64[k * nv + row]);
              const R zz = rr * a.dinv[k][row];
              a.r[k * nv + row] = rr;
              a.z[k * nv + row] = zz;
              v[0] += (double)rr * (double)zz;
              v[1] += (double)rr * (double)rr;
            }
          }
        } else if (st == ST_INNER) {
          const R alpha = R(__ldcg(sd + SD_ALPHA));
          const int par = __ldcg(si + SI_PAR);
          const R* pnew = a.p + (2 * k + par) * nv;
          for (int sl = T.s0 + warp; sl < T.s1; sl += kSolveThreads / 32) {
            const int row = sl * 32 + lane;
            const size_t o = k * nv + row;
            a.e[o] += alpha * pnew[row];
            const R rr = a.r[o] - alpha * a.q[o];
            const R zz = rr * a.dinv[k][row];
            a.r[o] = rr;
            a.z[o] = zz;
            v[0] += (double)rr * (double)zz;
            v[1] += (double)rr * (double)rr;
          }
        }
        double outv[2];
        block_reduce_store<2>(v, outv);
        if (threadIdx.x == 0) {
          a.part[(size_t)t * 2] = outv[0];
          a.part[(size_t)t * 2 + 1] = outv[1];
        }
      }
      if (cur_s >= 0) contribute<R, 1>(a, cur_s, touched);
    }
    if (!grid_sync(a.gb)) return;
  }
}

// ------------------------------------------------------------------ host
static std::vector<Tile> build_tiles(const Ctx& c, int ncomp, std::vector<int>& sys_t0) {
  std::vector<Tile> tiles;
  const int ni = (int)c.inst.size();
  sys_t0.assign(ncomp * ni + 1, 0);
  for (int k = 0; k < ncomp; ++k)
    for (int i = 0; i < ni; ++i) {
      const int s = k * ni + i;
      sys_t0[s] = (int)tiles.size();
      const int sl0 = c.inst[i].v_off / kSlice, sl1 = (c.inst[i].v_off + c.inst[i].nv_pad) / kSlice;
      for (int a = sl0; a < sl1; a += c.tile_slices) tiles.push_back(Tile{s, k, a, std::min(sl1, a + c.tile_slices)});
    }
  sys_t0[ncomp * ni] = (int)tiles.size();
  return tiles;
}

struct KrylovWs {
  Tile* tiles[2];
  int* sys_t0[2];
  int ntiles[2];
  int nsys[2];
  double* r64;
  void* e;
  void* r;
  void* z;
  void* p;
  void* q;
  double* part;
  int* cnt;
  double* sd[3];  // per solve kind (prediction, pressure, correction)
  int* si[3];
  int* active;
  int coop_blocks[2];  // per inner type: 0 float, 1 double
};

pfem2_status krylov_setup(Ctx& c) {
  KrylovWs* w = new KrylovWs();
  const int dim = c.dim;
  const size_t nv = c.nv;
  const size_t rs = c.mixed ? sizeof(float) : sizeof(double);
  int maxtiles = 0, maxsys = 0;
  for (int ph = 0; ph < 2; ++ph) {
    std::vector<int> st0;
    auto tiles = build_tiles(c, ph == 0 ? 1 : dim, st0);
    w->ntiles[ph] = (int)tiles.size();
    w->nsys[ph] = (int)st0.size() - 1;
    PFEM2_CUDA(cudaMalloc(&w->tiles[ph], sizeof(Tile) * tiles.size()));
    PFEM2_CUDA(cudaMemcpy(w->tiles[ph], tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice));
    PFEM2_CUDA(cudaMalloc(&w->sys_t0[ph], sizeof(int) * st0.size()));
    PFEM2_CUDA(cudaMemcpy(w->sys_t0[ph], st0.data(), sizeof(int) * st0.size(), cudaMemcpyHostToDevice));
    maxtiles = std::max(maxtiles, (int)tiles.size());
    maxsys = std::max(maxsys, w->nsys[ph]);
  }
  PFEM2_CUDA(cudaMalloc(&w->r64, sizeof(double) * nv * dim));
  PFEM2_CUDA(cudaMalloc(&w->e, rs * nv * dim));
  PFEM2_CUDA(cudaMalloc(&w->r, rs * nv * dim));
  PFEM2_CUDA(cudaMalloc(&w->z, rs * nv * dim));
  PFEM2_CUDA(cudaMalloc(&w->p, rs * nv * dim * 2));
  PFEM2_CUDA(cudaMalloc(&w->q, rs * nv * dim));
  PFEM2_CUDA(cudaMemset(w->p, 0, rs * nv * dim * 2));
  PFEM2_CUDA(cudaMemset(w->z, 0, rs * nv * dim));
  PFEM2_CUDA(cudaMemset(w->e, 0, rs * nv * dim));
  PFEM2_CUDA(cudaMalloc(&w->part, sizeof(double) * 2 * maxtiles));
  PFEM2_CUDA(cudaMalloc(&w->cnt, sizeof(int) * maxsys));
  PFEM2_CUDA(cudaMemset(w->cnt, 0, sizeof(int) * maxsys));
  for (int k = 0; k < 3; ++k) {
    PFEM2_CUDA(cudaMalloc(&w->sd[k], sizeof(double) * SD_N * maxsys));
    PFEM2_CUDA(cudaMalloc(&w->si[k], sizeof(int) * SI_N * maxsys));
    PFEM2_CUDA(cudaMemset(w->sd[k], 0, sizeof(double) * SD_N * maxsys));
    PFEM2_CUDA(cudaMemset(w->si[k], 0, sizeof(int) * SI_N * maxsys));
  }
  PFEM2_CUDA(cudaMalloc(&w->active, sizeof(int)));
  int nb = 0;
  PFEM2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_krylov<float>, kSolveThreads, 0));
  w->coop_blocks[0] = std::max(1, nb) * c.num_sms;
  PFEM2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_krylov<double>, kSolveThreads, 0));
  w->coop_blocks[1] = std::max(1, nb) * c.num_sms;
  c.kws = w;
  return PFEM2_OK;
}

// per-system initial scalars, uploaded before each phase (graph-capturable:
// a small kernel writes them from the instance table)
__global__ void k_init_sys(int nsys, int ninst, const double* __restrict__ tol_i,
                           const int* __restrict__ maxit_i, double* __restrict__ sd, int* __restrict__ si,
                           int* __restrict__ cnt, int* __restrict__ active, unsigned* __restrict__ barrier,
                           int* __restrict__ err) {
  for (int s = threadIdx.x; s < nsys; s += blockDim.x) {
    cnt[s] = 0;
    const int i = s % ninst;
    double* d = sd + (size_t)s * SD_N;
    int* q = si + (size_t)s * SI_N;
    d[SD_RHO] = 0.0; d[SD_ALPHA] = 0.0; d[SD_BETA] = 0.0; d[SD_RES] = 0.0;
    d[SD_INTOL] = 0.0; d[SD_RR] = 0.0; d[SD_TOL] = tol_i[i];
    q[SI_STATE] = ST_OUTER; q[SI_IT] = 0; q[SI_PAR] = 0; q[SI_DONEFLAG] = 0; q[SI_OUTER] = 0; q[SI_MAXIT] = maxit_i[i];
  }
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
  SolveArgs<R> a{};
  a.ncomp = ncomp;
  a.ninst = ni;
  a.nsys = w->nsys[ph];
  a.ntiles = w->ntiles[ph];
  a.nv = c.nv;
  a.tiles = w->tiles[ph];
  a.sys_t0 = w->sys_t0[ph];
  a.sl_ptr = c.sl_ptr;
  a.sl_len = c.sl_len;
  a.sl_col = c.sl_col;
  for (int k = 0; k < 3; ++k) {
    const int kk = k < ncomp ? k : 0;
    int m;
    if (which == 0) m = kk;
    else if (which == 1) m = 3;
    else m = 4 + kk;
    a.A64[k] = c.A64[m];
    a.Ain[k] = c.mixed ? (const R*)c.A32[m] : (const R*)c.A64[m];
    a.dinv[k] = c.mixed ? (const R*)c.dinv32[m] : (const R*)c.dinv64[m];
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
  a.r64 = w->r64;
  a.e = (R*)w->e;
  a.r = (R*)w->r;
  a.z = (R*)w->z;
  a.p = (R*)w->p;
  a.q = (R*)w->q;
  a.part = w->part;
  a.cnt = w->cnt;
  a.sd = w->sd[which];
  a.si = w->si[which];
  a.active = w->active;
  a.eta = c.mixed ? 1e-4 : 0.0;
  int mx = 0;
  for (auto& in : c.inst) mx = std::max(mx, in.cs.max_iter > 0 ? in.cs.max_iter : 10000);
  a.iter_cap = 2 * mx + 64;
  a.gb.count = c.barrier;
  a.gb.gen = c.barrier + 1;
  a.gb.err = c.d_err;
  // tolerances / max_iter per instance
  double* tol = (double*)c.sys_scalars + (which == 1 ? ni : 0);
  int* maxit = c.d_sysinfo;
  k_init_sys<<<1, 256, 0, c.stream>>>(a.nsys, ni, tol, maxit, a.sd, a.si, w->cnt, w->active, c.barrier, c.d_err);
  c.launches++;
  const int blocks = std::min(a.ntiles, w->coop_blocks[sizeof(R) == 8 ? 1 : 0]);
  void* args[] = {&a};
  PFEM2_CUDA(cudaLaunchCooperativeKernel((const void*)k_krylov<R>, dim3(blocks), dim3(kSolveThreads), args, 0, c.stream));
  c.launches++;
  return PFEM2_OK;
}

pfem2_status krylov_solve(Ctx& c, int which) {
  return c.mixed ? solve_impl<float>(c, which) : solve_impl<double>(c, which);
}

// copies per-system iteration counts / residuals into c.stats (max over
// instances); NOT_CONVERGED if any system ended above its tolerance
static pfem2_status read_stats_phase(Ctx& c, int which) {
  KrylovWs* w = (KrylovWs*)c.kws;
  const int ph = which == 1 ? 0 : 1;
  const int ns = w->nsys[ph];
  std::vector<double> sd((size_t)ns * SD_N);
  std::vector<int> si((size_t)ns * SI_N);
  PFEM2_CUDA(cudaMemcpyAsync(sd.data(), w->sd[which], sizeof(double) * sd.size(), cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(si.data(), w->si[which], sizeof(int) * si.size(), cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  const int ni = (int)c.inst.size();
  const int ncomp = which == 1 ? 1 : c.dim;
  bool notconv = false;
  for (int k = 0; k < ncomp; ++k) {
    int slot = which == 0 ? k : (which == 1 ? 3 : 4 + k);
    int it = 0;
    double res = 0.0;
    for (int i = 0; i < ni; ++i) {
      const int s = k * ni + i;
      it = std::max(it, si[(size_t)s * SI_N + SI_IT]);
      res = std::max(res, sd[(size_t)s * SD_N + SD_RES]);
      if (sd[(size_t)s * SD_N + SD_RES] > sd[(size_t)s * SD_N + SD_TOL]) notconv = true;
    }
    c.stats.iters[slot] = it;
    c.stats.residual[slot] = res;
    if (which == 1) c.stats.refinements_p = si[SI_OUTER];
  }
  return notconv ? PFEM2_NOT_CONVERGED : PFEM2_OK;
}

pfem2_status krylov_read_stats(Ctx& c) {
  pfem2_status worst = PFEM2_OK;
  for (int w = 0; w < 3; ++w) {
    pfem2_status s = read_stats_phase(c, w);
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
