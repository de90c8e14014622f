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
// The work between two synchronisation points is a "phase". A phase ends
// with every tile publishing its partial sums and a release add on its
// system's counter; the next phase starts once the counters of the block's
// running systems show every tile of those systems done (a per-system
// barrier: the instances of a batch do not wait for each other). Every
// block that owns tiles of a system computes that system's scalars itself,
// from the per-tile partial sums of the previous phase, in a fixed order:
// no block publishes scalars and no phase waits for a finalizer.
//
// Jacobi-preconditioned systems (prediction, mass) take two phases per
// iteration:
//   A  p' = z + beta p ; q = A p'                 (p double buffered) | (p', q)
//   B  e += alpha p' ; r -= alpha q ; z = D^-1 r                     | (r, z), (r, r)
// The pressure systems are preconditioned with one multigrid V(1,1) cycle
// in additive form (amg.h) and take four:
//   B   e += alpha p' ; r' = r - alpha q (r double buffered) ;
//       b1 = R01 r' on the block's own level-1 rows, with r' formed on
//       the fly from r and q                                        | (r', r')
//   B2  b2 = Pt1^T b1 on the own level-2 rows (b1 of the whole system)
//       and their contributions to b3 = Pt2^T b2
//       (below mg_split_min rows, b2 = R02 r' with the composite R02 in
//       phase B instead, and no B2)
//   UZ  first every global read: b2 of the block's systems, b3 (summing
//       the blocks' contributions), J1 b1 on its level-1 list, J0 r on
//       its own rows; then in shared memory J2 b2, x3 = E^-1 b3,
//       x2 = J2 b2 + Pt2 x3, x1 = J1 b1 + Pt1 x2 (own and halo coarse
//       dofs, redundant across blocks); z = J0 r + Pt0 x1           | (r, z)
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

enum { S_OUT_A = 0, S_OUT_B = 1, S_A = 2, S_B = 3, S_DONE = 4, S_UZ = 5, S_B2 = 6, S_C0 = 7, S_C1 = 8 };
enum {
  ACT_NONE = 0, ACT_OUT_A = 1, ACT_OUT_B = 2, ACT_OUT_DONE = 3, ACT_A = 4, ACT_B = 5, ACT_UZ = 6, ACT_B2 = 7,
  ACT_P1 = 8,   // BiCGStab: finish the previous step, y = K^-1 p, v = A y
  ACT_P2 = 9,   // BiCGStab: e += alpha y, s = r - alpha v, t = A K^-1 s
  ACT_BF = 10,  // BiCGStab: e += omega K^-1 s before a reliable update
  ACT_C0 = 11,  // Jacobi CG: w = A u after a restart
  ACT_C1 = 12   // Jacobi CG: one iteration in one phase (single reduction)
};
// partial sums per tile: CG uses 2, BiCGStab 5 (and the FP64 residual
// phase |r|^2 and |b|^2)
constexpr int kMaxSums = 5;

constexpr int kMaxBlockTiles = 64;

// categories of per-block static data copied into shared memory at kernel
// start (every phase start's GPU-scope acquire invalidates L1, so static
// indices read from global memory would cost an L2 round trip per phase)
enum {
  ST_L0META = 1,  // slice pointers / lengths of the block's slice range
  ST_L0COL = 2,   // SELL columns of that range
  ST_MGIDX = 4,   // multigrid row pointers and local system indices
  ST_MGCOL = 8,   // multigrid columns
  ST_MGVAL = 16,  // values of the multigrid operators applied to shared vectors
  ST_MIRROR = 32, // multigrid: shared copies of the block's own rows of r, z, p, q, e
};

// a read-only array seen either in global memory (base 0) or through a
// staged shared-memory copy of its range [base, ...)
template <typename T>
struct SV {
  const T* p;
  int base;
  __device__ __forceinline__ T operator[](int i) const { return p[i - base]; }
};

template <typename R> struct SolveArgs {
  int ncomp, ninst, nsys, ntiles, nv;
  const Tile* tiles;
  const int* sys_slot0;   // [nsys+1] first partial slot of each system
  const int* sys_owner;   // [nsys] block that reports the system's result
  const int* blk_t0;      // [grid+1] first tile of each block
  const int* blk_sys;     // systems of each block, at blk_sys_off[b]
  const int* blk_sys_off;
  const int* blk_sl;      // [2 grid] slice range [s0, s1) of each block's tiles
  const int* sl_ptr;
  const int* sl_len;
  const int* sl_col;
  const double* A64[3];
  const R* Ain[3];
  const R* dinv[3];
  int stage;              // ST_* categories staged in shared memory
  int ntl_max, items_max; // per block: tiles, (tile, slice) work items
  // multigrid (pressure phase), layout of MgHost
  const int *toff1, *toff2;             // [ntiles+1]
  const int *lk1, *lk2;                 // local system index of each level-1/2 dof (in its owner block)
  const int *r01_ptr, *r01_col, *r02_ptr, *r02_col;
  const R *r01_val, *r02_val;
  int split;                            // restriction to level 2 in a phase of its own (B2)
  const int *q2_ptr, *q2_col;           // split: Pt1^T per level-2 row, global level-1 columns
  const R* q2_val;
  const int *c3_blk, *c3_ptr, *c3_col, *c3_lk, *g3_ptr, *c3_pos;
  const R* c3_val;
  R* contrib;                           // [c3 rows] contributions to b3
  const R* j0;                          // [nell]
  const int *p0_ptr, *p0_len, *p0_col;  // SELL per slice, columns into the block's level-1 list
  const R* p0_val;
  const int *blk_s1, *s1_lk, *s1_jptr, *s1_jcol, *s1_pptr, *s1_pcol;
  const R *s1_jval, *s1_pval;
  const int *blk_s2, *s2_lk, *s2_jptr, *s2_jcol, *s2_pptr, *s2_pcol;
  const R *s2_jval, *s2_pval;
  const int *blk_s3, *s3_lk, *s3_eoff, *s3_estr, *blk_e;
  const float* s3_E;
  const int *sys_D3, *sys_off3, *sys_n2, *sys_off2;
  int dmax, s1max, s2max, s3max, b2max, o2max, emax;
  R *b1, *b2;
  double* x[3];
  const double* b[3];
  const unsigned char* isd[3];
  const double* g[3];    // Dirichlet values preset in x (nullptr -> 0)
  const double* tol_i;   // per instance
  const double* rtol_i;  // per instance: stop at max(tol, rtol |b|)
  const int* maxit_i;    // per instance
  int nsum;              // partial sums per tile (2, or kMaxSums for BiCGStab)
  int bicg;              // Jacobi path: BiCGStab instead of CG
  // BiCGStab vectors (nv entries per component slot): zr = K^-1 r, y and
  // w = K^-1 v double buffered (parity L.par; y in p), the shadow residual
  // rh, s, t and kt = K^-1 t; v in q, r in r's first buffer
  R *bz, *bw, *rh, *bs, *bt, *bkt;
  // Jacobi CG with one reduction per iteration: u = D^-1 r, wh = D^-1 w and
  // sh = D^-1 s double buffered (parity L.par), w = A u and s = A p on the
  // own rows only; p in p's first buffer, r in r's first buffer
  R *cu, *cwh, *csh, *cw, *cs;
  // workspace per component slot, nv entries each; r and p: 2 buffers
  R *e, *r, *z, *p, *q;
  double* r64;
  double* part;          // [2 parities][2 sums][ntiles slots]
  unsigned* scount;      // [nsys][32]: per-system count of tile phases published (one 128-byte line each, zeroed per launch)
  int* active;
  int* out_it;           // [nsys] iterations
  double* out_res;       // [nsys] final residual norm
  double* out_tol;       // [nsys] tolerance the system was solved to
  int* out_outer;        // [nsys] FP64 residual evaluations
  double eta;
  int iter_cap;
  GridBarrier gb;
};

__device__ __forceinline__ float fma_r(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_r(double a, double b, double c) { return fma(a, b, c); }

template <int GL, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = GL / 2; o > 0; o >>= 1) v += __shfl_xor_sync(PFEM2_FULL_MASK, v, o);
  return v;
}

// acc + sum over the entries of a SELL row of val(ei) * x(col), in entry
// order, with the loads of CH entries issued before their products are
// accumulated (one memory round trip per CH entries instead of one per entry)
template <typename T, int CH = 8, typename Cols, typename Val, typename X>
__device__ __forceinline__ T sell_dot(T acc, Cols cols, int base, int len, int lane, Val val, X x) {
  for (int j0 = 0; j0 < len; j0 += CH) {
    T av[CH], xv[CH];
#pragma unroll
    for (int u = 0; u < CH; ++u) {
      const int j = j0 + u;
      if (j < len) {
        const int ei = base + j * 32 + lane;
        av[u] = val(ei);
        xv[u] = x(cols[ei]);
      } else {
        av[u] = T(0);
        xv[u] = T(0);
      }
    }
#pragma unroll
    for (int u = 0; u < CH; ++u) acc = fma_r(av[u], xv[u], acc);
  }
  return acc;
}

// x[col] from the shared mirror m of the block's own rows [own0, own0 +
// nown) when there is one, else from global memory: one generic load, no
// branch (plain loads see the other blocks' writes of the previous phase,
// which the phase start's acquire ordered before them)
template <typename R>
__device__ __forceinline__ R ldm(const R* g, const R* m, int col, int own0, int nown) {
  const unsigned o = (unsigned)(col - own0);
  const R* src = (m != nullptr && o < (unsigned)nown) ? m + o : g + col;
  return *src;
}

// acc + sum over CSR entries [k0, k1) of val(k) * x(col(k)), the lanes of a
// group of GL taking every GL-th entry, loads issued CH entries at a time
template <int GL, int CH, typename T, typename Cols, typename Val, typename X>
__device__ __forceinline__ T csr_dot(T acc, int k0, int k1, int sub, Cols cols, Val val, X x) {
  for (int kb = k0 + sub; kb < k1; kb += CH * GL) {
    T av[CH], xv[CH];
#pragma unroll
    for (int u = 0; u < CH; ++u) {
      const int k = kb + u * GL;
      if (k < k1) {
        av[u] = val[k];
        xv[u] = x(cols[k]);
      } else {
        av[u] = T(0);
        xv[u] = T(0);
      }
    }
#pragma unroll
    for (int u = 0; u < CH; ++u) acc = fma_r(av[u], xv[u], acc);
  }
  return acc;
}

struct LocalSys {
  int sys, state, it, outer, par, rpar, first, owner, maxit, act, chk;
  int t0, t1;                       // partial slots of the system
  int D3, off3, n2, off2, b2off;    // multigrid: coarse sizes and offsets
  double tol, rtol, intol, res, rz_prev, alpha, beta;
  double omega;                     // BiCGStab (rz_prev holds rho = (rh, r))
  double rr_b;                      // split restriction: r'.r' of the B phase, for the UZ decision
  double sum[kMaxSums];
};

// copies src[lo, hi) into shared memory at `cur` (16-byte aligned pieces)
// and returns the view of that range; the caller syncs before reading it
__device__ __forceinline__ size_t al16_dev(size_t b) { return (b + 15) & ~(size_t)15; }

template <typename T>
__device__ __forceinline__ SV<T> stage_range(unsigned char*& cur, const T* src, int lo, int hi) {
  T* dst = reinterpret_cast<T*>(cur);
  for (int i = threadIdx.x; i < hi - lo; i += blockDim.x) dst[i] = src[lo + i];
  cur += ((size_t)(hi - lo) * sizeof(T) + 15) & ~(size_t)15;
  return SV<T>{dst, lo};
}

template <typename T>
__device__ __forceinline__ SV<T> maybe_stage(bool on, unsigned char*& cur, const T* src, int lo, int hi) {
  return on ? stage_range(cur, src, lo, hi) : SV<T>{src, 0};
}

template <typename R, bool MG, int MINB>
__global__ void __launch_bounds__(kSolveThreads, MINB) k_krylov(SolveArgs<R> a) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  // entries of a SELL row (and of a long restriction row) whose loads are
  // issued together: more with one block per SM, which has the registers;
  // with two, nine: a Q1 row of 9 entries (2D) in one round of loads and one
  // of 27 (3D) in three (eight took two and four: channel velocity solves
  // 0.64 -> 0.61 ms, pipe 31.0 -> 26.9 ms per step)
  constexpr int CH = MINB == 1 ? 16 : 9;
  // partial sums per work item: the multigrid path (CG) needs 2
  constexpr int NSMAX = MG ? 2 : kMaxSums;
  const int NS = MG ? 2 : a.nsum;
  __shared__ LocalSys ls[kMaxLocalSys];
  __shared__ Tile stile[kMaxBlockTiles];
  __shared__ int s_nls;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t nv = (size_t)a.nv;
  const int t_lo = a.blk_t0[blockIdx.x], t_hi = a.blk_t0[blockIdx.x + 1];
  const int ntl = t_hi - t_lo;
  const bool tiles_staged = ntl <= kMaxBlockTiles;
  unsigned bar_gen = 0;

  // ---- local systems of this block
  if (threadIdx.x == 0) {
    const int o = a.blk_sys_off[blockIdx.x];
    int n = a.blk_sys_off[blockIdx.x + 1] - o;
    if (n > kMaxLocalSys) n = kMaxLocalSys;  // the host guarantees n <= kMaxLocalSys
    s_nls = n;
    int b2off = 0;
    for (int k = 0; k < n; ++k) {
      LocalSys& L = ls[k];
      const int s = a.blk_sys[o + k], inst = s % a.ninst;
      L.sys = s;
      L.state = S_OUT_A;
      L.it = L.outer = L.par = L.rpar = L.chk = 0;
      L.first = 1;
      L.owner = a.sys_owner[s] == (int)blockIdx.x;
      L.t0 = a.sys_slot0[s];
      L.t1 = a.sys_slot0[s + 1];
      L.maxit = a.maxit_i[inst];
      L.tol = a.tol_i[inst];
      L.rtol = a.rtol_i[inst];
      L.intol = 0.5 * L.tol;
      L.res = L.rz_prev = L.alpha = L.beta = L.omega = 0.0;
      for (int q = 0; q < kMaxSums; ++q) L.sum[q] = 0.0;
      L.act = ACT_NONE;
      L.D3 = L.off3 = L.n2 = L.off2 = L.b2off = 0;
      if (MG) {
        L.D3 = a.sys_D3[s];
        L.off3 = a.sys_off3[s];
        L.n2 = a.sys_n2[s];
        L.off2 = a.sys_off2[s];
        L.b2off = b2off;
        b2off += L.n2;
      }
    }
  }
  if (tiles_staged)
    for (int i = threadIdx.x; i < ntl; i += kSolveThreads) stile[i] = a.tiles[t_lo + i];
  __syncthreads();
  const int nls = s_nls;
  auto tile_at = [&](int t) -> Tile { return tiles_staged ? stile[t - t_lo] : a.tiles[t]; };

  // ---- level-0 work items: (tile, slice) pairs in tile order; item0[t] is
  // the first item of local tile t. Every item's partial sums go to spart,
  // then each tile sums its items in order (deterministic).
  double* spart = reinterpret_cast<double*>(dyn_smem);
  int* item0 = reinterpret_cast<int*>(dyn_smem + al16_dev((size_t)a.items_max * NS * sizeof(double)));
  if (threadIdx.x == 0) {
    int n = 0;
    for (int t = 0; t < ntl; ++t) {
      item0[t] = n;
      const Tile T = tile_at(t_lo + t);
      n += T.s1 - T.s0;
    }
    item0[ntl] = n;
  }
  __syncthreads();
  const int nitems = item0[ntl];
  // local tile of item `it` (binary search; tiles are few)
  auto item_tile = [&](int it) -> int {
    int lo = 0, hi = ntl - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (item0[mid] <= it) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  };
  unsigned char* dyn_rest =
      dyn_smem + al16_dev((size_t)a.items_max * NS * sizeof(double)) + al16_dev((size_t)(a.ntl_max + 1) * sizeof(int));

  // ---- shared memory: multigrid vectors, then the staged static data
  R* sx1 = reinterpret_cast<R*>(dyn_rest);
  R* sx2 = sx1 + a.s1max;
  R* sx3 = sx2 + a.s2max;
  R* sb3 = sx3 + a.s3max;
  R* sb2 = sb3 + (size_t)nls * a.dmax;
  R* sb2o = sb2 + a.b2max;  // own level-2 rows during B (systems may be in UZ meanwhile)
  float* sE = reinterpret_cast<float*>(sb2o + a.o2max);
  unsigned char* cur =
      reinterpret_cast<unsigned char*>(sE) + (((size_t)a.emax * sizeof(float) + 15) & ~(size_t)15);
  const int bs0 = a.blk_sl[2 * blockIdx.x], bs1 = a.blk_sl[2 * blockIdx.x + 1];
  const SV<int> SLp = maybe_stage<int>(a.stage & ST_L0META, cur, a.sl_ptr, bs0, bs1 + 1);
  const SV<int> SLl = maybe_stage<int>(a.stage & ST_L0META, cur, a.sl_len, bs0, bs1);
  const SV<int> SLc = maybe_stage<int>(a.stage & ST_L0COL, cur, a.sl_col, a.sl_ptr[bs0], a.sl_ptr[bs1]);
  int s1_lo = 0, s1_hi = 0, s2_lo = 0, s2_hi = 0, s3_lo = 0, s3_hi = 0, o1lo = 0, o1hi = 0, o2lo = 0, o2hi = 0;
  SV<int> LK1{}, LK2{}, R01P{}, R01C{}, R02P{}, R02C{}, Q2P{}, Q2C{}, S1K{}, J1P{}, J1C{}, P1P{}, P1C{}, S2K{}, J2P{}, J2C{}, P2P{},
      P2C{}, S3K{}, S3E{}, S3S{}, C3K{}, C3P{}, C3Q{}, C3C{}, G3P{}, P0P{}, P0L{}, P0C{};
  SV<R> P1V{}, J2V{}, P2V{}, C3V{}, P0V{}, Q2V{};
  int c3lo = 0, c3hi = 0;
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
    const int e0 = a.blk_e[blockIdx.x], ne = a.blk_e[blockIdx.x + 1] - e0;
    for (int i = threadIdx.x; i < ne; i += kSolveThreads) sE[i] = a.s3_E[e0 + i];
    const bool si = a.stage & ST_MGIDX, sc = a.stage & ST_MGCOL, sv = a.stage & ST_MGVAL;
    // level-3 rows of the block's systems (consecutive systems, consecutive rows)
    const int r3lo = nls > 0 ? ls[0].off3 : 0, r3hi = nls > 0 ? ls[nls - 1].off3 + ls[nls - 1].D3 : 0;
    c3lo = a.c3_blk[blockIdx.x];
    c3hi = a.c3_blk[blockIdx.x + 1];
    LK1 = maybe_stage<int>(si, cur, a.lk1, o1lo, o1hi);
    R01P = maybe_stage<int>(si, cur, a.r01_ptr, o1lo, o1hi + 1);
    LK2 = maybe_stage<int>(si, cur, a.lk2, o2lo, o2hi);
    R02P = maybe_stage<int>(si, cur, a.r02_ptr, o2lo, o2hi + 1);
    Q2P = maybe_stage<int>(si, cur, a.q2_ptr, o2lo, o2hi + 1);
    S1K = maybe_stage<int>(si, cur, a.s1_lk, s1_lo, s1_hi);
    J1P = maybe_stage<int>(si, cur, a.s1_jptr, s1_lo, s1_hi + 1);
    P1P = maybe_stage<int>(si, cur, a.s1_pptr, s1_lo, s1_hi + 1);
    S2K = maybe_stage<int>(si, cur, a.s2_lk, s2_lo, s2_hi);
    J2P = maybe_stage<int>(si, cur, a.s2_jptr, s2_lo, s2_hi + 1);
    P2P = maybe_stage<int>(si, cur, a.s2_pptr, s2_lo, s2_hi + 1);
    S3K = maybe_stage<int>(si, cur, a.s3_lk, s3_lo, s3_hi);
    S3E = maybe_stage<int>(si, cur, a.s3_eoff, s3_lo, s3_hi);
    S3S = maybe_stage<int>(si, cur, a.s3_estr, s3_lo, s3_hi);
    C3K = maybe_stage<int>(si, cur, a.c3_lk, c3lo, c3hi);
    C3P = maybe_stage<int>(si, cur, a.c3_ptr, c3lo, c3hi + 1);
    G3P = maybe_stage<int>(si, cur, a.g3_ptr, r3lo, r3hi + 1);
    C3Q = maybe_stage<int>(si, cur, a.c3_pos, c3lo, c3hi);
    P0P = maybe_stage<int>(si, cur, a.p0_ptr, bs0, bs1 + 1);
    P0L = maybe_stage<int>(si, cur, a.p0_len, bs0, bs1);
    R01C = maybe_stage<int>(sc, cur, a.r01_col, a.r01_ptr[o1lo], a.r01_ptr[o1hi]);
    R02C = maybe_stage<int>(sc, cur, a.r02_col, a.r02_ptr[o2lo], a.r02_ptr[o2hi]);
    Q2C = maybe_stage<int>(sc, cur, a.q2_col, a.q2_ptr[o2lo], a.q2_ptr[o2hi]);
    Q2V = maybe_stage<R>(sc, cur, a.q2_val, a.q2_ptr[o2lo], a.q2_ptr[o2hi]);
    J1C = maybe_stage<int>(sc, cur, a.s1_jcol, a.s1_jptr[s1_lo], a.s1_jptr[s1_hi]);
    P1C = maybe_stage<int>(sc, cur, a.s1_pcol, a.s1_pptr[s1_lo], a.s1_pptr[s1_hi]);
    J2C = maybe_stage<int>(sc, cur, a.s2_jcol, a.s2_jptr[s2_lo], a.s2_jptr[s2_hi]);
    P2C = maybe_stage<int>(sc, cur, a.s2_pcol, a.s2_pptr[s2_lo], a.s2_pptr[s2_hi]);
    C3C = maybe_stage<int>(sc, cur, a.c3_col, a.c3_ptr[c3lo], a.c3_ptr[c3hi]);
    P0C = maybe_stage<int>(sc, cur, a.p0_col, a.p0_ptr[bs0], a.p0_ptr[bs1]);
    P1V = maybe_stage<R>(sv, cur, a.s1_pval, a.s1_pptr[s1_lo], a.s1_pptr[s1_hi]);
    J2V = maybe_stage<R>(sv, cur, a.s2_jval, a.s2_jptr[s2_lo], a.s2_jptr[s2_hi]);
    P2V = maybe_stage<R>(sv, cur, a.s2_pval, a.s2_pptr[s2_lo], a.s2_pptr[s2_hi]);
    C3V = maybe_stage<R>(sv, cur, a.c3_val, a.c3_ptr[c3lo], a.c3_ptr[c3hi]);
    P0V = maybe_stage<R>(sv, cur, a.p0_val, a.p0_ptr[bs0], a.p0_ptr[bs1]);
  }
  const SV<R> R01V{a.r01_val, 0}, R02V{a.r02_val, 0}, J1V{a.s1_jval, 0};
  // shared mirrors of the own rows of the pressure vectors (multigrid)
  const int own0 = bs0 * 32, nown = (bs1 - bs0) * 32;
  R *mr[2] = {nullptr, nullptr}, *mz = nullptr, *mp[2] = {nullptr, nullptr}, *mq = nullptr, *me = nullptr;
  if (MG && (a.stage & ST_MIRROR)) {
    R* m = reinterpret_cast<R*>(cur);
    mr[0] = m;
    mr[1] = m + nown;
    mz = m + 2 * nown;
    mp[0] = m + 3 * nown;
    mp[1] = m + 4 * nown;
    mq = m + 5 * nown;
    me = m + 6 * nown;
    cur += al16_dev((size_t)7 * nown * sizeof(R));
  }

  // ---- init: Dirichlet values preset in x, e = 0, p = 0
  for (int it = warp; it < nitems; it += kWarps) {
    const int tl = item_tile(it);
    const Tile T = tile_at(t_lo + tl);
    const int k = T.comp;
    {
      const int sl = T.s0 + (it - item0[tl]);
      const int row = sl * 32 + lane;
      if (a.isd[k][row]) a.x[k][row] = a.g[k] ? a.g[k][row] : 0.0;
      a.e[k * nv + row] = R(0);
      a.p[(2 * k) * nv + row] = R(0);
      a.p[(2 * k + 1) * nv + row] = R(0);
      if (me) {
        me[row - own0] = R(0);
        mp[0][row - own0] = R(0);
        mp[1][row - own0] = R(0);
      }
    }
  }
  __shared__ int s_stop;
  if (!grid_sync_ra(a.gb, bar_gen)) return;

  for (int iter = 0;; ++iter) {
    if (iter >= a.iter_cap) {
      if (threadIdx.x == 0) atomicCAS(a.gb.err, 0, 2);
      break;
    }
    const double* prev = a.part + (size_t)((iter + 1) & 1) * a.ntiles * NS;
    // ---- wait for the previous phase of the block's running systems: every
    // tile adds 1 to its system's counter with a release add once its phase
    // is written, so iter x (tiles of the system) means that every tile of
    // the system has finished phase iter - 1; lane k of warp 0 polls local
    // system k, then an acquire fence (and the block barrier) orders
    // everything those blocks wrote before this phase's reads. Blocks of
    // other systems are not waited for.
    if (warp == 0) {
      bool stop = true;
      for (int k = 0; k < nls; ++k) stop &= ls[k].state == S_DONE;
      if (!stop && iter > 0) {
        const bool mine = lane < nls && ls[lane].state != S_DONE;
        const unsigned target = mine ? (unsigned)iter * (unsigned)(ls[lane].t1 - ls[lane].t0) : 0u;
        const unsigned* cnt = a.scount + (size_t)(mine ? ls[lane].sys : 0) * 32;
        unsigned spins = 0;
        for (;;) {
          const bool ok = !mine || (int)(ld_relaxed_u32(cnt) - target) >= 0;
          if (__all_sync(PFEM2_FULL_MASK, ok)) {
            fence_acq_rel_gpu();
            break;
          }
          if (__any_sync(PFEM2_FULL_MASK, ++spins > a.gb.spin_limit || *(volatile int*)a.gb.err != 0)) {
            if (lane == 0) atomicCAS(a.gb.err, 0, 1);
            stop = true;
            break;
          }
          __nanosleep(20);
        }
      }
      if (lane == 0) s_stop = stop;
    }
    __syncthreads();
    if (s_stop) break;
    // the sums of the previous phase's partials: warp q sums partial q of
    // every local system over its tiles in a fixed order (lane l adds tiles
    // l, l + 32, ..., then the warp sum), all sums in one round of loads
    if (warp < NS) {
      const int q = warp;
      for (int k = 0; k < nls; ++k) {
        const int st = ls[k].state;
        if (st == S_DONE || st == S_OUT_A || (st == S_UZ && (!ls[k].chk || a.split))) continue;
        const int t0 = ls[k].t0, t1 = ls[k].t1;
        const double* pq = prev + (size_t)q * a.ntiles;
        double sq = 0.0;
        for (int tb = t0; tb < t1; tb += 256) {
          double v[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int t = tb + u * 32 + lane;
            v[u] = t < t1 ? __ldcg(pq + t) : 0.0;
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) sq += v[u];
        }
        sq = warp_sum(sq);
        if (lane == 0) ls[k].sum[q] = sq;
      }
    }
    __syncthreads();
    // ---- decisions (thread 0; identical in every block owning the system)
    if (threadIdx.x == 0) {
      for (int k = 0; k < nls; ++k) {
        LocalSys& L = ls[k];
        int act = ACT_NONE;
        // the first FP64 residual phase also summed |b|^2: the relative tolerance
        if (L.state == S_OUT_B && L.outer == 0) L.tol = fmax(L.tol, L.rtol * sqrt(L.sum[1]));
        if (!MG && a.bicg) {
          // BiCGStab with the Jacobi preconditioner K (right-preconditioned,
          // van der Vorst 1992) over the phases OUT_A (FP64 residual),
          // OUT_B (restart: r = rh = r64, zr = K^-1 r), then P1 / P2 per
          // iteration; BF completes the iterate before a reliable update
          switch (L.state) {
            case S_OUT_A:
              act = ACT_OUT_A;
              L.state = S_OUT_B;
              break;
            case S_OUT_B:
              L.res = sqrt(L.sum[0]);
              L.outer += 1;
              if (L.res <= L.tol || L.it >= L.maxit || L.outer > L.maxit || !(L.res == L.res)) {
                act = ACT_OUT_DONE;
                L.state = S_DONE;
              } else {
                L.intol = fmax(a.eta * L.res, 0.5 * L.tol);
                L.first = 1;
                L.rz_prev = L.res * L.res;  // rho = (rh, r) with rh = r
                act = ACT_OUT_B;
                L.state = S_A;
              }
              break;
            case S_A:
              if (L.first) {
                L.beta = 0.0;
                act = ACT_P1;
                L.state = S_B;
              } else {
                // sums of P2: (t,s), (t,t), (rh,s), (rh,t), (s,s)
                const double ts = L.sum[0], tt = L.sum[1], rs = L.sum[2], rt = L.sum[3], ss = L.sum[4];
                const double om = tt > 0.0 ? ts / tt : 0.0;
                const double rr = sqrt(fmax(ss - 2.0 * om * ts + om * om * tt, 0.0));
                const double rho = rs - om * rt;
                L.omega = om;
                L.it += 1;
                if (!(om != 0.0) || !(rho != 0.0) || rr <= L.intol || L.it >= L.maxit || !(rr == rr)) {
                  act = ACT_BF;  // x += omega K^-1 s, then a reliable update
                  L.state = S_OUT_A;
                } else {
                  L.beta = (rho / L.rz_prev) * (L.alpha / om);
                  L.rz_prev = rho;
                  act = ACT_P1;
                  L.state = S_B;
                }
              }
              break;
            case S_B: {
              const double rv = L.sum[0];  // (rh, v)
              L.first = 0;
              if (!(rv != 0.0) || !(rv == rv)) {
                act = ACT_OUT_A;  // breakdown: restart from the FP64 residual
                L.state = S_OUT_B;
              } else {
                L.alpha = L.rz_prev / rv;
                act = ACT_P2;
                L.state = S_A;
              }
              break;
            }
            default:
              break;
          }
        } else if (!MG) {
          // Jacobi CG with one reduction per iteration (Chronopoulos and
          // Gear 1989): u = D^-1 r, w = A u, gamma = (r, u), delta = (w, u);
          // beta = gamma / gamma_old, alpha = gamma / (delta - beta gamma /
          // alpha_old); p = u + beta p, s = w + beta s (= A p), x += alpha p,
          // r -= alpha s. One phase per iteration (C1), the w = A u of a
          // restart in a phase of its own (C0).
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
                L.chk = 0;
                act = ACT_OUT_B;
                L.state = S_C0;
              }
              break;
            case S_C0:
              act = ACT_C0;
              L.state = S_C1;
              break;
            case S_C1: {
              // sums of the previous phase: (r, u), (w, u), (r, r)
              const double g = L.sum[0], dl = L.sum[1], rr = sqrt(L.sum[2]);
              if (!L.chk) {
                L.alpha = dl != 0.0 ? g / dl : 0.0;
                L.beta = 0.0;
                L.rz_prev = g;
                act = ACT_C1;
              } else {
                L.it += 1;
                const double be = L.rz_prev != 0.0 ? g / L.rz_prev : 0.0;
                const double den = dl - (L.alpha != 0.0 ? be * g / L.alpha : 0.0);
                if (rr <= L.intol || L.it >= L.maxit || !(rr == rr) || !(den > 0.0)) {
                  act = ACT_OUT_A;  // reliable update in FP64
                  L.state = S_OUT_B;
                } else {
                  L.beta = be;
                  L.alpha = g / den;
                  L.rz_prev = g;
                  act = ACT_C1;
                }
              }
              break;
            }
            default:
              break;
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
                L.state = a.split ? S_B2 : S_UZ;
              }
              break;
            case S_B2:
              L.rr_b = L.sum[0];
              act = ACT_B2;
              L.state = S_UZ;
              break;
            case S_UZ: {
              const double rr = sqrt(a.split ? L.rr_b : L.sum[0]);
              if (L.chk && (rr <= L.intol || L.it >= L.maxit || !(rr == rr))) {
                act = ACT_OUT_A;  // reliable update in FP64
                L.state = S_OUT_B;
              } else {
                act = ACT_UZ;
                L.state = S_A;
              }
              break;
            }
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
              L.state = a.split ? S_B2 : S_UZ;
              break;
            default:
              break;
          }
        }
        L.act = act;
      }
    }
    __syncthreads();
    // ---- coarse-level work of the block (multigrid; pressure = component 0)
    if (MG) {
      bool any_b = false, any_uz = false, any_b2 = false;
      for (int k = 0; k < nls; ++k) {
        const int act = ls[k].act;
        any_b |= act == ACT_B || act == ACT_OUT_B;
        any_uz |= act == ACT_UZ;
        any_b2 |= act == ACT_B2;
      }
      // the phase that computes b2 and the contributions to b3
      const auto b2_act = [&](int act) { return a.split ? act == ACT_B2 : (act == ACT_B || act == ACT_OUT_B); };
      if (any_b) {
        // b_l = R0l r' on the own level-l rows; after a reliable update
        // r' = r64, else r' = r - alpha q formed on the fly. Level 1: 8 lanes
        // per row; level 2 (long rows): a warp per row.
        {
          constexpr int GL = 8, NG = kSolveThreads / GL;
          const int sub = threadIdx.x % GL, grp = threadIdx.x / GL;
          for (int base = o1lo; base < o1hi; base += NG) {
            const int i = base + grp;
            R acc = R(0);
            int act = ACT_NONE;
            if (i < o1hi) {
              const LocalSys& L = ls[LK1[i]];
              act = L.act;
              const int k0 = R01P[i], k1 = R01P[i + 1];
              if (act == ACT_B) {
                const R al = R(L.alpha);
                const R* rr = a.r + (size_t)L.rpar * nv;
                const R* mrr = mr[L.rpar];
                acc = csr_dot<GL, 8, R>(acc, k0, k1, sub, R01C, R01V, [&](int j) {
                  return fma_r(-al, ldm(a.q, mq, j, own0, nown), ldm(rr, mrr, j, own0, nown));
                });
              } else if (act == ACT_OUT_B) {
                acc = csr_dot<GL, 8, R>(acc, k0, k1, sub, R01C, R01V, [&](int j) { return R(__ldcg(a.r64 + j)); });
              }
            }
            acc = group_sum<GL>(acc);
            if (sub == 0 && (act == ACT_B || act == ACT_OUT_B)) a.b1[i] = acc;
          }
        }
        if (!a.split) {
          for (int i = o2lo + warp; i < o2hi; i += kWarps) {
            const LocalSys& L = ls[LK2[i]];
            const int act = L.act;
            if (act != ACT_B && act != ACT_OUT_B) continue;
            const int k0 = R02P[i], k1 = R02P[i + 1];
            R acc = R(0);
            if (act == ACT_B) {
              const R al = R(L.alpha);
              const R* rr = a.r + (size_t)L.rpar * nv;
              const R* mrr = mr[L.rpar];
              acc = csr_dot<32, CH, R>(acc, k0, k1, lane, R02C, R02V, [&](int j) {
                return fma_r(-al, ldm(a.q, mq, j, own0, nown), ldm(rr, mrr, j, own0, nown));
              });
            } else {
              acc = csr_dot<32, CH, R>(acc, k0, k1, lane, R02C, R02V, [&](int j) { return R(__ldcg(a.r64 + j)); });
            }
            acc = warp_sum(acc);
            if (lane == 0) {
              a.b2[i] = acc;
              sb2o[i - o2lo] = acc;
            }
          }
          __syncthreads();
        }
      }
      if (any_b2) {
        // split restriction: b2 = Pt1^T b1 on the own level-2 rows (a warp
        // per row, b1 of the whole system from the previous phase)
        for (int i = o2lo + warp; i < o2hi; i += kWarps) {
          const LocalSys& L = ls[LK2[i]];
          if (L.act != ACT_B2) continue;
          R acc = csr_dot<32, CH, R>(R(0), Q2P[i], Q2P[i + 1], lane, Q2C, Q2V, [&](int c) { return __ldcg(a.b1 + c); });
          acc = warp_sum(acc);
          if (lane == 0) {
            a.b2[i] = acc;
            sb2o[i - o2lo] = acc;
          }
        }
        __syncthreads();
      }
      if (any_b2 || (any_b && !a.split)) {
        // contributions of the own level-2 rows to b3 (thread per row)
        for (int rr = c3lo + threadIdx.x; rr < c3hi; rr += kSolveThreads) {
          if (!b2_act(ls[C3K[rr]].act)) continue;
          a.contrib[C3Q[rr]] = csr_dot<1, 4, R>(R(0), C3P[rr], C3P[rr + 1], 0, C3C, C3V, [&](int c) { return sb2o[c]; });
        }
      }
      if (any_uz) {
        // every global read first: b2 of the local systems, b3 (the
        // contiguous contributions of each level-3 dof summed by a warp,
        // four dofs per warp at a time so that their loads overlap), J1 b1
        // on the level-1 list, J0 r on the own rows (into z)
        for (int k = 0; k < nls; ++k) {
          if (ls[k].act != ACT_UZ) continue;
          const int n = ls[k].n2, o = ls[k].off2;
          for (int d = threadIdx.x; d < n; d += kSolveThreads) sb2[ls[k].b2off + d] = __ldcg(a.b2 + o + d);
          const int D = ls[k].D3, o3 = ls[k].off3;
          // (blocks start at different dofs, so that they do not all read
          // the same L2 lines at the same moment)
          const int ng4 = (D + 3) / 4, rot = (int)((blockIdx.x * 7u) % (unsigned)max(ng4, 1));
          for (int g4 = warp; g4 < ng4; g4 += kWarps) {
            const int d0 = 4 * ((g4 + rot) % ng4);
            R v[4][8];
            int q0[4], q1[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              q0[r] = d0 + r < D ? G3P[o3 + d0 + r] : 0;
              q1[r] = d0 + r < D ? G3P[o3 + d0 + r + 1] : 0;
            }
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
              for (int u = 0; u < 8; ++u) {
                const int q = q0[r] + u * 32 + lane;
                v[r][u] = q < q1[r] ? __ldcg(a.contrib + q) : R(0);
              }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              R acc = R(0);
#pragma unroll
              for (int u = 0; u < 8; ++u) acc += v[r][u];
              for (int q = q0[r] + 256 + lane; q < q1[r]; q += 32) acc += __ldcg(a.contrib + q);
              acc = warp_sum(acc);
              if (lane == 0 && d0 + r < D) sb3[k * a.dmax + d0 + r] = acc;
            }
          }
        }
        {
          constexpr int GL = 2, NG = kSolveThreads / GL;
          const int sub = threadIdx.x % GL, grp = threadIdx.x / GL;
          for (int base = s1_lo; base < s1_hi; base += NG) {
            const int j = base + grp;
            R acc = R(0);
            bool on = false;
            if (j < s1_hi && ls[S1K[j]].act == ACT_UZ) {
              on = true;
              acc = csr_dot<GL, 8, R>(acc, J1P[j], J1P[j + 1], sub, J1C, J1V, [&](int c) { return __ldcg(a.b1 + c); });
            }
            acc = group_sum<GL>(acc);
            if (on && sub == 0) sx1[j - s1_lo] = acc;
          }
        }
        for (int it = warp; it < nitems; it += kWarps) {
          const int tl = item_tile(it);
          const Tile T = tile_at(t_lo + tl);
          if (ls[T.lk].act != ACT_UZ) continue;
          const R* r = a.r + (size_t)ls[T.lk].rpar * nv;
          const R* mrr = mr[ls[T.lk].rpar];
          {
            const int sl = T.s0 + (it - item0[tl]);
            const R v = sell_dot<R, CH>(
                R(0), SLc, SLp[sl], SLl[sl], lane, [&](int ei) { return __ldg(a.j0 + ei); },
                [&](int col) { return ldm(r, mrr, col, own0, nown); });
            if (mz) mz[sl * 32 + lane - own0] = v;
            else a.z[sl * 32 + lane] = v;
          }
        }
        __syncthreads();
        // J2 b2 on the level-2 list (4 lanes per row, shared memory)
        {
          constexpr int GL = 4, NG = kSolveThreads / GL;
          const int sub = threadIdx.x % GL, grp = threadIdx.x / GL;
          for (int base = s2_lo; base < s2_hi; base += NG) {
            const int j = base + grp;
            R acc = R(0);
            bool on = false;
            if (j < s2_hi) {
              const LocalSys& L = ls[S2K[j]];
              if (L.act == ACT_UZ) {
                on = true;
                const R* b2k = sb2 + L.b2off;
                acc = csr_dot<GL, 8, R>(acc, J2P[j], J2P[j + 1], sub, J2C, J2V, [&](int c) { return b2k[c]; });
              }
            }
            acc = group_sum<GL>(acc);
            if (on && sub == 0) sx2[j - s2_lo] = acc;
          }
        }
        __syncthreads();
        // x3 = E^-1 b3 on the level-3 list (4 lanes per entry, transposed rows)
        {
          constexpr int GL = 4, NG = kSolveThreads / GL;
          const int sub = threadIdx.x % GL, grp = threadIdx.x / GL;
          for (int base = s3_lo; base < s3_hi; base += NG) {
            const int j = base + grp;
            R acc = R(0);
            const int k = j < s3_hi ? S3K[j] : 0;
            const bool on = j < s3_hi && ls[k].act == ACT_UZ;
            if (on) {
              const int D = ls[k].D3, str = S3S[j];
              const float* E = sE + S3E[j];
              const R* bb = sb3 + k * a.dmax;
              for (int d = sub; d < D; d += GL) acc = fma_r(R(E[d * str]), bb[d], acc);
            }
            acc = group_sum<GL>(acc);
            if (on && sub == 0) sx3[j - s3_lo] = acc;
          }
        }
        __syncthreads();
        // x2 += Pt2 x3, then x1 += Pt1 x2 (shared memory)
        {
          constexpr int GL = 4, NG = kSolveThreads / GL;
          const int sub = threadIdx.x % GL, grp = threadIdx.x / GL;
          for (int base = s2_lo; base < s2_hi; base += NG) {
            const int j = base + grp;
            R acc = R(0);
            const bool on = j < s2_hi && ls[S2K[j]].act == ACT_UZ;
            if (on) acc = csr_dot<GL, 8, R>(acc, P2P[j], P2P[j + 1], sub, P2C, P2V, [&](int c) { return sx3[c]; });
            acc = group_sum<GL>(acc);
            if (on && sub == 0) sx2[j - s2_lo] += acc;
          }
        }
        __syncthreads();
        {
          constexpr int GL = 2, NG = kSolveThreads / GL;
          const int sub = threadIdx.x % GL, grp = threadIdx.x / GL;
          for (int base = s1_lo; base < s1_hi; base += NG) {
            const int j = base + grp;
            R acc = R(0);
            const bool on = j < s1_hi && ls[S1K[j]].act == ACT_UZ;
            if (on) acc = csr_dot<GL, 8, R>(acc, P1P[j], P1P[j + 1], sub, P1C, P1V, [&](int c) { return sx2[c]; });
            acc = group_sum<GL>(acc);
            if (on && sub == 0) sx1[j - s1_lo] += acc;
          }
        }
      }
      __syncthreads();
    }
    // ---- level-0 work on the own (tile, slice) items, a warp per item
    for (int it = warp; it < nitems; it += kWarps) {
      const int tl = item_tile(it);
      const Tile T = tile_at(t_lo + tl);
      const int sl = T.s0 + (it - item0[tl]);
      const int k = T.comp;
      const LocalSys& L = ls[T.lk];
      const int act = L.act;
      if (act == ACT_NONE) continue;
      double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0, v4 = 0.0;
      const R* dinv = a.dinv[k];
      R* e = a.e + k * nv;
      R* r = a.r + (2 * k + L.rpar) * nv;
      R* z = a.z + k * nv;
      R* q = a.q + k * nv;
      double* r64 = a.r64 + k * nv;
      if (act == ACT_OUT_A) {
        const double* A = a.A64[k];
        const double* xk = a.x[k];
        {
          const int row = sl * 32 + lane;
          const double acc = sell_dot<double, CH>(
              0.0, SLc, SLp[sl], SLl[sl], lane, [&](int ei) { return A[ei]; },
              [&](int col) { return __ldcg(xk + col) + (double)ldm(e, me, col, own0, nown); });
          const double bb = a.b[k][row];
          const double rr = bb - acc;
          r64[row] = rr;
          v0 += rr * rr;
          v1 += bb * bb;
        }
      } else if (act == ACT_OUT_B || act == ACT_OUT_DONE) {
        {
          const int row = sl * 32 + lane;
          a.x[k][row] += (double)(me ? me[row - own0] : e[row]);
          e[row] = R(0);
          if (me) me[row - own0] = R(0);
          if (act == ACT_OUT_B) {
            const R rr = R(r64[row]);
            r[row] = rr;
            if (me) mr[L.rpar][row - own0] = rr;
            if (!MG && a.bicg) {
              a.rh[k * nv + row] = rr;
              a.bz[(2 * k + L.par) * nv + row] = rr * dinv[row];
            } else if (!MG) {
              a.cu[(2 * k + L.par) * nv + row] = rr * dinv[row];
            }
          }
        }
      } else if (!MG && act == ACT_C0) {
        // w = A u, wh = D^-1 w after a restart; (r, u), (w, u), (r, r)
        const int row = sl * 32 + lane;
        const R* u = a.cu + (2 * k + L.par) * nv;
        const R* A = a.Ain[k];
        const R w = sell_dot<R, CH>(R(0), SLc, SLp[sl], SLl[sl], lane, [&](int ei) { return A[ei]; },
                                    [&](int j) { return u[j]; });
        a.cw[k * nv + row] = w;
        a.cwh[(2 * k + L.par) * nv + row] = w * dinv[row];
        const double rr = (double)r[row], uu = (double)u[row];
        v0 += rr * uu;
        v1 += (double)w * uu;
        v2 += rr * rr;
      } else if (!MG && act == ACT_C1) {
        // p = u + beta p, s = w + beta s, sh = wh + beta sh, e += alpha p,
        // r -= alpha s, u' = u - alpha sh (= D^-1 r'), w' = A u' with u'
        // formed on the fly at the columns from u, wh and the old sh, wh' =
        // D^-1 w'; (r', u'), (w', u'), (r', r'). The first iteration after a
        // restart has p = u, s = w, sh = wh.
        const int row = sl * 32 + lane;
        const bool first = L.chk == 0;
        const R al = R(L.alpha), be = R(L.beta);
        const R* uo = a.cu + (2 * k + L.par) * nv;
        const R* who = a.cwh + (2 * k + L.par) * nv;
        const R* sho = a.csh + (2 * k + L.par) * nv;
        const auto unew = [&](int j) -> R {
          const R sh = first ? who[j] : fma_r(be, sho[j], who[j]);
          return fma_r(-al, sh, uo[j]);
        };
        R* pk = a.p + (2 * k) * nv;
        R* sk = a.cs + k * nv;
        const R sh = first ? who[row] : fma_r(be, sho[row], who[row]);
        const R pp = first ? uo[row] : fma_r(be, pk[row], uo[row]);
        const R ss = first ? a.cw[k * nv + row] : fma_r(be, sk[row], a.cw[k * nv + row]);
        pk[row] = pp;
        sk[row] = ss;
        e[row] = fma_r(al, pp, e[row]);
        const R rn = fma_r(-al, ss, r[row]);
        r[row] = rn;
        const R un = unew(row);
        const R* A = a.Ain[k];
        const R w = sell_dot<R, CH>(R(0), SLc, SLp[sl], SLl[sl], lane, [&](int ei) { return A[ei]; }, unew);
        a.csh[(2 * k + (L.par ^ 1)) * nv + row] = sh;
        a.cu[(2 * k + (L.par ^ 1)) * nv + row] = un;
        a.cwh[(2 * k + (L.par ^ 1)) * nv + row] = w * dinv[row];
        a.cw[k * nv + row] = w;
        v0 += (double)rn * (double)un;
        v1 += (double)w * (double)un;
        v2 += (double)rn * (double)rn;
      } else if (!MG && act == ACT_P1) {
        // y' = zr' + beta (y - omega w), zr' = zr - alpha w - omega kt the
        // preconditioned new residual (first step after a restart: y' = zr),
        // v = A y' with y' formed on the fly at the columns, w' = K^-1 v
        const int row = sl * 32 + lane;
        const bool first = L.first != 0;
        const R al = R(L.alpha), om = R(L.omega), be = R(L.beta);
        const R* zo = a.bz + (2 * k + L.par) * nv;
        const R* wo = a.bw + (2 * k + L.par) * nv;
        const R* yo = a.p + (2 * k + L.par) * nv;
        const R* kt = a.bkt + k * nv;
        const auto ynew = [&](int j) -> R {
          if (first) return zo[j];
          const R zr = fma_r(-om, kt[j], fma_r(-al, wo[j], zo[j]));
          return fma_r(be, fma_r(-om, wo[j], yo[j]), zr);
        };
        R zr_row = zo[row];
        if (!first) {
          const R zs = fma_r(-al, wo[row], zo[row]);
          e[row] = fma_r(om, zs, e[row]);
          r[row] = fma_r(-om, a.bt[k * nv + row], a.bs[k * nv + row]);
          zr_row = fma_r(-om, kt[row], zs);
        }
        const R yrow = ynew(row);
        const R* A = a.Ain[k];
        const R acc = sell_dot<R, CH>(R(0), SLc, SLp[sl], SLl[sl], lane, [&](int ei) { return A[ei]; }, ynew);
        a.bz[(2 * k + (L.par ^ 1)) * nv + row] = zr_row;
        a.p[(2 * k + (L.par ^ 1)) * nv + row] = yrow;
        a.bw[(2 * k + (L.par ^ 1)) * nv + row] = acc * dinv[row];
        q[row] = acc;
        v0 += (double)a.rh[k * nv + row] * (double)acc;
      } else if (!MG && act == ACT_P2) {
        // e += alpha y, s = r - alpha v, t = A K^-1 s (K^-1 s = zr - alpha w
        // formed on the fly), kt = K^-1 t; sums (t,s) (t,t) (rh,s) (rh,t) (s,s)
        const int row = sl * 32 + lane;
        const R al = R(L.alpha);
        const R* zc = a.bz + (2 * k + L.par) * nv;
        const R* wc = a.bw + (2 * k + L.par) * nv;
        e[row] = fma_r(al, a.p[(2 * k + L.par) * nv + row], e[row]);
        const R sv = fma_r(-al, q[row], r[row]);
        const R* A = a.Ain[k];
        const R tv = sell_dot<R, CH>(R(0), SLc, SLp[sl], SLl[sl], lane, [&](int ei) { return A[ei]; },
                                     [&](int j) { return fma_r(-al, wc[j], zc[j]); });
        a.bs[k * nv + row] = sv;
        a.bt[k * nv + row] = tv;
        a.bkt[k * nv + row] = tv * dinv[row];
        const double rh = (double)a.rh[k * nv + row];
        v0 += (double)tv * (double)sv;
        v1 += (double)tv * (double)tv;
        v2 += rh * (double)sv;
        v3 += rh * (double)tv;
        v4 += (double)sv * (double)sv;
      } else if (!MG && act == ACT_BF) {
        // the last step's x += omega K^-1 s (K^-1 s = zr - alpha w)
        const int row = sl * 32 + lane;
        const R zs = fma_r(-R(L.alpha), a.bw[(2 * k + L.par) * nv + row], a.bz[(2 * k + L.par) * nv + row]);
        e[row] = fma_r(R(L.omega), zs, e[row]);
      } else if (act == ACT_A) {
        const R beta = R(L.beta);
        R* pn = a.p + (2 * k + L.par) * nv;
        const R* po = a.p + (2 * k + (L.par ^ 1)) * nv;
        const R* A = a.Ain[k];
        {
          const int row = sl * 32 + lane;
          const R* mpo = mp[L.par ^ 1];
          const R acc = sell_dot<R, CH>(
              R(0), SLc, SLp[sl], SLl[sl], lane, [&](int ei) { return A[ei]; },
              [&](int col) { return fma_r(beta, ldm(po, mpo, col, own0, nown), ldm(z, mz, col, own0, nown)); });
          const R pp = me ? fma_r(beta, mpo[row - own0], mz[row - own0]) : fma_r(beta, po[row], z[row]);
          pn[row] = pp;
          q[row] = acc;
          if (me) {
            mp[L.par][row - own0] = pp;
            mq[row - own0] = acc;
          }
          v0 += (double)pp * (double)acc;
        }
      } else if (act == ACT_B) {
        const R alpha = R(L.alpha);
        const R* pn = a.p + (2 * k + L.par) * nv;
        R* rn = MG ? a.r + (2 * k + (L.rpar ^ 1)) * nv : r;
        {
          const int row = sl * 32 + lane;
          R rr;
          if (me) {
            const int o = row - own0;
            const R ee = me[o] + alpha * mp[L.par][o];
            me[o] = ee;
            e[row] = ee;
            rr = fma_r(-alpha, mq[o], mr[L.rpar][o]);
            mr[L.rpar ^ 1][o] = rr;
          } else {
            e[row] += alpha * pn[row];
            rr = fma_r(-alpha, q[row], r[row]);
          }
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
        // z = J0 r (first stage) + Pt0 x1
        {
          const int row = sl * 32 + lane;
          const R acc = sell_dot<R, CH>(
              mz ? mz[row - own0] : z[row], P0C, P0P[sl], P0L[sl], lane, [&](int ei) { return P0V[ei]; },
              [&](int col) { return sx1[col]; });
          z[row] = acc;
          if (mz) mz[row - own0] = acc;
          v0 += (double)(mz ? mr[L.rpar][row - own0] : __ldcg(r + row)) * (double)acc;
        }
      }
      // the item's partial sums (warp order is fixed: deterministic)
      v0 = warp_sum(v0);
      v1 = warp_sum(v1);
      if (lane == 0) {
        spart[NS * it] = v0;
        spart[NS * it + 1] = v1;
      }
      if (NSMAX > 2 && NS > 2) {
        const double vx[3] = {warp_sum(v2), NS > 3 ? warp_sum(v3) : 0.0, NS > 4 ? warp_sum(v4) : 0.0};
        if (lane == 0)
#pragma unroll
          for (int q = 2; q < NSMAX; ++q)
            if (q < NS) spart[NS * it + q] = vx[q - 2];
      }
    }
    __syncthreads();
    // per tile: its items' partials in order, into this phase's parity buffer
    // and the tile's count on its system's counter (a release add: after
    // the block barrier above it publishes every write of the block in this
    // phase)
    for (int tl = threadIdx.x; tl < ntl; tl += kSolveThreads) {
      const Tile T = tile_at(t_lo + tl);
      if (ls[T.lk].act != ACT_NONE) {
        double sm[NSMAX];
#pragma unroll
        for (int q = 0; q < NSMAX; ++q) sm[q] = 0.0;
        for (int it = item0[tl]; it < item0[tl + 1]; ++it) {
#pragma unroll
          for (int q = 0; q < NSMAX; ++q)
            if (q < NS) sm[q] += spart[NS * it + q];
        }
        double* dst = a.part + (size_t)(iter & 1) * a.ntiles * NS + T.slot;
#pragma unroll
        for (int q = 0; q < NSMAX; ++q)
          if (q < NS) dst[(size_t)q * a.ntiles] = sm[q];
      }
      red_release_add_u32(a.scount + (size_t)T.sys * 32, 1u);
    }
    // ---- bookkeeping
    if (threadIdx.x == 0) {
      for (int k = 0; k < nls; ++k) {
        LocalSys& L = ls[k];
        if (L.act == ACT_B) {
          L.par ^= 1;
          if (MG) L.rpar ^= 1;
        }
        if (L.act == ACT_P1) L.par ^= 1;
        if (L.act == ACT_C1) {
          L.par ^= 1;
          L.chk = 1;
        }
        if (L.act == ACT_OUT_DONE && L.owner) {
          a.out_it[L.sys] = L.it;
          a.out_res[L.sys] = L.res;
          a.out_tol[L.sys] = L.tol;
          a.out_outer[L.sys] = L.outer;
          atomicSub(a.active, 1);
        }
        L.act = ACT_NONE;
      }
    }
  }
}

// ------------------------------------------------------------------ host
struct KrylovWs {
  Tile* tiles[2];
  int* sys_slot0[2];
  int* sys_owner[2];
  int* blk_t0[2];
  int* blk_sys[2];
  int* blk_sys_off[2];
  int* blk_sl[2];
  int ntiles[2], nsys[2], grid[2];
  int stage[2] = {0, 0};   // staged categories per phase
  size_t smem[2] = {0, 0}; // dynamic shared memory per phase
  std::vector<Tile> h_tiles0;
  std::vector<int> h_sys_t0_0, h_blk_t0_0;
  std::vector<int> h_blk_sl[2];
  size_t l0_meta[2] = {0, 0}, l0_col[2] = {0, 0};  // max bytes per block of the level-0 categories
  int ntl_max[2] = {0, 0}, items_max[2] = {0, 0};  // per block: tiles, (tile, slice) items
  size_t items_bytes[2] = {0, 0};                  // shared memory of the item partials and offsets
  int nsum[2] = {2, 2};                            // partial sums per tile of each phase
  bool bicg[2] = {false, false};                   // phase solved by BiCGStab
  void *bz = nullptr, *bw = nullptr, *rh = nullptr, *bs = nullptr, *bt = nullptr, *bkt = nullptr;
  void *cu = nullptr, *cwh = nullptr, *csh = nullptr, *cw = nullptr, *cs = nullptr;
  // multigrid of the pressure phase (phase 0)
  bool mg = false;
  int mg_minb = 1;  // resident blocks per SM of the pressure solve: 2 for batches (many tiles per block)
  int vel_minb = 2;  // resident blocks per SM of the velocity solves
  int nls0 = 1;
  int dmax = 1, s1max = 0, s2max = 0, s3max = 0, b2max = 0, o2max = 0, emax = 0;
  int n1 = 0, n2 = 0, n3 = 0;
  long long mg_sizes[12] = {};           // see pfem2_solver_sizes
  int *toff[4] = {}, *lk[3] = {};
  int *r01_ptr = nullptr, *r01_col = nullptr, *r02_ptr = nullptr, *r02_col = nullptr;
  int *q2_ptr = nullptr, *q2_col = nullptr;
  void* q2_val = nullptr;
  bool split = false;
  void *r01_val = nullptr, *r02_val = nullptr, *j0 = nullptr;
  int *c3_blk = nullptr, *c3_ptr = nullptr, *c3_col = nullptr, *c3_lk = nullptr, *g3_ptr = nullptr, *c3_pos = nullptr;
  void *c3_val = nullptr, *contrib = nullptr;
  int *p0_ptr = nullptr, *p0_len = nullptr, *p0_col = nullptr;
  void* p0_val = nullptr;
  int *blk_s[3] = {}, *s_lk[3] = {}, *s_jptr[3] = {}, *s_jcol[3] = {}, *s_pptr[3] = {}, *s_pcol[3] = {};
  void *s_jval[3] = {}, *s_pval[3] = {};
  int *blk_s3 = nullptr, *s3_lk = nullptr, *s3_eoff = nullptr, *s3_estr = nullptr, *blk_e = nullptr;
  float* s3_E = nullptr;
  int *sys_D3 = nullptr, *sys_off3 = nullptr, *sys_n2 = nullptr, *sys_off2 = nullptr;
  void *b1 = nullptr, *b2 = nullptr;
  void *e = nullptr, *r = nullptr, *z = nullptr, *q = nullptr, *p = nullptr;
  double* r64 = nullptr;
  double* part = nullptr;
  unsigned* scount = nullptr;
  int* active = nullptr;
  int* out_it[3];
  double* out_res[3];
  double* out_tol[3];
  int* out_outer[3];
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

static size_t al16(size_t b) { return (b + 15) & ~(size_t)15; }

// shared-memory budget of the solver kernel (dynamic part)
// shared-memory budget of a block (dynamic part) with MINB resident blocks per SM
constexpr size_t smem_budget(int minb) { return minb == 1 ? 200 * 1024 : 110 * 1024; }

template <typename R, bool MG, int MINB>
static int occupancy(size_t smem) {
  int occ = 0;
  // one process-wide upper bound, so contexts with different hierarchies coexist
  cudaFuncSetAttribute((const void*)k_krylov<R, MG, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem_budget(MINB));
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_krylov<R, MG, MINB>, kSolveThreads, smem) != cudaSuccess)
    return 0;
  return occ;
}

// the multigrid kernel with MINB resident blocks per SM
template <bool MG>
static int occupancy_any(bool mixed, int minb, size_t smem) {
  if (minb == 1) return mixed ? occupancy<float, MG, 1>(smem) : occupancy<double, MG, 1>(smem);
  return mixed ? occupancy<float, MG, 2>(smem) : occupancy<double, MG, 2>(smem);
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
  // one system of moderate size: one block per SM (its coarse lists are
  // replicated per block, so smaller blocks cost more than their extra
  // warps bring); a batch, or one system from mg_wide_min rows on (where the
  // solve is bound by memory parallelism, not by latency): two
  w->mg_minb = (c.inst.size() > 1 || (long long)c.nv >= c.mg_wide_min) ? 2 : 1;
  // a single system may be tuned to one or two blocks per SM (one block has
  // the registers of the whole SM share, two hide more latency)
  if (c.inst.size() == 1 && c.tune.p_blocks_per_sm) w->mg_minb = c.tune.p_blocks_per_sm;
  c.tune.p_blocks_per_sm = w->mg_minb;
  // the velocity solves: two blocks per SM hide more latency, one has fewer
  // blocks to wait for at every phase and the registers of the SM share
  w->vel_minb = c.tune.vel_blocks_per_sm ? c.tune.vel_blocks_per_sm : 2;
  c.tune.vel_blocks_per_sm = w->vel_minb;
  const int dim = c.dim, ni = (int)c.inst.size();
  const size_t nv = c.nv;
  const int bps = std::max(1, c.solve_blocks_per_sm);
  int maxtiles = 0, maxsys = 0;
  for (int ph = 0; ph < 2; ++ph) {
    const int ncomp = ph == 0 ? 1 : dim;
    const int nsys = ncomp * ni;
    std::vector<Tile> tiles;
    if (ph == 0) {
      // pressure: tiles = the aggregation domains of the multigrid; about
      // one per block of the persistent grid (balanced work), at most dcap
      // per system (a batch: tiles of ~8 slices, at most dcap per system,
      // so every instance gets a coarse space of its own size)
      const int dcap = ni == 1 ? (w->mg_minb == 2 ? 2 * c.num_sms : 160) : 96;
      const int nb = w->mg_minb * c.num_sms;
      long long tot_sl = 0;
      for (int i = 0; i < ni; ++i) tot_sl += c.inst[i].nv_pad / kSlice;
      for (int i = 0; i < ni; ++i) {
        const int sl0 = c.inst[i].v_off / kSlice, nsl = c.inst[i].nv_pad / kSlice;
        const long long share = ni == 1 ? std::max<long long>(1, (long long)nb * nsl / tot_sl) : (nsl + 7) / 8;
        int D = (int)std::min<long long>(std::min<long long>(share, dcap), nsl);
        const int sps = (nsl + D - 1) / D;
        for (int a = 0; a < nsl; a += sps) tiles.push_back(Tile{i, 0, sl0 + a, sl0 + std::min(nsl, a + sps), 0, 0});
      }
    } else {
      // velocity components: tiles ordered (instance, slice run, component)
      // so that the slices of a block form one contiguous range
      const long long slices = (long long)c.nslices * ncomp;
      const long long target = 4LL * bps * c.num_sms;
      int ts = (int)std::max<long long>(8, (slices + target - 1) / target);
      if (c.tune.vel_tile_slices > 0) ts = c.tune.vel_tile_slices;
      c.tune.vel_tile_slices = ts;
      for (int i = 0; i < ni; ++i) {
        const int sl0 = c.inst[i].v_off / kSlice, sl1 = (c.inst[i].v_off + c.inst[i].nv_pad) / kSlice;
        for (int a = sl0; a < sl1; a += ts)
          for (int k = 0; k < ncomp; ++k) tiles.push_back(Tile{k * ni + i, k, a, std::min(sl1, a + ts), 0, 0});
      }
    }
    const int T = (int)tiles.size();
    // partial slots: the tiles of a system, contiguous
    std::vector<int> slot0(nsys + 1, 0), cnt(nsys, 0);
    for (const Tile& t : tiles) slot0[t.sys + 1]++;
    for (int s = 0; s < nsys; ++s) slot0[s + 1] += slot0[s];
    std::vector<int> owner(nsys, -1);
    // the multigrid grid is sized before its shared memory is known
    // (mg_minb blocks per SM); krylov_setup_precond checks residency
    // afterwards. The Jacobi kernel runs two blocks per SM.
    const int occ = ph == 0 ? w->mg_minb : std::min(w->vel_minb, occupancy_any<false>(c.kmixed, w->vel_minb, 0));
    if (occ < 1) {
      set_error("krylov: the solver kernel cannot be resident");
      return PFEM2_CUDA_ERROR;
    }
    const int G = std::min(T, occ * c.num_sms);
    std::vector<int> bt0(G + 1), bsys_off(1, 0), bsys, bsl(2 * G, 0);
    // split the tile sequence where the running slice count crosses
    // b / G of the total (a tile goes to the block holding its midpoint):
    // blocks get equal work when tiles differ in size
    {
      std::vector<long long> pre(T + 1, 0);
      for (int u = 0; u < T; ++u) pre[u + 1] = pre[u] + (tiles[u].s1 - tiles[u].s0);
      bt0[0] = 0;
      int t = 0;
      for (int b = 1; b < G; ++b) {
        const long long goal = pre[T] * b / G;
        while (t < T && 2 * pre[t] + (pre[t + 1] - pre[t]) < 2 * goal) ++t;
        // every block keeps at least one tile and leaves one for each later block
        t = std::min(std::max(t, bt0[b - 1] + 1), T - (G - b));
        bt0[b] = t;
      }
      bt0[G] = T;
    }
    size_t meta = 0, col = 0;
    int ntl_max = 0, items_max = 0;
    for (int b = 0; b < G; ++b) {
      std::vector<int> lst;
      int s0 = 1 << 30, s1 = -1, items = 0;
      ntl_max = std::max(ntl_max, bt0[b + 1] - bt0[b]);
      for (int t = bt0[b]; t < bt0[b + 1]; ++t) items += tiles[t].s1 - tiles[t].s0;
      items_max = std::max(items_max, items);
      for (int t = bt0[b]; t < bt0[b + 1]; ++t) {
        Tile& tl = tiles[t];
        int k = (int)(std::find(lst.begin(), lst.end(), tl.sys) - lst.begin());
        if (k == (int)lst.size()) lst.push_back(tl.sys);
        tl.lk = k;
        tl.slot = slot0[tl.sys] + cnt[tl.sys]++;
        if (owner[tl.sys] < 0) owner[tl.sys] = b;
        s0 = std::min(s0, tl.s0);
        s1 = std::max(s1, tl.s1);
      }
      if ((int)lst.size() > kMaxLocalSys) {
        set_error("krylov: more than 16 systems would share one block (instances too small for the batch)");
        return PFEM2_INVALID_ARG;
      }
      if (ph == 0 && lst.size() > 1)
        for (size_t k = 1; k < lst.size(); ++k)
          if (lst[k] != lst[0] + (int)k) {
            set_error("krylov: pressure systems of a block must be consecutive");
            return PFEM2_INVALID_ARG;
          }
      bsys.insert(bsys.end(), lst.begin(), lst.end());
      bsys_off.push_back((int)bsys.size());
      if (s1 < s0) s0 = s1 = 0;
      // the block's tiles are ordered so that their slices form one range
      bsl[2 * b] = s0;
      bsl[2 * b + 1] = s1;
      meta = std::max(meta, al16(4 * (size_t)(s1 - s0 + 1)) + al16(4 * (size_t)(s1 - s0)));
      col = std::max(col, al16(4 * (size_t)(c.h_sl_ptr[s1] - c.h_sl_ptr[s0])));
      w->nls0 = ph == 0 ? std::max(w->nls0, (int)lst.size()) : w->nls0;
    }
    w->l0_meta[ph] = meta;
    w->l0_col[ph] = col;
    w->ntl_max[ph] = ntl_max;
    w->items_max[ph] = items_max;
    w->bicg[ph] = ph == 0 ? c.p_bicg : c.vel_bicg;
    // BiCGStab 5 sums, Jacobi CG 3 (one reduction per iteration), the
    // multigrid CG of the pressure 2
    w->nsum[ph] = w->bicg[ph] ? kMaxSums : (ph == 1 || !c.two_level ? 3 : 2);
    w->items_bytes[ph] =
        al16(sizeof(double) * w->nsum[ph] * (size_t)items_max) + al16(sizeof(int) * (size_t)(ntl_max + 1));
    if (ph == 0) {
      w->h_tiles0 = tiles;
      w->h_sys_t0_0 = slot0;
      w->h_blk_t0_0 = bt0;
    }
    // level-0 staging of the velocity solves (the pressure phase decides
    // once its multigrid data are known)
    if (ph == 1) {
      w->stage[1] = 0;
      w->smem[1] = w->items_bytes[1];
      if (w->smem[1] + meta <= smem_budget(w->vel_minb)) {
        w->stage[1] |= ST_L0META;
        w->smem[1] += meta;
      }
      if (w->smem[1] + col <= smem_budget(w->vel_minb)) {
        w->stage[1] |= ST_L0COL;
        w->smem[1] += col;
      }
      const int occ2 = occupancy_any<false>(c.kmixed, w->vel_minb, w->smem[1]);
      if (occ2 * c.num_sms < G) {
        w->stage[1] = 0;
        w->smem[1] = w->items_bytes[1];
      }
    }
    w->h_blk_sl[ph] = bsl;
    w->ntiles[ph] = T;
    w->nsys[ph] = nsys;
    w->grid[ph] = G;
    PFEM2_TRY(ws_upload(w, &w->tiles[ph], tiles));
    PFEM2_TRY(ws_upload(w, &w->sys_slot0[ph], slot0));
    PFEM2_TRY(ws_upload(w, &w->sys_owner[ph], owner));
    PFEM2_TRY(ws_upload(w, &w->blk_t0[ph], bt0));
    PFEM2_TRY(ws_upload(w, &w->blk_sys[ph], bsys));
    PFEM2_TRY(ws_upload(w, &w->blk_sys_off[ph], bsys_off));
    PFEM2_TRY(ws_upload(w, &w->blk_sl[ph], bsl));
    maxtiles = std::max(maxtiles, T);
    maxsys = std::max(maxsys, nsys);
  }
  if (c.kmixed) {
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
  PFEM2_TRY(ws_alloc(w, &w->r64, nv * dim));
  PFEM2_TRY(ws_alloc(w, &w->part, 2 * (size_t)kMaxSums * maxtiles));
  {
    // single-reduction Jacobi CG vectors: u, wh, sh double buffered, w, s
    const size_t rs = c.kmixed ? sizeof(float) : sizeof(double);
    unsigned char* b[5];
    const size_t n[5] = {2 * nv * dim, 2 * nv * dim, 2 * nv * dim, nv * dim, nv * dim};
    for (int k = 0; k < 5; ++k) PFEM2_TRY(ws_alloc(w, &b[k], n[k] * rs));
    w->cu = b[0]; w->cwh = b[1]; w->csh = b[2]; w->cw = b[3]; w->cs = b[4];
  }
  if (c.vel_bicg || c.p_bicg) {
    // BiCGStab vectors: zr and w double buffered, rh, s, t, kt
    const size_t rs = c.kmixed ? sizeof(float) : sizeof(double);
    unsigned char* b[6];
    const size_t n[6] = {2 * nv * dim, 2 * nv * dim, nv * dim, nv * dim, nv * dim, nv * dim};
    for (int k = 0; k < 6; ++k) PFEM2_TRY(ws_alloc(w, &b[k], n[k] * rs));
    w->bz = b[0]; w->bw = b[1]; w->rh = b[2]; w->bs = b[3]; w->bt = b[4]; w->bkt = b[5];
  }
  PFEM2_TRY(ws_alloc(w, &w->scount, 32 * (size_t)maxsys));
  PFEM2_TRY(ws_alloc(w, &w->active, 1));
  for (int k = 0; k < 3; ++k) {
    PFEM2_TRY(ws_alloc(w, &w->out_it[k], maxsys));
    PFEM2_TRY(ws_alloc(w, &w->out_res[k], maxsys));
    PFEM2_TRY(ws_alloc(w, &w->out_tol[k], maxsys));
    PFEM2_TRY(ws_alloc(w, &w->out_outer[k], maxsys));
  }
  // pressure phase without multigrid: level-0 staging only
  w->stage[0] = 0;
  w->smem[0] = w->items_bytes[0];
  if (w->smem[0] + w->l0_meta[0] + w->l0_col[0] <= smem_budget(2)) {
    w->stage[0] = ST_L0META | ST_L0COL;
    w->smem[0] += w->l0_meta[0] + w->l0_col[0];
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
  // large systems restrict to level 2 in a phase of their own: the composite
  // R02 of the twice-smoothed prolongators grows faster than the extra
  // synchronisation costs (3D pipe: 52M entries against Pt1's few million)
  long long nvmax = 0;
  for (const HostInst& in : c.inst) nvmax = std::max<long long>(nvmax, in.nv);
  w->split = nvmax >= c.mg_split_min;
  // the dense level-3 inverse rows of a block (up to coarse_max^2 floats)
  // must leave room in the two-blocks-per-SM shared-memory budget
  const int coarse_max = w->mg_minb == 1 ? 160 : 128;
  PFEM2_TRY(mg_build(c, A, col, len, w->h_tiles0, w->h_sys_t0_0, w->h_blk_t0_0, w->split, coarse_max, H));
  const size_t rs = c.kmixed ? sizeof(float) : sizeof(double);
  w->dmax = H.dmax;
  w->s1max = H.s1max;
  w->s2max = H.s2max;
  w->s3max = H.s3max;
  w->b2max = H.b2max;
  w->emax = H.emax;
  // shared memory: multigrid vectors and coarse-inverse rows, then the
  // static data staged per category while the budget lasts (maximum over
  // blocks of each category; the kernel stages them in the same pieces)
  for (int b = 0; b < w->grid[0]; ++b)
    w->o2max = std::max(w->o2max, H.toff[2][w->h_blk_t0_0[b + 1]] - H.toff[2][w->h_blk_t0_0[b]]);
  const size_t base = w->items_bytes[0] +
                      rs * ((size_t)H.s1max + H.s2max + H.s3max + (size_t)w->nls0 * H.dmax + H.b2max + w->o2max) +
                      al16(sizeof(float) * H.emax);
  size_t idx = 0, cols = 0, vals = 0;
  {
    const std::vector<int>& bt0 = w->h_blk_t0_0;
    const std::vector<Tile>& tl = w->h_tiles0;
    for (int b = 0; b < w->grid[0]; ++b) {
      const int t_lo = bt0[b], t_hi = bt0[b + 1];
      const int bs0 = w->h_blk_sl[0][2 * b], bs1 = w->h_blk_sl[0][2 * b + 1];
      const int o1lo = H.toff[1][t_lo], o1hi = H.toff[1][t_hi], o2lo = H.toff[2][t_lo], o2hi = H.toff[2][t_hi];
      const int s1lo = H.blk_s[1][b], s1hi = H.blk_s[1][b + 1], s2lo = H.blk_s[2][b], s2hi = H.blk_s[2][b + 1];
      const int s3lo = H.blk_s3[b], s3hi = H.blk_s3[b + 1];
      int r3lo = 0, r3hi = 0;
      if (t_hi > t_lo) {
        const int sf = tl[t_lo].sys, sl = tl[t_hi - 1].sys;
        r3lo = H.sys_off3[sf];
        r3hi = H.sys_off3[sl] + H.sys_D3[sl];
      }
      const int c3lo = H.c3_blk[b], c3hi = H.c3_blk[b + 1];
      const size_t i4 = 4;
      size_t bi = al16(i4 * (o1hi - o1lo)) + al16(i4 * (o1hi - o1lo + 1)) + al16(i4 * (o2hi - o2lo)) +
                  al16(i4 * (o2hi - o2lo + 1)) + al16(i4 * (s1hi - s1lo)) + 2 * al16(i4 * (s1hi - s1lo + 1)) +
                  al16(i4 * (s2hi - s2lo)) + 2 * al16(i4 * (s2hi - s2lo + 1)) + 3 * al16(i4 * (s3hi - s3lo)) +
                  al16(i4 * (c3hi - c3lo)) + al16(i4 * (c3hi - c3lo + 1)) + al16(i4 * (r3hi - r3lo + 1)) +
                  al16(i4 * (c3hi - c3lo)) + al16(i4 * (bs1 - bs0 + 1)) + al16(i4 * (bs1 - bs0)) +
                  al16(i4 * (o2hi - o2lo + 1));
      const size_t n01 = H.r01_ptr[o1hi] - H.r01_ptr[o1lo], n02 = H.r02_ptr[o2hi] - H.r02_ptr[o2lo];
      const size_t nq2 = H.q2_ptr[o2hi] - H.q2_ptr[o2lo];
      const size_t nj1 = H.s_jptr[1][s1hi] - H.s_jptr[1][s1lo], np1 = H.s_pptr[1][s1hi] - H.s_pptr[1][s1lo];
      const size_t nj2 = H.s_jptr[2][s2hi] - H.s_jptr[2][s2lo], np2 = H.s_pptr[2][s2hi] - H.s_pptr[2][s2lo];
      const size_t n23 = H.c3_ptr[c3hi] - H.c3_ptr[c3lo], np0 = H.p0_ptr[bs1] - H.p0_ptr[bs0];
      const size_t bc = al16(i4 * n01) + al16(i4 * n02) + al16(i4 * nq2) + al16(rs * nq2) + al16(i4 * nj1) + al16(i4 * np1) + al16(i4 * nj2) +
                        al16(i4 * np2) + al16(i4 * n23) + al16(i4 * np0);
      const size_t bv = al16(rs * np1) + al16(rs * nj2) + al16(rs * np2) + al16(rs * n23) + al16(rs * np0);
      idx = std::max(idx, bi);
      cols = std::max(cols, bc);
      vals = std::max(vals, bv);
    }
  }
  size_t smem = base;
  int stage = 0;
  size_t mirror = 0;
  for (int b = 0; b < w->grid[0]; ++b)
    mirror = std::max(mirror, al16((size_t)7 * 32 * (w->h_blk_sl[0][2 * b + 1] - w->h_blk_sl[0][2 * b]) * rs));
  const std::pair<int, size_t> cats[] = {{ST_L0META, w->l0_meta[0]}, {ST_MGIDX, idx}, {ST_MIRROR, mirror},
                                         {ST_L0COL, w->l0_col[0]}, {ST_MGCOL, cols}, {ST_MGVAL, vals}};
  for (const auto& cs : cats)
    if (smem + cs.second <= smem_budget(w->mg_minb)) {
      stage |= cs.first;
      smem += cs.second;
    }
  if (base > smem_budget(w->mg_minb)) {
    set_error("krylov: the pressure multigrid's per-block data exceed shared memory");
    return PFEM2_INVALID_ARG;
  }
  const int occ = occupancy_any<true>(c.kmixed, w->mg_minb, smem);
  if (occ * c.num_sms < w->grid[0]) {
    set_error("krylov: the multigrid solver grid cannot be resident");
    return PFEM2_CUDA_ERROR;
  }
  w->stage[0] = stage;
  w->smem[0] = smem;
  {
    const long long sz[12] = {c.nv, H.n[1], H.n[2], H.n[3], (long long)H.r01_col.size(),
                              (long long)(w->split ? H.q2_col.size() : H.r02_col.size()),
                              (long long)H.c3_col.size(), (long long)H.p0_col.size(), (long long)H.s_jcol[1].size(),
                              (long long)H.s_pcol[1].size(), (long long)H.s_jcol[2].size(),
                              (long long)H.s_pcol[2].size()};
    for (int k = 0; k < 12; ++k) w->mg_sizes[k] = sz[k];
  }
  w->n1 = H.n[1];
  w->n2 = H.n[2];
  w->n3 = H.n[3];
  for (int l = 1; l <= 2; ++l) {
    PFEM2_TRY(ws_upload(w, &w->toff[l], H.toff[l]));
    PFEM2_TRY(ws_upload(w, &w->lk[l], H.lk[l]));
  }
  PFEM2_TRY(ws_upload(w, &w->r01_ptr, H.r01_ptr));
  PFEM2_TRY(ws_upload(w, &w->r01_col, H.r01_col));
  PFEM2_TRY(ws_upload_r(w, c.kmixed, &w->r01_val, H.r01_val));
  PFEM2_TRY(ws_upload(w, &w->r02_ptr, H.r02_ptr));
  PFEM2_TRY(ws_upload(w, &w->r02_col, H.r02_col));
  PFEM2_TRY(ws_upload(w, &w->q2_ptr, H.q2_ptr));
  PFEM2_TRY(ws_upload(w, &w->q2_col, H.q2_col));
  PFEM2_TRY(ws_upload_r(w, c.kmixed, &w->q2_val, H.q2_val));
  PFEM2_TRY(ws_upload_r(w, c.kmixed, &w->r02_val, H.r02_val));
  PFEM2_TRY(ws_upload(w, &w->c3_blk, H.c3_blk));
  PFEM2_TRY(ws_upload(w, &w->c3_ptr, H.c3_ptr));
  PFEM2_TRY(ws_upload(w, &w->c3_col, H.c3_col));
  PFEM2_TRY(ws_upload(w, &w->c3_lk, H.c3_lk));
  PFEM2_TRY(ws_upload_r(w, c.kmixed, &w->c3_val, H.c3_val));
  PFEM2_TRY(ws_upload(w, &w->g3_ptr, H.g3_ptr));
  PFEM2_TRY(ws_upload(w, &w->c3_pos, H.c3_pos));
  {
    std::vector<double> zero(std::max<size_t>(1, H.c3_lk.size()), 0.0);
    PFEM2_TRY(ws_upload_r(w, c.kmixed, &w->contrib, zero));
  }
  PFEM2_TRY(ws_upload_r(w, c.kmixed, &w->j0, H.j0));
  PFEM2_TRY(ws_upload(w, &w->p0_ptr, H.p0_ptr));
  PFEM2_TRY(ws_upload(w, &w->p0_len, H.p0_len));
  PFEM2_TRY(ws_upload(w, &w->p0_col, H.p0_col));
  PFEM2_TRY(ws_upload_r(w, c.kmixed, &w->p0_val, H.p0_val));
  for (int l = 1; l <= 2; ++l) {
    PFEM2_TRY(ws_upload(w, &w->blk_s[l], H.blk_s[l]));
    PFEM2_TRY(ws_upload(w, &w->s_lk[l], H.s_sys[l]));
    PFEM2_TRY(ws_upload(w, &w->s_jptr[l], H.s_jptr[l]));
    PFEM2_TRY(ws_upload(w, &w->s_jcol[l], H.s_jcol[l]));
    PFEM2_TRY(ws_upload_r(w, c.kmixed, &w->s_jval[l], H.s_jval[l]));
    PFEM2_TRY(ws_upload(w, &w->s_pptr[l], H.s_pptr[l]));
    PFEM2_TRY(ws_upload(w, &w->s_pcol[l], H.s_pcol[l]));
    PFEM2_TRY(ws_upload_r(w, c.kmixed, &w->s_pval[l], H.s_pval[l]));
  }
  PFEM2_TRY(ws_upload(w, &w->blk_s3, H.blk_s3));
  PFEM2_TRY(ws_upload(w, &w->s3_lk, H.s3_sys));
  PFEM2_TRY(ws_upload(w, &w->s3_eoff, H.s3_eoff));
  PFEM2_TRY(ws_upload(w, &w->s3_estr, H.s3_estr));
  PFEM2_TRY(ws_upload(w, &w->blk_e, H.blk_e));
  PFEM2_TRY(ws_upload(w, &w->s3_E, H.s3_E));
  PFEM2_TRY(ws_upload(w, &w->sys_D3, H.sys_D3));
  PFEM2_TRY(ws_upload(w, &w->sys_off3, H.sys_off3));
  PFEM2_TRY(ws_upload(w, &w->sys_n2, H.sys_n2));
  PFEM2_TRY(ws_upload(w, &w->sys_off2, H.sys_off2));
  if (c.kmixed) {
    float *b1, *b2;
    PFEM2_TRY(ws_alloc(w, &b1, H.n[1]));
    PFEM2_TRY(ws_alloc(w, &b2, H.n[2]));
    w->b1 = b1; w->b2 = b2;
  } else {
    double *b1, *b2;
    PFEM2_TRY(ws_alloc(w, &b1, H.n[1]));
    PFEM2_TRY(ws_alloc(w, &b2, H.n[2]));
    w->b1 = b1; w->b2 = b2;
  }
  w->mg = true;
  return PFEM2_OK;
}

// resets the solve's state; the previous solve's exit code (1 timeout,
// 2 iteration cap) is kept as bit (1 << code) in *sticky until the host
// reads it, so that the stats read after a whole step see every solve
__global__ void k_init_solve(int nsys, int* __restrict__ active, unsigned* __restrict__ barrier,
                             int* __restrict__ err, int* __restrict__ sticky, unsigned* __restrict__ scount,
                             int ncount) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    *active = nsys;
    barrier[0] = 0;
    barrier[1] = 0;
    const int e = *err;
    if (e > 0 && e < 8) *sticky |= 1 << e;
    *err = 0;
  }
  for (int j = i; j < ncount; j += gridDim.x * blockDim.x) scount[j] = 0u;
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
  a.sys_slot0 = w->sys_slot0[ph];
  a.sys_owner = w->sys_owner[ph];
  a.blk_t0 = w->blk_t0[ph];
  a.blk_sys = w->blk_sys[ph];
  a.blk_sys_off = w->blk_sys_off[ph];
  a.blk_sl = w->blk_sl[ph];
  a.stage = w->stage[ph];
  a.ntl_max = w->ntl_max[ph];
  a.items_max = w->items_max[ph];
  a.sl_ptr = c.sl_ptr;
  a.sl_len = c.sl_len;
  a.sl_col = c.sl_col;
  if (mg) {
    a.toff1 = w->toff[1]; a.toff2 = w->toff[2];
    a.lk1 = w->lk[1]; a.lk2 = w->lk[2];
    a.r01_ptr = w->r01_ptr; a.r01_col = w->r01_col; a.r01_val = (const R*)w->r01_val;
    a.r02_ptr = w->r02_ptr; a.r02_col = w->r02_col; a.r02_val = (const R*)w->r02_val;
    a.split = w->split ? 1 : 0;
    a.q2_ptr = w->q2_ptr; a.q2_col = w->q2_col; a.q2_val = (const R*)w->q2_val;
    a.c3_blk = w->c3_blk; a.c3_ptr = w->c3_ptr; a.c3_col = w->c3_col; a.c3_lk = w->c3_lk;
    a.c3_val = (const R*)w->c3_val; a.g3_ptr = w->g3_ptr; a.c3_pos = w->c3_pos; a.contrib = (R*)w->contrib;
    a.j0 = (const R*)w->j0;
    a.p0_ptr = w->p0_ptr; a.p0_len = w->p0_len; a.p0_col = w->p0_col; a.p0_val = (const R*)w->p0_val;
    a.blk_s1 = w->blk_s[1]; a.s1_lk = w->s_lk[1]; a.s1_jptr = w->s_jptr[1]; a.s1_jcol = w->s_jcol[1];
    a.s1_jval = (const R*)w->s_jval[1]; a.s1_pptr = w->s_pptr[1]; a.s1_pcol = w->s_pcol[1];
    a.s1_pval = (const R*)w->s_pval[1];
    a.blk_s2 = w->blk_s[2]; a.s2_lk = w->s_lk[2]; a.s2_jptr = w->s_jptr[2]; a.s2_jcol = w->s_jcol[2];
    a.s2_jval = (const R*)w->s_jval[2]; a.s2_pptr = w->s_pptr[2]; a.s2_pcol = w->s_pcol[2];
    a.s2_pval = (const R*)w->s_pval[2];
    a.blk_s3 = w->blk_s3; a.s3_lk = w->s3_lk; a.s3_eoff = w->s3_eoff; a.s3_estr = w->s3_estr; a.blk_e = w->blk_e; a.s3_E = w->s3_E;
    a.sys_D3 = w->sys_D3; a.sys_off3 = w->sys_off3; a.sys_n2 = w->sys_n2; a.sys_off2 = w->sys_off2;
    a.dmax = w->dmax; a.s1max = w->s1max; a.s2max = w->s2max; a.s3max = w->s3max; a.b2max = w->b2max;
    a.emax = w->emax; a.o2max = w->o2max;
    a.b1 = (R*)w->b1; a.b2 = (R*)w->b2;
  }
  for (int k = 0; k < 3; ++k) {
    const int kk = k < ncomp ? k : 0;
    const int mtx = which == 0 ? kk : (which == 1 ? 3 : 4 + kk);
    a.A64[k] = c.A64[mtx];
    a.Ain[k] = c.kmixed ? (const R*)c.A32[mtx] : (const R*)c.A64[mtx];
    a.dinv[k] = c.kmixed ? (const R*)c.dinv32[mtx] : (const R*)c.dinv64[mtx];
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
  a.rtol_i = (const double*)c.sys_scalars + 2 * ni + (which == 1 ? ni : 0);
  a.bicg = w->bicg[ph] ? 1 : 0;
  a.nsum = mg ? 2 : w->nsum[ph];
  a.bz = (R*)w->bz; a.bw = (R*)w->bw; a.rh = (R*)w->rh; a.bs = (R*)w->bs; a.bt = (R*)w->bt; a.bkt = (R*)w->bkt;
  a.cu = (R*)w->cu; a.cwh = (R*)w->cwh; a.csh = (R*)w->csh; a.cw = (R*)w->cw; a.cs = (R*)w->cs;
  a.maxit_i = c.d_sysinfo;
  a.e = (R*)w->e; a.r = (R*)w->r; a.z = (R*)w->z; a.q = (R*)w->q; a.p = (R*)w->p;
  a.r64 = w->r64;
  a.part = w->part;
  a.scount = w->scount;
  a.active = w->active;
  a.out_it = w->out_it[which];
  a.out_res = w->out_res[which];
  a.out_tol = w->out_tol[which];
  a.out_outer = w->out_outer[which];
  a.eta = c.kmixed ? c.refine_eta : 0.0;
  int mx = 0;
  for (auto& in : c.inst) mx = std::max(mx, in.cs.max_iter > 0 ? in.cs.max_iter : 10000);
  // phases per iteration, and BiCGStab's restarts (three phases each, at most max_iter)
  a.iter_cap = (mg ? (w->split ? 4 : 3) : (a.bicg ? 5 : 4)) * mx + 256;
  a.gb.count = c.barrier;
  a.gb.gen = c.barrier + 1;
  a.gb.err = c.d_err;
  a.gb.spin_limit = c.spin_limit;
  k_init_solve<<<std::max(1, std::min(64, (32 * a.nsys + 255) / 256)), 256, 0, c.stream>>>(
      a.nsys, w->active, c.barrier, c.d_err, c.d_err_sticky, w->scount, 32 * a.nsys);
  c.launches++;
  void* args[] = {&a};
  const void* kmg = w->mg_minb == 1 ? (const void*)k_krylov<R, true, 1> : (const void*)k_krylov<R, true, 2>;
  // the Jacobi kernel: the velocity solves at vel_minb blocks per SM, a
  // pressure solve without multigrid at two
  const void* kj = (ph == 1 && w->vel_minb == 1) ? (const void*)k_krylov<R, false, 1> : (const void*)k_krylov<R, false, 2>;
  PFEM2_CUDA(cudaLaunchCooperativeKernel(mg ? kmg : kj, dim3(w->grid[ph]), dim3(kSolveThreads), args, w->smem[ph],
                                         c.stream));
  c.launches++;
  return PFEM2_OK;
}

pfem2_status krylov_solve(Ctx& c, int which) {
  return c.kmixed ? solve_impl<float>(c, which) : solve_impl<double>(c, which);
}

// per-system iteration counts / residuals into c.stats (max over
// instances); NOT_CONVERGED if a system ended above its tolerance
static pfem2_status read_stats_phase(Ctx& c, int which) {
  KrylovWs* w = (KrylovWs*)c.kws;
  const int ph = which == 1 ? 0 : 1;
  const int ns = w->nsys[ph];
  std::vector<int> it(ns), outer(ns);
  std::vector<double> res(ns), tolv(ns);
  PFEM2_CUDA(cudaMemcpyAsync(it.data(), w->out_it[which], sizeof(int) * ns, cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(res.data(), w->out_res[which], sizeof(double) * ns, cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(tolv.data(), w->out_tol[which], sizeof(double) * ns, cudaMemcpyDeviceToHost, c.stream));
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
      // (the tolerance the kernel applied: max(tol, rtol |b|))
      if (!(res[s] <= tolv[s])) notconv = true;
    }
    c.stats.iters[slot] = mit;
    c.stats.residual[slot] = mres;
    if (which == 1) c.stats.refinements_p = mo;
  }
  return notconv ? PFEM2_NOT_CONVERGED : PFEM2_OK;
}

// sub-phase times of block 0 (ns): sums, coarse, decisions, work, barrier, loop
void krylov_sizes(Ctx& c, long long* out12) {
  KrylovWs* w = (KrylovWs*)c.kws;
  for (int k = 0; k < 12; ++k) out12[k] = (w && w->mg) ? w->mg_sizes[k] : 0;
}

pfem2_status krylov_read_stats(Ctx& c) {
  pfem2_status worst = PFEM2_OK;
  for (int wch = 0; wch < 3; ++wch) {
    pfem2_status s = read_stats_phase(c, wch);
    if (s != PFEM2_OK && worst == PFEM2_OK) worst = s;
  }
  // the last solve's exit code and those of the solves before it
  int err = 0, sticky = 0;
  PFEM2_CUDA(cudaMemcpy(&err, c.d_err, sizeof(int), cudaMemcpyDeviceToHost));
  PFEM2_CUDA(cudaMemcpy(&sticky, c.d_err_sticky, sizeof(int), cudaMemcpyDeviceToHost));
  if (err > 0 && err < 8) sticky |= 1 << err;
  if (sticky) {
    PFEM2_CUDA(cudaMemset(c.d_err_sticky, 0, sizeof(int)));
    PFEM2_CUDA(cudaMemset(c.d_err, 0, sizeof(int)));
  }
  if (sticky & 2) {
    set_error("krylov: a wait for the other blocks timed out");
    c.failed = true;
    return PFEM2_TIMEOUT;
  }
  if (sticky & 4) {
    set_error("krylov: iteration cap reached");
    return PFEM2_NOT_CONVERGED;
  }
  return worst;
}

}  // namespace pfem2
