// ale.cu -- the moving mesh of the reference's cylinderDyM case on the GPU:
// the pseudo-solid elasticity solve for the mesh displacement
// (problem_of_elasticity + solveU, cylinderDyM/cylinderDyM.cc:926-976,
// 886-903), the reinterpolation of the nodal fields at the displaced
// vertices (reinterpolate_fields, cylinderDyM/pfem2particle.cpp:1144-1235),
// the grid transformation (transform_grid, :1237-1261) with the rebuilt
// per-cell records, and the particles' relocation in the moved mesh
// (sort_particles_into_subdomains_and_cells, then check_empty_cells).
//
// The elasticity system couples the dim displacement components: its
// dim x dim blocks live on the scalar SELL pattern (entry 0 of a row is the
// diagonal), assembled node-centric like the flow matrices (a thread owns a
// row and sums its cells in ascending order: deterministic, no atomics),
// Dirichlet rows and columns eliminated symmetrically, then solved by one
// persistent cooperative CG kernel (Jacobi, FP64) with two grid barriers per
// iteration and per-block partial sums that every block adds in the same
// order, so that all blocks take the same decisions.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "fe.cuh"

namespace pfem2 {

constexpr int kAleThreads = 256;

__device__ __forceinline__ int ale_entry(const int* __restrict__ sl_ptr, int row, int j) {
  return sl_ptr[row >> 5] + j * 32 + (row & 31);
}

// K[ci * DIM + cj][(a, b)] += sum over the cells around a and their QGauss(2)
// points of (lambda d_ci N_a d_cj N_b + mu d_cj N_a d_ci N_b
// + delta_ci,cj mu grad N_a . grad N_b) JxW
template <int DIM>
__global__ void __launch_bounds__(128) k_elastic_assemble(int nv, const int* __restrict__ v2c_ptr,
                                                          const int* __restrict__ v2c_cell,
                                                          const unsigned char* __restrict__ v2c_loc,
                                                          const int* __restrict__ inc_slot, const double* __restrict__ X,
                                                          const int* __restrict__ cv, double lambda, double mu,
                                                          double* __restrict__ K0, double* __restrict__ K1,
                                                          double* __restrict__ K2, double* __restrict__ K3,
                                                          double* __restrict__ K4, double* __restrict__ K5,
                                                          double* __restrict__ K6, double* __restrict__ K7,
                                                          double* __restrict__ K8) {
  constexpr int NV = Dims<DIM>::NV;
  double* K[9] = {K0, K1, K2, K3, K4, K5, K6, K7, K8};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nv; row += gridDim.x * blockDim.x) {
    for (int k = v2c_ptr[row]; k < v2c_ptr[row + 1]; ++k) {
      const int c = v2c_cell[k], la = v2c_loc[k];
      LocalCell<DIM, double> L;
      double x0[DIM];
      load_local_cell<DIM, double>(X, cv, c, L, x0);
      for (int iq = 0; iq < NV; ++iq) {
        double xi[DIM];
        cell_qp_xi<DIM, double>(iq, xi);
        QP<DIM, double> q;
        eval_qp<DIM, double>(L, xi, cell_qp_w<DIM>(), -1, q);
        for (int lb = 0; lb < NV; ++lb) {
          const int e = inc_slot[(size_t)k * NV + lb];
          double gg = 0.0;
#pragma unroll
          for (int d = 0; d < DIM; ++d) gg += q.G[la][d] * q.G[lb][d];
#pragma unroll
          for (int ci = 0; ci < DIM; ++ci)
#pragma unroll
            for (int cj = 0; cj < DIM; ++cj) {
              double v = lambda * q.G[la][ci] * q.G[lb][cj] + mu * q.G[la][cj] * q.G[lb][ci];
              if (ci == cj) v += mu * gg;
              K[ci * DIM + cj][e] += v * q.JxW;
            }
        }
      }
    }
  }
}

// symmetric elimination of the constrained vertices (fix[v]: all
// components, values g[d * nv + v]): a constrained row keeps its diagonal
// blocks' diagonal (1 where it is 0: padding rows) and gets rhs = K_aa g_a;
// a free row moves its constrained columns to the right-hand side
template <int DIM>
__global__ void k_elastic_eliminate(int nv, const int* __restrict__ sl_ptr, const int* __restrict__ sl_len,
                                    const int* __restrict__ sl_col, double* __restrict__ K0, double* __restrict__ K1,
                                    double* __restrict__ K2, double* __restrict__ K3, double* __restrict__ K4,
                                    double* __restrict__ K5, double* __restrict__ K6, double* __restrict__ K7,
                                    double* __restrict__ K8, const unsigned char* __restrict__ fix,
                                    const double* __restrict__ g, double* __restrict__ rhs,
                                    double* __restrict__ dinv) {
  double* K[9] = {K0, K1, K2, K3, K4, K5, K6, K7, K8};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nv; row += gridDim.x * blockDim.x) {
    const int len = sl_len[row >> 5];
    const int e0 = ale_entry(sl_ptr, row, 0);
    if (fix[row]) {
      for (int j = 0; j < len; ++j) {
        const int e = ale_entry(sl_ptr, row, j);
        const bool diag = sl_col[e] == row && j == 0;
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int b = 0; b < DIM; ++b)
            if (!(diag && a == b)) K[a * DIM + b][e] = 0.0;
      }
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        double& d = K[a * DIM + a][e0];
        if (d == 0.0) d = 1.0;
        rhs[(size_t)a * nv + row] = d * g[(size_t)a * nv + row];
        dinv[(size_t)a * nv + row] = 1.0 / d;
      }
    } else {
      double s[DIM];
#pragma unroll
      for (int a = 0; a < DIM; ++a) s[a] = 0.0;
      for (int j = 1; j < len; ++j) {
        const int e = ale_entry(sl_ptr, row, j);
        const int col = sl_col[e];
        if (col == row || !fix[col]) continue;
#pragma unroll
        for (int a = 0; a < DIM; ++a)
#pragma unroll
          for (int b = 0; b < DIM; ++b) {
            s[a] -= K[a * DIM + b][e] * g[(size_t)b * nv + col];
            K[a * DIM + b][e] = 0.0;
          }
      }
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        rhs[(size_t)a * nv + row] = s[a];
        dinv[(size_t)a * nv + row] = 1.0 / K[a * DIM + a][e0];
      }
    }
  }
}

struct ElasticArgs {
  int nv, maxit;
  double tol, rtol;
  const int *sl_ptr, *sl_len, *sl_col;
  const double* K[9];
  const double *rhs, *dinv, *g;
  const unsigned char* fix;
  double *x, *r, *z, *q, *p;  // p: 2 buffers of [dim][nv]
  double* part;               // [2][grid][4]
  int* out;                   // iterations, converged
  double* res;                // final residual, tolerance
  GridBarrier gb;
};

// block sum of NS values in a fixed order (warp shuffles, then warp 0)
template <int NS>
__device__ __forceinline__ void block_sums(double* v, double* out) {
  __shared__ double sh[kAleThreads / 32][NS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NS; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NS; ++k) sh[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      double s = 0.0;
      for (int w = 0; w < kAleThreads / 32; ++w) s += sh[w][k];
      out[k] = s;
    }
  __syncthreads();
}

// every block adds the blocks' partials in block order (same result in all)
template <int NS>
__device__ __forceinline__ void grid_sums(const double* part, double* out) {
  __shared__ double sh[NS];
  if (threadIdx.x < 32) {
    double s[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) s[k] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += 32)
#pragma unroll
      for (int k = 0; k < NS; ++k) s[k] += __ldcg(part + (size_t)b * 4 + k);
#pragma unroll
    for (int k = 0; k < NS; ++k) s[k] = warp_sum(s[k]);
    if (threadIdx.x == 0)
#pragma unroll
      for (int k = 0; k < NS; ++k) sh[k] = s[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NS; ++k) out[k] = sh[k];
  __syncthreads();
}

// y_a(row) = sum_b sum_entries K_ab x_b(col), x_b(col) given by the functor
template <int DIM, typename XF>
__device__ __forceinline__ void kmul_row(const ElasticArgs& a, int row, XF xf, double* y) {
  const int len = a.sl_len[row >> 5];
#pragma unroll
  for (int c = 0; c < DIM; ++c) y[c] = 0.0;
  for (int j = 0; j < len; ++j) {
    const int e = ale_entry(a.sl_ptr, row, j);
    const int col = a.sl_col[e];
    double xv[DIM];
#pragma unroll
    for (int b = 0; b < DIM; ++b) xv[b] = xf(b, col);
#pragma unroll
    for (int c = 0; c < DIM; ++c)
#pragma unroll
      for (int b = 0; b < DIM; ++b) y[c] += a.K[c * DIM + b][e] * xv[b];
  }
}

// The partial sums of consecutive reductions alternate between two buffers
// of [grid][4]: a block writes reduction k + 1 while slower blocks may still
// read reduction k, and reduction k + 2 only after the barrier that all of
// them passed after reading k.
template <int DIM>
__global__ void __launch_bounds__(kAleThreads) k_elastic_cg(ElasticArgs a) {
  const size_t nv = (size_t)a.nv;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
  unsigned bar = 0;
  int red = 0;  // reductions so far (buffer parity)
  auto publish = [&](const double* v, int ns) {
    if (threadIdx.x == 0)
      for (int k = 0; k < ns; ++k) a.part[(size_t)(red & 1) * gridDim.x * 4 + blockIdx.x * 4 + k] = v[k];
  };
  auto buf = [&]() { return a.part + (size_t)(red & 1) * gridDim.x * 4; };
  // x0 = g on the constrained vertices, 0 elsewhere
  for (int row = gtid; row < a.nv; row += gstride)
#pragma unroll
    for (int c = 0; c < DIM; ++c) a.x[c * nv + row] = a.fix[row] ? a.g[c * nv + row] : 0.0;
  if (!grid_sync_ra(a.gb, bar)) return;
  // r = b - K x0, z = D^-1 r; |r|^2, |b|^2, (r, z)
  double s0[3];
  {
    double v[3] = {0.0, 0.0, 0.0};
    for (int row = gtid; row < a.nv; row += gstride) {
      double y[DIM];
      kmul_row<DIM>(a, row, [&](int b, int col) { return __ldcg(a.x + b * nv + col); }, y);
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        const double bb = a.rhs[c * nv + row], rr = bb - y[c];
        const double zz = rr * a.dinv[c * nv + row];
        a.r[c * nv + row] = rr;
        a.z[c * nv + row] = zz;
        v[0] += rr * rr;
        v[1] += bb * bb;
        v[2] += rr * zz;
      }
    }
    double out[3];
    block_sums<3>(v, out);
    publish(out, 3);
  }
  if (!grid_sync_ra(a.gb, bar)) return;
  grid_sums<3>(buf(), s0);
  ++red;
  const double tol = fmax(a.tol, a.rtol * sqrt(s0[1]));
  double res = sqrt(s0[0]), rho = s0[2], beta = 0.0;
  int it = 0, par = 0;
  bool ok = res <= tol;
  while (!ok && it < a.maxit) {
    // A: p' = z + beta p (formed on the fly at the columns), q = K p', (p', q)
    const double* po = a.p + (size_t)par * DIM * nv;
    double* pn = a.p + (size_t)(par ^ 1) * DIM * nv;
    {
      double v[1] = {0.0};
      for (int row = gtid; row < a.nv; row += gstride) {
        double y[DIM];
        kmul_row<DIM>(a, row,
                      [&](int b, int col) { return fma(beta, __ldcg(po + b * nv + col), __ldcg(a.z + b * nv + col)); }, y);
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
          const double pp = fma(beta, po[c * nv + row], a.z[c * nv + row]);
          pn[c * nv + row] = pp;
          a.q[c * nv + row] = y[c];
          v[0] += pp * y[c];
        }
      }
      double out[1];
      block_sums<1>(v, out);
      publish(out, 1);
    }
    if (!grid_sync_ra(a.gb, bar)) return;
    double pq[1];
    grid_sums<1>(buf(), pq);
    ++red;
    const double alpha = pq[0] != 0.0 ? rho / pq[0] : 0.0;
    // B: x += alpha p', r -= alpha q, z = D^-1 r, (r, z), (r, r)
    {
      double v[2] = {0.0, 0.0};
      for (int row = gtid; row < a.nv; row += gstride)
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
          const size_t i = c * nv + row;
          a.x[i] = fma(alpha, pn[i], a.x[i]);
          const double rr = fma(-alpha, a.q[i], a.r[i]);
          const double zz = rr * a.dinv[i];
          a.r[i] = rr;
          a.z[i] = zz;
          v[0] += rr * zz;
          v[1] += rr * rr;
        }
      double out[2];
      block_sums<2>(v, out);
      publish(out, 2);
    }
    if (!grid_sync_ra(a.gb, bar)) return;
    double rz[2];
    grid_sums<2>(buf(), rz);
    ++red;
    ++it;
    res = sqrt(rz[1]);
    ok = res <= tol || !(res == res);
    beta = rho != 0.0 ? rz[0] / rho : 0.0;
    rho = rz[0];
    par ^= 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.out[0] = it;
    a.out[1] = res <= tol ? 1 : 0;
    a.res[0] = res;
    a.res[1] = tol;
  }
}

// reinterpolate_fields: interior vertices take Vx, Vy(, Vz), P at their
// displaced position from the lowest-index cell around them that contains
// it (inside with tolerance 1e-5), then the others in ascending order;
// boundary vertices and vertices found nowhere keep their values
template <int DIM>
__global__ void k_reinterpolate(int nv, const double* __restrict__ X, const int* __restrict__ cv,
                                const int* __restrict__ v2c_ptr, const int* __restrict__ v2c_cell,
                                const unsigned char* __restrict__ bnd, const double* __restrict__ U0,
                                const double* __restrict__ U1, const double* __restrict__ U2,
                                const double* __restrict__ F0, const double* __restrict__ F1,
                                const double* __restrict__ F2, const double* __restrict__ F3,
                                double* __restrict__ out) {
  constexpr int NV = Dims<DIM>::NV;
  const double* U[3] = {U0, U1, U2};
  const double* F[4] = {F0, F1, F2, F3};
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    double val[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) val[k] = F[k] ? F[k][v] : 0.0;
    if (!bnd[v]) {
      for (int k = v2c_ptr[v]; k < v2c_ptr[v + 1]; ++k) {
        const int c = v2c_cell[k];
        LocalCell<DIM, double> L;
        double x0[DIM], xl[DIM], xi[DIM];
        load_local_cell<DIM, double>(X, cv, c, L, x0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) xl[d] = (X[(size_t)v * DIM + d] + U[d][v]) - x0[d];
        if (!local_inverse<DIM, double>(L, xl, xi)) continue;
        bool in = true;
#pragma unroll
        for (int d = 0; d < DIM; ++d) in = in && xi[d] >= -1e-5 && xi[d] <= 1.0 + 1e-5;
        if (!in) continue;
        double N[NV];
        shape_values<DIM, double>(xi, N);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          if (!F[f]) continue;
          double s = 0.0;
#pragma unroll
          for (int b = 0; b < NV; ++b) s += N[b] * F[f][cv[(size_t)c * NV + b]];
          val[f] = s;
        }
        break;
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) out[(size_t)k * nv + v] = val[k];
  }
}

template <int DIM>
__global__ void k_transform(int nv, double* __restrict__ X, const double* __restrict__ U0,
                            const double* __restrict__ U1, const double* __restrict__ U2) {
  const double* U[3] = {U0, U1, U2};
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
#pragma unroll
    for (int d = 0; d < DIM; ++d) X[(size_t)v * DIM + d] += U[d][v];
}

// unit direction vertex -> cell centre of every incidence (FP64 and the
// particle kernels' type)
template <int DIM>
__global__ void k_v2c_dir(int nv, const double* __restrict__ X, const int* __restrict__ cv,
                          const int* __restrict__ v2c_ptr, const int* __restrict__ v2c_cell, double* __restrict__ dir,
                          float* __restrict__ dirf) {
  constexpr int NV = Dims<DIM>::NV;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
    for (int k = v2c_ptr[v]; k < v2c_ptr[v + 1]; ++k) {
      const int c = v2c_cell[k];
      double ctr[DIM], nn = 0.0;
#pragma unroll
      for (int a = 0; a < DIM; ++a) ctr[a] = 0.0;
      for (int b = 0; b < NV; ++b)
#pragma unroll
        for (int a = 0; a < DIM; ++a) ctr[a] += X[(size_t)cv[(size_t)c * NV + b] * DIM + a];
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        ctr[a] = ctr[a] / NV - X[(size_t)v * DIM + a];
        nn += ctr[a] * ctr[a];
      }
      nn = sqrt(nn);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        dir[(size_t)k * DIM + a] = ctr[a] / nn;
        if (dirf) dirf[(size_t)k * DIM + a] = (float)(ctr[a] / nn);
      }
    }
}

static pfem2_status ale_alloc(Ctx& c) {
  if (c.ale_vec) return PFEM2_OK;
  const size_t nv = c.nv, dim = c.dim;
  auto al = [&](void** p, size_t bytes) -> pfem2_status {
    PFEM2_CUDA(cudaMalloc(p, bytes));
    PFEM2_CUDA(cudaMemset(*p, 0, bytes));
    return PFEM2_OK;
  };
  for (int k = 0; k < c.dim * c.dim; ++k) PFEM2_TRY(al((void**)&c.ale_K[k], sizeof(double) * c.nell));
  PFEM2_TRY(al((void**)&c.ale_fix, nv));
  PFEM2_TRY(al((void**)&c.ale_g, sizeof(double) * dim * nv));
  PFEM2_TRY(al((void**)&c.ale_rhs, sizeof(double) * dim * nv));
  PFEM2_TRY(al((void**)&c.ale_dinv, sizeof(double) * dim * nv));
  PFEM2_TRY(al((void**)&c.ale_vec, sizeof(double) * 6 * dim * nv));
  PFEM2_TRY(al((void**)&c.ale_new, sizeof(double) * 4 * nv));
  PFEM2_TRY(al((void**)&c.ale_out, sizeof(int) * 2));
  PFEM2_TRY(al((void**)&c.ale_res, sizeof(double) * 2));
  PFEM2_TRY(al((void**)&c.ale_flag, sizeof(int)));
  // the CG's persistent grid: every block resident
  int occ = 0;
  const void* k = c.dim == 2 ? (const void*)k_elastic_cg<2> : (const void*)k_elastic_cg<3>;
  PFEM2_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, kAleThreads, 0));
  if (occ < 1) {
    set_error("moving mesh: the elasticity solver cannot be resident");
    return PFEM2_CUDA_ERROR;
  }
  c.ale_grid = (int)std::min<long long>((long long)occ * c.num_sms, std::max<long long>(1, (c.nv + kAleThreads - 1) / kAleThreads));
  PFEM2_TRY(al((void**)&c.ale_part, sizeof(double) * 2 * 4 * c.ale_grid));
  return PFEM2_OK;
}

// boundary vertices (on any boundary face) of the mesh, once at setup
pfem2_status ale_setup(Ctx& c) {
  const int NV = 1 << c.dim, NF = 2 * c.dim;
  std::vector<unsigned char> bnd(c.nv, 0);
  for (const HostInst& in : c.inst)
    for (int ce = 0; ce < in.nc; ++ce)
      for (int f = 0; f < NF; ++f) {
        if (in.fb[(size_t)ce * NF + f] < 0) continue;
        for (int v = 0; v < NV; ++v)
          if (((v >> (f / 2)) & 1) == f % 2) bnd[in.v_off + in.cells[(size_t)ce * NV + v]] = 1;
      }
  PFEM2_CUDA(cudaMalloc((void**)&c.ale_bnd, c.nv));
  PFEM2_CUDA(cudaMemcpy(c.ale_bnd, bnd.data(), c.nv, cudaMemcpyHostToDevice));
  return PFEM2_OK;
}

void ale_free(Ctx& c) {
  void* p[] = {c.ale_bnd, c.ale_fix, c.ale_g, c.ale_rhs, c.ale_dinv, c.ale_vec, c.ale_part,
               c.ale_out, c.ale_res, c.ale_xphys, c.ale_new, c.ale_flag};
  for (void* q : p)
    if (q) cudaFree(q);
  for (int k = 0; k < 9; ++k)
    if (c.ale_K[k]) cudaFree(c.ale_K[k]);
}

pfem2_status ale_elasticity(Ctx& c, const pfem2_elasticity& e, const double* body_disp, int* iters, double* res) {
  PFEM2_TRY(ale_alloc(c));
  const int dim = c.dim, NV = 1 << dim, NF = 2 * dim;
  const size_t nv = c.nv;
  // constrained vertices: fixed boundaries (zero) and the body; padding rows
  std::vector<unsigned char> fix(nv, 0);
  std::vector<double> g(dim * nv, 0.0);
  for (const HostInst& in : c.inst) {
    for (int k = in.nv; k < in.nv_pad; ++k) fix[in.v_off + k] = 1;
    for (int ce = 0; ce < in.nc; ++ce)
      for (int f = 0; f < NF; ++f) {
        const int b = in.fb[(size_t)ce * NF + f];
        if (b < 0) continue;
        const bool isfix = b < 32 && ((e.fixed_mask >> b) & 1u), isbody = b == e.body_id;
        if (!isfix && !isbody) continue;
        for (int v = 0; v < NV; ++v)
          if (((v >> (f / 2)) & 1) == f % 2) {
            const int gv = in.v_off + in.cells[(size_t)ce * NV + v];
            fix[gv] = 1;
            for (int d = 0; d < dim; ++d) g[(size_t)d * nv + gv] = isbody ? body_disp[d] : 0.0;
          }
      }
  }
  PFEM2_CUDA(cudaMemcpyAsync(c.ale_fix, fix.data(), nv, cudaMemcpyHostToDevice, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(c.ale_g, g.data(), sizeof(double) * dim * nv, cudaMemcpyHostToDevice, c.stream));
  for (int k = 0; k < dim * dim; ++k) PFEM2_CUDA(cudaMemsetAsync(c.ale_K[k], 0, sizeof(double) * c.nell, c.stream));
  double** K = c.ale_K;
  const int grid = grid_for(c, c.nv, 128, 8);
  if (dim == 2)
    k_elastic_assemble<2><<<grid, 128, 0, c.stream>>>(c.nv, c.v2c_ptr, c.v2c_cell, c.v2c_loc, c.inc_slot, c.X, c.cv,
                                                      e.lambda, e.mu, K[0], K[1], K[2], K[3], K[4], K[5], K[6], K[7],
                                                      K[8]);
  else
    k_elastic_assemble<3><<<grid, 128, 0, c.stream>>>(c.nv, c.v2c_ptr, c.v2c_cell, c.v2c_loc, c.inc_slot, c.X, c.cv,
                                                      e.lambda, e.mu, K[0], K[1], K[2], K[3], K[4], K[5], K[6], K[7],
                                                      K[8]);
  const int g2 = grid_for(c, c.nv, 256, 8);
  if (dim == 2)
    k_elastic_eliminate<2><<<g2, 256, 0, c.stream>>>(c.nv, c.sl_ptr, c.sl_len, c.sl_col, K[0], K[1], K[2], K[3], K[4],
                                                     K[5], K[6], K[7], K[8], c.ale_fix, c.ale_g, c.ale_rhs, c.ale_dinv);
  else
    k_elastic_eliminate<3><<<g2, 256, 0, c.stream>>>(c.nv, c.sl_ptr, c.sl_len, c.sl_col, K[0], K[1], K[2], K[3], K[4],
                                                     K[5], K[6], K[7], K[8], c.ale_fix, c.ale_g, c.ale_rhs, c.ale_dinv);
  c.launches += 2;
  ElasticArgs a{};
  a.nv = c.nv;
  a.maxit = e.max_iter > 0 ? e.max_iter : 10000;
  a.tol = e.tol;
  a.rtol = e.rtol;
  a.sl_ptr = c.sl_ptr;
  a.sl_len = c.sl_len;
  a.sl_col = c.sl_col;
  for (int k = 0; k < 9; ++k) a.K[k] = K[k];
  a.rhs = c.ale_rhs;
  a.dinv = c.ale_dinv;
  a.g = c.ale_g;
  a.fix = c.ale_fix;
  const size_t blk = (size_t)dim * nv;
  a.x = c.ale_vec;
  a.r = c.ale_vec + blk;
  a.z = c.ale_vec + 2 * blk;
  a.q = c.ale_vec + 3 * blk;
  a.p = c.ale_vec + 4 * blk;
  a.part = c.ale_part;
  a.out = c.ale_out;
  a.res = c.ale_res;
  a.gb.count = c.barrier;
  a.gb.gen = c.barrier + 1;
  a.gb.err = c.d_err;
  a.gb.spin_limit = c.spin_limit;
  PFEM2_CUDA(cudaMemsetAsync(c.barrier, 0, 2 * sizeof(unsigned), c.stream));
  PFEM2_CUDA(cudaMemsetAsync(c.d_err, 0, sizeof(int), c.stream));
  PFEM2_CUDA(cudaMemsetAsync(c.ale_out, 0, 2 * sizeof(int), c.stream));
  void* args[] = {&a};
  const void* kern = dim == 2 ? (const void*)k_elastic_cg<2> : (const void*)k_elastic_cg<3>;
  PFEM2_CUDA(cudaLaunchCooperativeKernel(kern, dim3(c.ale_grid), dim3(kAleThreads), args, 0, c.stream));
  c.launches++;
  // the displacement into the fields
  for (int d = 0; d < dim; ++d)
    PFEM2_CUDA(cudaMemcpyAsync(c.F[PFEM2_FIELD_DISP_X + d], a.x + (size_t)d * nv, sizeof(double) * nv,
                               cudaMemcpyDeviceToDevice, c.stream));
  int out[2] = {0, 0}, err = 0;
  double rr[2] = {0.0, 0.0};
  PFEM2_CUDA(cudaMemcpyAsync(out, c.ale_out, sizeof(out), cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(rr, c.ale_res, sizeof(rr), cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaMemcpyAsync(&err, c.d_err, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  if (iters) *iters = out[0];
  if (res) *res = rr[0];
  if (err) {
    set_error("mesh elasticity: a wait of the solver timed out");
    c.failed = true;
    return PFEM2_TIMEOUT;
  }
  if (!out[1]) {
    set_error("mesh elasticity: the CG did not converge within max_iter");
    return PFEM2_NOT_CONVERGED;
  }
  return PFEM2_OK;
}

pfem2_status ale_move_mesh(Ctx& c) {
  PFEM2_TRY(ale_alloc(c));
  const int dim = c.dim;
  const size_t nv = c.nv;
  const double* U[3] = {c.F[PFEM2_FIELD_DISP_X], c.F[PFEM2_FIELD_DISP_Y], dim == 3 ? c.F[PFEM2_FIELD_DISP_Z] : nullptr};
  // 1. the particles' physical positions in the old mesh
  if (c.seeded) {
    if (c.ale_xphys_cap < (size_t)c.pcap) {
      if (c.ale_xphys) cudaFree(c.ale_xphys);
      PFEM2_CUDA(cudaMalloc((void**)&c.ale_xphys, sizeof(double) * dim * (size_t)c.pcap));
      c.ale_xphys_cap = c.pcap;
    }
    PFEM2_TRY(launch_particle_positions(c, c.ale_xphys));
  }
  // 2. the fields at the displaced vertices (old mesh)
  const int grid = grid_for(c, c.nv, 128, 8);
  const double* Fv[4] = {c.F[PFEM2_FIELD_VX], c.F[PFEM2_FIELD_VY], dim == 3 ? c.F[PFEM2_FIELD_VZ] : nullptr,
                         c.F[PFEM2_FIELD_P]};
  if (dim == 2)
    k_reinterpolate<2><<<grid, 128, 0, c.stream>>>(c.nv, c.X, c.cv, c.v2c_ptr, c.v2c_cell, c.ale_bnd, U[0], U[1], U[2],
                                                   Fv[0], Fv[1], Fv[2], Fv[3], c.ale_new);
  else
    k_reinterpolate<3><<<grid, 128, 0, c.stream>>>(c.nv, c.X, c.cv, c.v2c_ptr, c.v2c_cell, c.ale_bnd, U[0], U[1], U[2],
                                                   Fv[0], Fv[1], Fv[2], Fv[3], c.ale_new);
  c.launches++;
  for (int k = 0; k < 4; ++k)
    if (Fv[k])
      PFEM2_CUDA(cudaMemcpyAsync((void*)Fv[k], c.ale_new + (size_t)k * nv, sizeof(double) * nv,
                                 cudaMemcpyDeviceToDevice, c.stream));
  // the particle kernels' mirrors of V and V - V_old follow (the re-seeding
  // of check_empty_cells below interpolates V)
  PFEM2_TRY(launch_sync_real_fields(c));
  // 3. move the vertices; the per-cell records and directions follow
  if (dim == 2) k_transform<2><<<grid, 128, 0, c.stream>>>(c.nv, c.X, U[0], U[1], U[2]);
  else k_transform<3><<<grid, 128, 0, c.stream>>>(c.nv, c.X, U[0], U[1], U[2]);
  if (dim == 2)
    k_v2c_dir<2><<<grid, 128, 0, c.stream>>>(c.nv, c.X, c.cv, c.v2c_ptr, c.v2c_cell, c.v2c_dir,
                                             c.pmixed ? (float*)c.v2c_dir_r : nullptr);
  else
    k_v2c_dir<3><<<grid, 128, 0, c.stream>>>(c.nv, c.X, c.cv, c.v2c_ptr, c.v2c_cell, c.v2c_dir,
                                             c.pmixed ? (float*)c.v2c_dir_r : nullptr);
  c.launches += 2;
  PFEM2_CUDA(cudaMemsetAsync(c.ale_flag, 0, sizeof(int), c.stream));
  PFEM2_TRY(launch_cell_geo(c, c.ale_flag));
  // 4. the particles in the moved mesh, then check_empty_cells
  if (c.seeded) PFEM2_TRY(launch_relocate(c, c.ale_xphys));
  int flag = 0;
  PFEM2_CUDA(cudaMemcpyAsync(&flag, c.ale_flag, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  PFEM2_CUDA(cudaStreamSynchronize(c.stream));
  PFEM2_CUDA(cudaGetLastError());
  if (flag) {
    set_error("move_mesh: a cell turned inside out (non-positive Jacobian)");
    return PFEM2_MESH_ERROR;
  }
  return PFEM2_OK;
}

}  // namespace pfem2
