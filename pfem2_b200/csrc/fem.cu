// fem.cu -- element-by-element assembly of the fractional-step systems into
// the fixed SELL-32 pattern, Dirichlet elimination, and the load integrals.
//
// Assembly is node-centric: one thread owns one matrix row / rhs entry and
// sums the element contributions of the cells around its vertex in
// ascending cell order, so every value is produced deterministically and
// without atomics. The element terms restate (2D) cylinder2D/cylinder2D.cc:
// 412-447 (prediction), 566-597 (pressure Poisson), 629-640 (correction) and
// (3D) tubePoiseuille3D/tube.cc:231-273, 480-510, 545-555; the elimination
// restates MatrixTools::apply_boundary_values with column elimination.
#include "common.cuh"
#include "ctx.h"
#include "fe.cuh"

namespace pfem2 {

template <int DIM> __device__ __forceinline__ double face_qp_w() { return DIM == 2 ? 0.5 : 0.25; }

__device__ __forceinline__ bool is_open(unsigned mask, int b) { return b >= 0 && b < 32 && ((mask >> b) & 1u); }

// SELL entry of (row, j): sl_ptr[row/32] + j*32 + row%32
__device__ __forceinline__ int sell_entry(const int* sl_ptr, int row, int j) {
  return sl_ptr[row >> 5] + j * 32 + (row & 31);
}

// ------------------------------------------------------------ matrices
// FP64, once at setup (the matrices depend only on mesh, dt, mu and rho).
// Outputs the un-eliminated prediction matrices of every component, the
// Poisson matrix and the mass matrix.
template <int DIM>
__global__ void __launch_bounds__(128) k_assemble_matrices(
    int nv, const int* __restrict__ v2c_ptr, const int* __restrict__ v2c_cell, const unsigned char* __restrict__ v2c_loc,
    const int* __restrict__ inc_slot, const double* __restrict__ X, const int* __restrict__ cv,
    const int* __restrict__ cell_inst, const DevInst* __restrict__ inst, const int* __restrict__ sl_ptr,
    const int* __restrict__ sl_len, double* __restrict__ A0, double* __restrict__ A1, double* __restrict__ A2,
    double* __restrict__ K, double* __restrict__ M) {
  constexpr int NV = Dims<DIM>::NV;
  double* Ap[3] = {A0, A1, A2};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nv; row += gridDim.x * blockDim.x) {
    const int len = sl_len[row >> 5];
    for (int j = 0; j < len; ++j) {
      const int e = sell_entry(sl_ptr, row, j);
#pragma unroll
      for (int c = 0; c < DIM; ++c) Ap[c][e] = 0.0;
      K[e] = 0.0;
      M[e] = 0.0;
    }
    const int k0 = v2c_ptr[row], k1 = v2c_ptr[row + 1];
    if (k0 == k1) {  // padding row: identity
      const int e = sell_entry(sl_ptr, row, 0);
#pragma unroll
      for (int c = 0; c < DIM; ++c) Ap[c][e] = 1.0;
      K[e] = 1.0;
      M[e] = 1.0;
      continue;
    }
    for (int k = k0; k < k1; ++k) {
      const int c = v2c_cell[k], a = v2c_loc[k];
      const DevInst& I = inst[cell_inst[c]];
      LocalCell<DIM, double> L;
      double x0[DIM];
      load_local_cell<DIM, double>(X, cv, c, L, x0);
      double va[3][NV], vk[NV], vm[NV];
#pragma unroll
      for (int b = 0; b < NV; ++b) {
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) va[cc][b] = 0.0;
        vk[b] = 0.0;
        vm[b] = 0.0;
      }
      for (int iq = 0; iq < NV; ++iq) {
        double xi[DIM];
        cell_qp_xi<DIM, double>(iq, xi);
        QP<DIM, double> q;
        eval_qp<DIM, double>(L, xi, cell_qp_w<DIM>(), -1, q);
#pragma unroll
        for (int b = 0; b < NV; ++b) {
          double gg[DIM];
          double lap = 0.0;
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            gg[d] = q.G[a][d] * q.G[b][d];
            lap += gg[d];
          }
          const double mass = q.N[a] * q.N[b];
#pragma unroll
          for (int cc = 0; cc < DIM; ++cc) {
            // rho Ni Nj + mu dt (sum_{d != c} di dj + 4/3 ci cj)
            const double s = lap + (4.0 / 3.0 - 1.0) * gg[cc];
            va[cc][b] += (I.rho * mass + I.mu * I.dt * s) * q.JxW;
          }
          vk[b] += lap * q.JxW;
          vm[b] += mass * q.JxW;
        }
      }
#pragma unroll
      for (int b = 0; b < NV; ++b) {
        const int e = inc_slot[(size_t)k * NV + b];
#pragma unroll
        for (int cc = 0; cc < DIM; ++cc) Ap[cc][e] += va[cc][b];
        K[e] += vk[b];
        M[e] += vm[b];
      }
    }
  }
}

// Dirichlet elimination of one matrix with field table (isd, g); writes the
// rhs shift (Aorig(i,i) g_i on Dirichlet rows, sum_j Aorig(i,j) g_j over
// Dirichlet columns on free rows) and 1/diag.
__global__ void k_eliminate(int nv, const int* __restrict__ sl_ptr, const int* __restrict__ sl_len,
                            const int* __restrict__ sl_col, double* __restrict__ A, const unsigned char* __restrict__ isd,
                            const double* __restrict__ g, double* __restrict__ shift, double* __restrict__ dinv64,
                            float* __restrict__ dinv32, float* __restrict__ A32) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nv; row += gridDim.x * blockDim.x) {
    const int len = sl_len[row >> 5];
    const bool rd = isd[row] != 0;
    double s = 0.0;
    const int e0 = sell_entry(sl_ptr, row, 0);
    if (rd) {
      if (g) s = A[e0] * g[row];
    } else if (g) {
      for (int j = 1; j < len; ++j) {
        const int e = sell_entry(sl_ptr, row, j);
        const int col = sl_col[e];
        if (col != row && isd[col]) s += A[e] * g[col];
      }
    }
    if (shift) shift[row] = s;
    for (int j = 1; j < len; ++j) {
      const int e = sell_entry(sl_ptr, row, j);
      const int col = sl_col[e];
      if (col != row && (rd || isd[col])) A[e] = 0.0;
    }
    const double dg = A[e0];
    dinv64[row] = 1.0 / dg;
    dinv32[row] = (float)(1.0 / dg);
    for (int j = 0; j < len; ++j) {
      const int e = sell_entry(sl_ptr, row, j);
      A32[e] = (float)A[e];
    }
  }
}

pfem2_status assemble_matrices(Ctx& c) {
  // systems: 0..dim-1 prediction, 3 pressure, 4..4+dim-1 mass (one mass
  // assembled into slot 4 and copied before per-component elimination)
  const int grid = grid_for(c, c.nv, 128, 8);
  double* A[3] = {c.A64[0], c.A64[1], c.dim == 3 ? c.A64[2] : c.A64[2]};
  if (c.dim == 2)
    k_assemble_matrices<2><<<grid, 128, 0, c.stream>>>(c.nv, c.v2c_ptr, c.v2c_cell, c.v2c_loc, c.inc_slot, c.X, c.cv,
                                                      c.cell_inst, c.d_inst, c.sl_ptr, c.sl_len, A[0], A[1], A[2],
                                                      c.A64[3], c.A64[4]);
  else
    k_assemble_matrices<3><<<grid, 128, 0, c.stream>>>(c.nv, c.v2c_ptr, c.v2c_cell, c.v2c_loc, c.inc_slot, c.X, c.cv,
                                                      c.cell_inst, c.d_inst, c.sl_ptr, c.sl_len, A[0], A[1], A[2],
                                                      c.A64[3], c.A64[4]);
  c.launches++;
  for (int k = 1; k < c.dim; ++k)
    PFEM2_CUDA(cudaMemcpyAsync(c.A64[4 + k], c.A64[4], sizeof(double) * c.nell, cudaMemcpyDeviceToDevice, c.stream));
  const int g2 = grid_for(c, c.nv, 256, 8);
  for (int k = 0; k < c.dim; ++k) {
    k_eliminate<<<g2, 256, 0, c.stream>>>(c.nv, c.sl_ptr, c.sl_len, c.sl_col, c.A64[k], c.isdir[k], c.dirval[k],
                                          c.shift[k], c.dinv64[k], c.dinv32[k], c.A32[k]);
    k_eliminate<<<g2, 256, 0, c.stream>>>(c.nv, c.sl_ptr, c.sl_len, c.sl_col, c.A64[4 + k], c.isdir[k], nullptr,
                                          nullptr, c.dinv64[4 + k], c.dinv32[4 + k], c.A32[4 + k]);
    c.launches += 2;
  }
  k_eliminate<<<g2, 256, 0, c.stream>>>(c.nv, c.sl_ptr, c.sl_len, c.sl_col, c.A64[3], c.isdir[3], c.dirval[3],
                                        c.shift[3], c.dinv64[3], c.dinv32[3], c.A32[3]);
  c.launches++;
  PFEM2_CUDA(cudaGetLastError());
  return PFEM2_OK;
}

// ------------------------------------------------------------------ rhs
// Prediction rhs of all velocity components (R = assembly precision):
//   rho M u_old - mu dt sum_{d != c} (di Nj' - 2/3 ci dj) u_inner_d
//   + open faces: mu dt Ni T_c n_x
// followed by the Dirichlet shift.
template <int DIM, typename R>
__global__ void __launch_bounds__(128) k_rhs_prediction(
    int nv, const int* __restrict__ v2c_ptr, const int* __restrict__ v2c_cell, const unsigned char* __restrict__ v2c_loc,
    const double* __restrict__ X, const int* __restrict__ cv, const signed char* __restrict__ fb,
    const int* __restrict__ cell_inst, const DevInst* __restrict__ inst, const double* __restrict__ O0,
    const double* __restrict__ O1, const double* __restrict__ O2, const double* __restrict__ I0,
    const double* __restrict__ I1, const double* __restrict__ I2, const unsigned char* __restrict__ d0,
    const unsigned char* __restrict__ d1, const unsigned char* __restrict__ d2, const double* __restrict__ s0,
    const double* __restrict__ s1, const double* __restrict__ s2, double* __restrict__ r0, double* __restrict__ r1,
    double* __restrict__ r2) {
  constexpr int NV = Dims<DIM>::NV;
  const double* Old[3] = {O0, O1, O2};
  const double* Inn[3] = {I0, I1, I2};
  const unsigned char* isd[3] = {d0, d1, d2};
  const double* sh[3] = {s0, s1, s2};
  double* out[3] = {r0, r1, r2};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nv; row += gridDim.x * blockDim.x) {
    R acc[DIM];
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc) acc[cc] = R(0);
    const int k1 = v2c_ptr[row + 1];
    for (int k = v2c_ptr[row]; k < k1; ++k) {
      const int c = v2c_cell[k], a = v2c_loc[k];
      const DevInst& I = inst[cell_inst[c]];
      const R mdt = R(I.mu * I.dt), rho = R(I.rho);
      LocalCell<DIM, R> L;
      double x0[DIM];
      load_local_cell<DIM, R>(X, cv, c, L, x0);
      R uo[DIM][NV], ui[DIM][NV];
#pragma unroll
      for (int b = 0; b < NV; ++b) {
        const int g = cv[(size_t)c * NV + b];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          uo[d][b] = R(Old[d][g]);
          ui[d][b] = R(Inn[d][g]);
        }
      }
      for (int iq = 0; iq < NV; ++iq) {
        R xi[DIM];
        cell_qp_xi<DIM, R>(iq, xi);
        QP<DIM, R> q;
        eval_qp<DIM, R>(L, xi, R(cell_qp_w<DIM>()), -1, q);
        // sum_j Nj u_old_c(j) and sum_j dNj/dx_e u_inner_d(j)
        R uoq[DIM], gi[DIM][DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          uoq[d] = R(0);
#pragma unroll
          for (int e = 0; e < DIM; ++e) gi[d][e] = R(0);
        }
#pragma unroll
        for (int b = 0; b < NV; ++b)
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            uoq[d] += q.N[b] * uo[d][b];
#pragma unroll
            for (int e = 0; e < DIM; ++e) gi[d][e] += q.G[b][e] * ui[d][b];
          }
#pragma unroll
        for (int cc = 0; cc < DIM; ++cc) {
          R t = R(0);
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            if (d == cc) continue;
            // (di Ni)(dc u_d) - 2/3 (dc Ni)(dd u_d)
            t += q.G[a][d] * gi[d][cc] - R(2.0 / 3.0) * q.G[a][cc] * gi[d][d];
          }
          acc[cc] += (rho * q.N[a] * uoq[cc] - mdt * t) * q.JxW;
        }
      }
      for (int f = 0; f < Dims<DIM>::NF; ++f) {
        if (!is_open(I.open_mask, fb[(size_t)c * Dims<DIM>::NF + f])) continue;
        if (((a >> (f >> 1)) & 1) != (f & 1)) continue;  // vertex not on this face: N_a = 0 there
        for (int iq = 0; iq < (DIM == 2 ? 2 : 4); ++iq) {
          R xi[DIM];
          face_qp_xi<DIM, R>(f, iq, xi);
          QP<DIM, R> q;
          eval_qp<DIM, R>(L, xi, R(face_qp_w<DIM>()), f, q);
          R g[DIM][DIM];
#pragma unroll
          for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int e = 0; e < DIM; ++e) {
              R s = R(0);
#pragma unroll
              for (int b = 0; b < NV; ++b) s += q.G[b][e] * ui[d][b];
              g[d][e] = s;
            }
#pragma unroll
          for (int cc = 0; cc < DIM; ++cc) {
            R T;
            if (DIM == 2) T = cc == 0 ? (R(4.0 / 3.0) * g[0][0] - R(2.0 / 3.0) * g[1][1]) : (g[0][1] + g[1][0]);
            else T = cc == 0 ? (R(-2.0) * (g[1][1] + g[DIM - 1][DIM - 1]) / R(3.0)) : g[0][cc];
            acc[cc] += mdt * q.N[a] * T * q.n[0] * q.JxW;
          }
        }
      }
    }
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc) {
      const double v = (double)acc[cc];
      out[cc][row] = isd[cc][row] ? sh[cc][row] : v - sh[cc][row];
    }
  }
}

// Pressure rhs: rho/dt sum_j (u*_d(j) di Ni) Nj - rho/dt Ni u*_x n_x on open
// faces + G Ni n_x on open faces; then the Dirichlet shift.
template <int DIM, typename R>
__global__ void __launch_bounds__(128) k_rhs_pressure(
    int nv, const int* __restrict__ v2c_ptr, const int* __restrict__ v2c_cell, const unsigned char* __restrict__ v2c_loc,
    const double* __restrict__ X, const int* __restrict__ cv, const signed char* __restrict__ fb,
    const int* __restrict__ cell_inst, const DevInst* __restrict__ inst, const double* __restrict__ P0,
    const double* __restrict__ P1, const double* __restrict__ P2, const unsigned char* __restrict__ isd,
    const double* __restrict__ sh, double* __restrict__ out) {
  constexpr int NV = Dims<DIM>::NV;
  const double* Pr[3] = {P0, P1, P2};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nv; row += gridDim.x * blockDim.x) {
    R acc = R(0);
    const int k1 = v2c_ptr[row + 1];
    for (int k = v2c_ptr[row]; k < k1; ++k) {
      const int c = v2c_cell[k], a = v2c_loc[k];
      const DevInst& I = inst[cell_inst[c]];
      const R rdt = R(I.rho / I.dt), G = R(I.open_flux);
      LocalCell<DIM, R> L;
      double x0[DIM];
      load_local_cell<DIM, R>(X, cv, c, L, x0);
      R up[DIM][NV];
#pragma unroll
      for (int b = 0; b < NV; ++b) {
        const int g = cv[(size_t)c * NV + b];
#pragma unroll
        for (int d = 0; d < DIM; ++d) up[d][b] = R(Pr[d][g]);
      }
      for (int iq = 0; iq < NV; ++iq) {
        R xi[DIM];
        cell_qp_xi<DIM, R>(iq, xi);
        QP<DIM, R> q;
        eval_qp<DIM, R>(L, xi, R(cell_qp_w<DIM>()), -1, q);
        R s = R(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          R uq = R(0);
#pragma unroll
          for (int b = 0; b < NV; ++b) uq += q.N[b] * up[d][b];
          s += uq * q.G[a][d];
        }
        acc += rdt * s * q.JxW;
      }
      for (int f = 0; f < Dims<DIM>::NF; ++f) {
        if (!is_open(I.open_mask, fb[(size_t)c * Dims<DIM>::NF + f])) continue;
        if (((a >> (f >> 1)) & 1) != (f & 1)) continue;
        for (int iq = 0; iq < (DIM == 2 ? 2 : 4); ++iq) {
          R xi[DIM];
          face_qp_xi<DIM, R>(f, iq, xi);
          QP<DIM, R> q;
          eval_qp<DIM, R>(L, xi, R(face_qp_w<DIM>()), f, q);
          R ux = R(0);
#pragma unroll
          for (int b = 0; b < NV; ++b) ux += q.N[b] * up[0][b];
          acc -= rdt * q.N[a] * ux * q.n[0] * q.JxW;
          if (G != R(0)) acc += q.N[a] * G * q.n[0] * q.JxW;
        }
      }
    }
    out[row] = isd[row] ? sh[row] : (double)acc - sh[row];
  }
}

// Correction rhs: -dt/rho sum_j Ni dc Nj p(j); zero on Dirichlet rows.
template <int DIM, typename R>
__global__ void __launch_bounds__(128) k_rhs_correction(
    int nv, const int* __restrict__ v2c_ptr, const int* __restrict__ v2c_cell, const unsigned char* __restrict__ v2c_loc,
    const double* __restrict__ X, const int* __restrict__ cv, const int* __restrict__ cell_inst,
    const DevInst* __restrict__ inst, const double* __restrict__ P, const unsigned char* __restrict__ d0,
    const unsigned char* __restrict__ d1, const unsigned char* __restrict__ d2, double* __restrict__ r0,
    double* __restrict__ r1, double* __restrict__ r2) {
  constexpr int NV = Dims<DIM>::NV;
  const unsigned char* isd[3] = {d0, d1, d2};
  double* out[3] = {r0, r1, r2};
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nv; row += gridDim.x * blockDim.x) {
    R acc[DIM];
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc) acc[cc] = R(0);
    const int k1 = v2c_ptr[row + 1];
    for (int k = v2c_ptr[row]; k < k1; ++k) {
      const int c = v2c_cell[k], a = v2c_loc[k];
      const DevInst& I = inst[cell_inst[c]];
      const R dtr = R(I.dt / I.rho);
      LocalCell<DIM, R> L;
      double x0[DIM];
      load_local_cell<DIM, R>(X, cv, c, L, x0);
      R pp[NV];
#pragma unroll
      for (int b = 0; b < NV; ++b) pp[b] = R(P[cv[(size_t)c * NV + b]]);
      for (int iq = 0; iq < NV; ++iq) {
        R xi[DIM];
        cell_qp_xi<DIM, R>(iq, xi);
        QP<DIM, R> q;
        eval_qp<DIM, R>(L, xi, R(cell_qp_w<DIM>()), -1, q);
#pragma unroll
        for (int cc = 0; cc < DIM; ++cc) {
          R gp = R(0);
#pragma unroll
          for (int b = 0; b < NV; ++b) gp += q.G[b][cc] * pp[b];
          acc[cc] -= dtr * q.N[a] * gp * q.JxW;
        }
      }
    }
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc) out[cc][row] = isd[cc][row] ? 0.0 : (double)acc[cc];
  }
}

template <int DIM, typename R>
static void rhs_pred_impl(Ctx& c) {
  const double* O[3] = {c.F[PFEM2_FIELD_OLD_VX], c.F[PFEM2_FIELD_OLD_VY], c.F[PFEM2_FIELD_OLD_VZ]};
  const double* Iv[3] = {c.F[PFEM2_FIELD_VX], c.F[PFEM2_FIELD_VY], c.F[PFEM2_FIELD_VZ]};
  k_rhs_prediction<DIM, R><<<grid_for(c, c.nv, 128, 16), 128, 0, c.stream>>>(
      c.nv, c.v2c_ptr, c.v2c_cell, c.v2c_loc, c.X, c.cv, c.fb, c.cell_inst, c.d_inst, O[0], O[1], O[2], Iv[0], Iv[1],
      Iv[2], c.isdir[0], c.isdir[1], c.isdir[2], c.shift[0], c.shift[1], c.shift[2], c.rhs[0], c.rhs[1], c.rhs[2]);
  c.launches++;
}
pfem2_status launch_rhs_prediction(Ctx& c) {
  if (c.dim == 2) { if (c.amixed) rhs_pred_impl<2, float>(c); else rhs_pred_impl<2, double>(c); }
  else { if (c.amixed) rhs_pred_impl<3, float>(c); else rhs_pred_impl<3, double>(c); }
  return PFEM2_OK;
}

template <int DIM, typename R>
static void rhs_p_impl(Ctx& c) {
  k_rhs_pressure<DIM, R><<<grid_for(c, c.nv, 128, 16), 128, 0, c.stream>>>(
      c.nv, c.v2c_ptr, c.v2c_cell, c.v2c_loc, c.X, c.cv, c.fb, c.cell_inst, c.d_inst, c.F[PFEM2_FIELD_PRED_VX],
      c.F[PFEM2_FIELD_PRED_VY], c.F[PFEM2_FIELD_PRED_VZ], c.isdir[3], c.shift[3], c.rhs[0]);
  c.launches++;
}
pfem2_status launch_rhs_pressure(Ctx& c) {
  if (c.dim == 2) { if (c.prmixed) rhs_p_impl<2, float>(c); else rhs_p_impl<2, double>(c); }
  else { if (c.prmixed) rhs_p_impl<3, float>(c); else rhs_p_impl<3, double>(c); }
  return PFEM2_OK;
}

template <int DIM, typename R>
static void rhs_c_impl(Ctx& c) {
  k_rhs_correction<DIM, R><<<grid_for(c, c.nv, 128, 16), 128, 0, c.stream>>>(
      c.nv, c.v2c_ptr, c.v2c_cell, c.v2c_loc, c.X, c.cv, c.cell_inst, c.d_inst, c.F[PFEM2_FIELD_P], c.isdir[0],
      c.isdir[1], c.isdir[2], c.rhs[0], c.rhs[1], c.rhs[2]);
  c.launches++;
}
pfem2_status launch_rhs_correction(Ctx& c) {
  if (c.dim == 2) { if (c.amixed) rhs_c_impl<2, float>(c); else rhs_c_impl<2, double>(c); }
  else { if (c.amixed) rhs_c_impl<3, float>(c); else rhs_c_impl<3, double>(c); }
  return PFEM2_OK;
}

// u = u* + du, P_old = P, and the Real mirrors of the particle kernels
template <int DIM, typename R>
__global__ void k_finish(int nv, double* __restrict__ V0, double* __restrict__ V1, double* __restrict__ V2,
                         const double* __restrict__ P0, const double* __restrict__ P1, const double* __restrict__ P2,
                         const double* __restrict__ C0, const double* __restrict__ C1, const double* __restrict__ C2,
                         const double* __restrict__ O0, const double* __restrict__ O1, const double* __restrict__ O2,
                         const double* __restrict__ P, double* __restrict__ Pold, R* __restrict__ Vr,
                         R* __restrict__ dVr) {
  double* V[3] = {V0, V1, V2};
  const double* Pr[3] = {P0, P1, P2};
  const double* Co[3] = {C0, C1, C2};
  const double* O[3] = {O0, O1, O2};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const double v = Pr[d][i] + Co[d][i];
      V[d][i] = v;
      Vr[(size_t)d * nv + i] = R(v);
      dVr[(size_t)d * nv + i] = R(v - O[d][i]);
    }
    Pold[i] = P[i];
  }
}

template <int DIM, typename R>
static void finish_impl(Ctx& c) {
  k_finish<DIM, R><<<grid_for(c, c.nv, 256, 8), 256, 0, c.stream>>>(
      c.nv, c.F[PFEM2_FIELD_VX], c.F[PFEM2_FIELD_VY], c.F[PFEM2_FIELD_VZ], c.F[PFEM2_FIELD_PRED_VX],
      c.F[PFEM2_FIELD_PRED_VY], c.F[PFEM2_FIELD_PRED_VZ], c.corr[0], c.corr[1], c.corr[2], c.F[PFEM2_FIELD_OLD_VX],
      c.F[PFEM2_FIELD_OLD_VY], c.F[PFEM2_FIELD_OLD_VZ], c.F[PFEM2_FIELD_P], c.F[PFEM2_FIELD_OLD_P], (R*)c.Vr,
      (R*)c.dVr);
  c.launches++;
}
pfem2_status launch_finish_fem(Ctx& c) {
  if (c.dim == 2) { if (c.pmixed) finish_impl<2, float>(c); else finish_impl<2, double>(c); }
  else { if (c.pmixed) finish_impl<3, float>(c); else finish_impl<3, double>(c); }
  return PFEM2_OK;
}

// particles-only step: V_old = the new projection, V = the frozen field
template <int DIM, typename R>
__global__ void k_restore_frozen(int nv, double* __restrict__ V0, double* __restrict__ V1, double* __restrict__ V2,
                                 double* __restrict__ O0, double* __restrict__ O1, double* __restrict__ O2,
                                 const double* __restrict__ F0, const double* __restrict__ F1,
                                 const double* __restrict__ F2, R* __restrict__ Vr, R* __restrict__ dVr) {
  double* V[3] = {V0, V1, V2};
  double* O[3] = {O0, O1, O2};
  const double* Fz[3] = {F0, F1, F2};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const double proj = V[d][i], fz = Fz[d][i];
      O[d][i] = proj;
      V[d][i] = fz;
      Vr[(size_t)d * nv + i] = R(fz);
      dVr[(size_t)d * nv + i] = R(fz - proj);
    }
  }
}

template <int DIM, typename R>
static void restore_impl(Ctx& c) {
  k_restore_frozen<DIM, R><<<grid_for(c, c.nv, 256, 8), 256, 0, c.stream>>>(
      c.nv, c.F[PFEM2_FIELD_VX], c.F[PFEM2_FIELD_VY], c.F[PFEM2_FIELD_VZ], c.F[PFEM2_FIELD_OLD_VX],
      c.F[PFEM2_FIELD_OLD_VY], c.F[PFEM2_FIELD_OLD_VZ], c.F[PFEM2_FIELD_PRED_VX], c.F[PFEM2_FIELD_PRED_VY],
      c.F[PFEM2_FIELD_PRED_VZ], (R*)c.Vr, (R*)c.dVr);
  c.launches++;
}
pfem2_status launch_restore_frozen(Ctx& c) {
  if (c.dim == 2) { if (c.pmixed) restore_impl<2, float>(c); else restore_impl<2, double>(c); }
  else { if (c.pmixed) restore_impl<3, float>(c); else restore_impl<3, double>(c); }
  return PFEM2_OK;
}

// ---------------------------------------------------------------- loads
// One block over the patch's boundary faces; FP64 face integrals with a
// fixed-order block reduction, so the result is deterministic.
template <int DIM>
__global__ void __launch_bounds__(256) k_loads(const int* __restrict__ faces, int nfaces,
                                               const double* __restrict__ X, const int* __restrict__ cv,
                                               const double* __restrict__ P, const double* __restrict__ Vx,
                                               const double* __restrict__ Vy, double mu, double* __restrict__ out5) {
  constexpr int NV = Dims<DIM>::NV;
  double acc[5] = {0, 0, 0, 0, 0};  // 2D: Fx_nu, Fx_p, Fy_nu, Fy_p ; 3D: Fx, Fy, Fz
  for (int k = threadIdx.x; k < nfaces; k += blockDim.x) {
    const int c = faces[k] / Dims<DIM>::NF, f = faces[k] % Dims<DIM>::NF;
    LocalCell<DIM, double> L;
    double x0[DIM];
    load_local_cell<DIM, double>(X, cv, c, L, x0);
    for (int iq = 0; iq < (DIM == 2 ? 2 : 4); ++iq) {
      double xi[DIM];
      face_qp_xi<DIM, double>(f, iq, xi);
      QP<DIM, double> q;
      eval_qp<DIM, double>(L, xi, face_qp_w<DIM>(), f, q);
      double pq = 0.0, dv = 0.0;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const int g = cv[(size_t)c * NV + v];
        pq += P[g] * q.N[v];
        if (DIM == 2)
          dv += (Vx[g] * q.n[1] - Vy[g] * q.n[0]) * (q.G[v][0] * q.n[0] + q.G[v][1] * q.n[1]);
      }
      if (DIM == 2) {
        acc[0] += mu * dv * q.n[1] * q.JxW;
        acc[1] -= pq * q.n[0] * q.JxW;
        acc[2] -= mu * dv * q.n[0] * q.JxW;
        acc[3] -= pq * q.n[1] * q.JxW;
      } else {
#pragma unroll
        for (int d = 0; d < DIM; ++d) acc[d] += pq * q.n[d] * q.JxW;
      }
    }
  }
  __shared__ double red[5][256];
#pragma unroll
  for (int k = 0; k < 5; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
#pragma unroll
      for (int k = 0; k < 5; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 5; ++k) out5[k] = red[k][0];
}

pfem2_status launch_loads(Ctx& c, int instance, int patch, double* out_dev) {
  const HostInst& in = c.inst[instance];
  const Ctx::LoadFaces* lf = nullptr;
  for (const Ctx::LoadFaces& e : c.load_faces)
    if (e.inst == instance && e.patch == patch) lf = &e;
  if (!lf) {
    // first use: the faces of the instance that carry this boundary id, in
    // cell order (the order of the reference's loop over cells and faces)
    const int NF = c.dim == 2 ? 4 : 6;
    std::vector<int> h;
    for (int k = 0; k < in.nc; ++k)
      for (int f = 0; f < NF; ++f)
        if (in.fb[(size_t)k * NF + f] == patch) h.push_back((in.c_off + k) * NF + f);
    Ctx::LoadFaces e{instance, patch, (int)h.size(), nullptr};
    if (e.n > 0) {
      PFEM2_CUDA(cudaMalloc(&e.d, sizeof(int) * h.size()));
      PFEM2_CUDA(cudaMemcpy(e.d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice));
    }
    c.load_faces.push_back(e);
    lf = &c.load_faces.back();
  }
  if (c.dim == 2)
    k_loads<2><<<1, 256, 0, c.stream>>>(lf->d, lf->n, c.X, c.cv, c.F[PFEM2_FIELD_P], c.F[PFEM2_FIELD_VX],
                                        c.F[PFEM2_FIELD_VY], in.cs.mu, out_dev);
  else
    k_loads<3><<<1, 256, 0, c.stream>>>(lf->d, lf->n, c.X, c.cv, c.F[PFEM2_FIELD_P], c.F[PFEM2_FIELD_VX],
                                        c.F[PFEM2_FIELD_VY], in.cs.mu, out_dev);
  c.launches++;
  return PFEM2_OK;
}

// ---------------------------------------------------------------- vorticity
// calculate_vorticity (cylinderDyM/pfem2particle.cpp:1000-1050), 2D, FP64.
// Node-centric: a thread per vertex walks the cells around it in ascending
// order; per cell it sums N_loc(q) w(q) and N_loc(q) over the QGauss(2)
// points (x fastest), w = sum_i (dN_i/dx Vy_i - dN_i/dy Vx_i), and adds the
// cell sums, as the reference's distribute_local_to_global does; the node
// value is the quotient (0 where the weight is 0).
__global__ void __launch_bounds__(256) k_vorticity(int nv, const int* __restrict__ v2c_ptr,
                                                   const int* __restrict__ v2c_cell,
                                                   const unsigned char* __restrict__ v2c_loc,
                                                   const double* __restrict__ X, const int* __restrict__ cv,
                                                   const double* __restrict__ Vx, const double* __restrict__ Vy,
                                                   double* __restrict__ out) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    double acc = 0.0, wsum = 0.0;
    const int k1 = v2c_ptr[v + 1];
    for (int k = v2c_ptr[v]; k < k1; ++k) {
      const int c = v2c_cell[k], loc = v2c_loc[k];
      LocalCell<2, double> L;
      double x0[2];
      load_local_cell<2, double>(X, cv, c, L, x0);
      double vx[4], vy[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int g = __ldg(cv + (size_t)c * 4 + i);
        vx[i] = Vx[g];
        vy[i] = Vy[g];
      }
      double lv = 0.0, lw = 0.0;
#pragma unroll
      for (int iq = 0; iq < 4; ++iq) {
        double xi[2];
        cell_qp_xi<2, double>(iq, xi);
        QP<2, double> q;
        eval_qp<2, double>(L, xi, cell_qp_w<2>(), -1, q);
        double w = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) w += q.G[i][0] * vy[i] - q.G[i][1] * vx[i];
        lv += q.N[loc] * w;
        lw += q.N[loc];
      }
      acc += lv;
      wsum += lw;
    }
    out[v] = wsum != 0.0 ? acc / wsum : 0.0;
  }
}

pfem2_status launch_vorticity(Ctx& c) {
  k_vorticity<<<grid_for(c, c.nv, 256, 8), 256, 0, c.stream>>>(c.nv, c.v2c_ptr, c.v2c_cell, c.v2c_loc, c.X, c.cv,
                                                              c.F[PFEM2_FIELD_VX], c.F[PFEM2_FIELD_VY],
                                                              c.F[PFEM2_FIELD_VORTICITY]);
  c.launches++;
  return PFEM2_OK;
}

}  // namespace pfem2
