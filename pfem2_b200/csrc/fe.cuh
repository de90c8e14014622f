// fe.cuh -- QGauss(2) element values of the Q1 cells (quadrature points,
// shape values, physical gradients, JxW, face normals), shared by the
// assembly kernels of fem.cu and the moving-mesh kernels of ale.cu.
#pragma once
#include "common.cuh"

namespace pfem2 {

template <int DIM, typename R> struct QP {
  R N[Dims<DIM>::NV];
  R G[Dims<DIM>::NV][DIM];
  R JxW;
  R n[DIM];
};

template <typename R> __device__ __forceinline__ R gauss_pt(int i) {
  return i ? R(0.78867513459481288225) : R(0.21132486540518711775);
}

template <int DIM, typename R>
__device__ __forceinline__ void eval_qp(const LocalCell<DIM, R>& L, const R* xi, R w, int face, QP<DIM, R>& q) {
  constexpr int NV = Dims<DIM>::NV;
  R dN[NV * DIM], J[DIM * DIM], Ji[DIM * DIM];
  shape_values<DIM, R>(xi, q.N);
  shape_grads_ref<DIM, R>(xi, dN);
  local_jacobian<DIM, R>(L, xi, J);
  R det = det_inv<DIM, R>(J, Ji);
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      R s = R(0);
#pragma unroll
      for (int b = 0; b < DIM; ++b) s += dN[v * DIM + b] * Ji[b * DIM + a];
      q.G[v][a] = s;
    }
  if (face < 0) {
    q.JxW = det * w;
  } else {
    const int ax = face >> 1;
    const R sgn = (face & 1) ? R(1) : R(-1);
    R nn = R(0);
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      q.n[a] = Ji[ax * DIM + a] * sgn;
      nn += q.n[a] * q.n[a];
    }
    nn = sqrt(nn);
#pragma unroll
    for (int a = 0; a < DIM; ++a) q.n[a] /= nn;
    q.JxW = det * nn * w;
  }
}

// cell quadrature point iq of QGauss(2)
template <int DIM, typename R>
__device__ __forceinline__ void cell_qp_xi(int iq, R* xi) {
#pragma unroll
  for (int d = 0; d < DIM; ++d) xi[d] = gauss_pt<R>((iq >> d) & 1);
}
template <int DIM> __device__ __forceinline__ double cell_qp_w() { return DIM == 2 ? 0.25 : 0.125; }

// face quadrature point iq on face f
template <int DIM, typename R>
__device__ __forceinline__ void face_qp_xi(int f, int iq, R* xi) {
  const int ax = f >> 1;
  int k = 0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    if (d == ax) xi[d] = R(f & 1);
    else { xi[d] = gauss_pt<R>((iq >> k) & 1); ++k; }
  }
}

}  // namespace pfem2
