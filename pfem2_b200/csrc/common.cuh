// common.cuh -- device helpers shared by the PFEM2 kernels (sm_100a).
//
// Q1 / Q1-hex shape functions, the multilinear cell map and its Newton
// inverse in a cell-local frame, the counter-based SplitMix64 stream, the
// bounded grid barrier and small warp utilities.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define PFEM2_FULL_MASK 0xffffffffu

namespace pfem2 {

template <int DIM> struct Dims {
  static constexpr int NV = 1 << DIM;  // vertices per cell
  static constexpr int NF = 2 * DIM;   // faces per cell
};

// FE_Q(1) shape values in deal.II lexicographic order:
// N_v(xi) = prod_d (bit_d(v) ? xi_d : 1 - xi_d)
template <int DIM, typename R>
__device__ __forceinline__ void shape_values(const R* xi, R* N) {
#pragma unroll
  for (int v = 0; v < Dims<DIM>::NV; ++v) {
    R s = R(1);
#pragma unroll
    for (int d = 0; d < DIM; ++d) s *= ((v >> d) & 1) ? xi[d] : (R(1) - xi[d]);
    N[v] = s;
  }
}

template <int DIM, typename R>
__device__ __forceinline__ void shape_grads_ref(const R* xi, R* dN) {
#pragma unroll
  for (int v = 0; v < Dims<DIM>::NV; ++v)
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      R s = ((v >> d) & 1) ? R(1) : R(-1);
#pragma unroll
      for (int e = 0; e < DIM; ++e)
        if (e != d) s *= ((v >> e) & 1) ? xi[e] : (R(1) - xi[e]);
      dN[v * DIM + d] = s;
    }
}

template <int DIM, typename R>
__device__ __forceinline__ R det_inv(const R* J, R* Ji) {
  if constexpr (DIM == 2) {
    R det = J[0] * J[3] - J[1] * J[2];
    R id = R(1) / det;
    Ji[0] = J[3] * id; Ji[1] = -J[1] * id;
    Ji[2] = -J[2] * id; Ji[3] = J[0] * id;
    return det;
  } else {
    R a = J[0], b = J[1], c = J[2], d = J[3], e = J[4], f = J[5], g = J[6], h = J[7], i = J[8];
    R A = e * i - f * h, B = -(d * i - f * g), Cc = d * h - e * g;
    R det = a * A + b * B + c * Cc;
    R id = R(1) / det;
    Ji[0] = A * id; Ji[1] = -(b * i - c * h) * id; Ji[2] = (b * f - c * e) * id;
    Ji[3] = B * id; Ji[4] = (a * i - c * g) * id;  Ji[5] = -(a * f - c * d) * id;
    Ji[6] = Cc * id; Ji[7] = -(a * h - b * g) * id; Ji[8] = (a * e - b * d) * id;
    return det;
  }
}

// Cell geometry in the cell-local frame: D[v][a] = X_v - X_0 (D[0] = 0).
template <int DIM, typename R> struct LocalCell {
  R D[Dims<DIM>::NV][DIM];
};

template <int DIM, typename R>
__device__ __forceinline__ void load_local_cell(const double* __restrict__ X, const int* __restrict__ cv, int c,
                                                LocalCell<DIM, R>& L, double* x0) {
  constexpr int NV = Dims<DIM>::NV;
  int g0 = __ldg(cv + (size_t)c * NV);
#pragma unroll
  for (int a = 0; a < DIM; ++a) x0[a] = __ldg(X + (size_t)g0 * DIM + a);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    int g = __ldg(cv + (size_t)c * NV + v);
#pragma unroll
    for (int a = 0; a < DIM; ++a) L.D[v][a] = R(__ldg(X + (size_t)g * DIM + a) - x0[a]);
  }
}

// local position F(xi) - X_0 = sum_v N_v D_v
template <int DIM, typename R>
__device__ __forceinline__ void local_map(const LocalCell<DIM, R>& L, const R* xi, R* x) {
  R N[Dims<DIM>::NV];
  shape_values<DIM, R>(xi, N);
#pragma unroll
  for (int a = 0; a < DIM; ++a) x[a] = R(0);
#pragma unroll
  for (int v = 1; v < Dims<DIM>::NV; ++v)
#pragma unroll
    for (int a = 0; a < DIM; ++a) x[a] += N[v] * L.D[v][a];
}

template <int DIM, typename R>
__device__ __forceinline__ void local_jacobian(const LocalCell<DIM, R>& L, const R* xi, R* J) {
  R dN[Dims<DIM>::NV * DIM];
  shape_grads_ref<DIM, R>(xi, dN);
#pragma unroll
  for (int k = 0; k < DIM * DIM; ++k) J[k] = R(0);
#pragma unroll
  for (int v = 1; v < Dims<DIM>::NV; ++v)
#pragma unroll
    for (int a = 0; a < DIM; ++a)
#pragma unroll
      for (int b = 0; b < DIM; ++b) J[a * DIM + b] += L.D[v][a] * dN[v * DIM + b];
}

// Per-cell geometry record of the particle kernels: origin X_0 (FP64),
// vertex offsets D_v = X_v - X_0 (v >= 1) and the inverse Jacobian at the
// cell centre in the arithmetic type, and whether the map is affine (then
// xi = Ji (x - X_0) exactly and no Newton iteration is needed).
template <int DIM, typename R> struct __align__(16) CellGeo {
  double x0[DIM];
  R D[Dims<DIM>::NV - 1][DIM];
  R Ji[DIM * DIM];
  int affine;
};

template <int DIM, typename R>
__device__ __forceinline__ void geo_to_local(const CellGeo<DIM, R>& g, LocalCell<DIM, R>& L, double* x0) {
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    x0[a] = g.x0[a];
    L.D[0][a] = R(0);
  }
#pragma unroll
  for (int v = 1; v < Dims<DIM>::NV; ++v)
#pragma unroll
    for (int a = 0; a < DIM; ++a) L.D[v][a] = g.D[v - 1][a];
}

template <typename R> struct NewtonTol;
template <> struct NewtonTol<double> {
  static constexpr double step = 1e-12;
  static constexpr int iters = 30;
};
template <> struct NewtonTol<float> {
  static constexpr float step = 2e-6f;
  static constexpr int iters = 12;
};

// Inverse of the multilinear map (MappingQ1::transform_real_to_unit_cell)
// for a point given in the cell-local frame. Returns false when Newton fails
// (the reference treats that as "not in this cell").
template <int DIM, typename R>
__device__ __forceinline__ bool local_inverse(const LocalCell<DIM, R>& L, const R* x, R* xi) {
#pragma unroll
  for (int d = 0; d < DIM; ++d) xi[d] = R(0.5);
  for (int it = 0; it < NewtonTol<R>::iters; ++it) {
    R F[DIM], J[DIM * DIM], Ji[DIM * DIM];
    local_map<DIM, R>(L, xi, F);
    local_jacobian<DIM, R>(L, xi, J);
    R det = det_inv<DIM, R>(J, Ji);
    if (!(det > R(0))) return false;
    R mx = R(0);
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      R s = R(0);
#pragma unroll
      for (int b = 0; b < DIM; ++b) s += Ji[a * DIM + b] * (F[b] - x[b]);
      xi[a] -= s;
      mx = fmax(mx, fabs(s));
    }
#pragma unroll
    for (int a = 0; a < DIM; ++a)
      if (!(fabs(xi[a]) < R(1e6))) return false;
    if (mx < NewtonTol<R>::step) return true;
  }
  return false;
}

// Inverse map with the cell record: direct for affine cells, otherwise
// Newton started from the linearisation at the cell centre.
template <int DIM, typename R>
__device__ __forceinline__ bool geo_inverse(const CellGeo<DIM, R>& g, const LocalCell<DIM, R>& L, const R* x,
                                            R* xi) {
  if (g.affine) {
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      R s = R(0);
#pragma unroll
      for (int b = 0; b < DIM; ++b) s += g.Ji[a * DIM + b] * x[b];
      xi[a] = s;
    }
    return true;
  }
  R c[DIM];
  R half[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) half[d] = R(0.5);
  local_map<DIM, R>(L, half, c);
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    R s = R(0.5);
#pragma unroll
    for (int b = 0; b < DIM; ++b) s += g.Ji[a * DIM + b] * (x[b] - c[b]);
    xi[a] = s;
  }
  for (int it = 0; it < NewtonTol<R>::iters; ++it) {
    R F[DIM], J[DIM * DIM], Ji[DIM * DIM];
    local_map<DIM, R>(L, xi, F);
    local_jacobian<DIM, R>(L, xi, J);
    R det = det_inv<DIM, R>(J, Ji);
    if (!(det > R(0))) return false;
    R mx = R(0);
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      R s = R(0);
#pragma unroll
      for (int b = 0; b < DIM; ++b) s += Ji[a * DIM + b] * (F[b] - x[b]);
      xi[a] -= s;
      mx = fmax(mx, fabs(s));
    }
#pragma unroll
    for (int a = 0; a < DIM; ++a)
      if (!(fabs(xi[a]) < R(1e6))) return false;
    if (mx < NewtonTol<R>::step) return true;
  }
  return false;
}

template <int DIM, typename R>
__device__ __forceinline__ bool inside_unit(const R* xi) {
  bool ok = true;
#pragma unroll
  for (int d = 0; d < DIM; ++d) ok = ok && (xi[d] >= R(0) && xi[d] <= R(1));
  return ok;
}

// Counter-based SplitMix64 stream (identical to the oracle's).
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ double uniform01(uint64_t seed, uint64_t ordinal, int axis) {
  uint64_t key = seed * 0xD1B54A32D192ED03ULL + ordinal * 4ULL + (uint64_t)axis;
  return (double)(splitmix64(key) >> 11) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Bounded software grid barrier for cooperative (co-resident) grids.
// Every wait is capped; on timeout the barrier sets *err and returns false,
// and callers leave their loops so the kernel always terminates.
struct GridBarrier {
  unsigned* count;
  unsigned* gen;
  int* err;
  unsigned spin_limit;  // polls before a wait gives up and sets *err = 1
};

// polls before a wait gives up (the default; contexts may lower it)
#define PFEM2_BARRIER_SPIN_LIMIT (1u << 26)

// Release/acquire grid barrier on an arrival counter that is never reset
// within a launch: barrier k is passed once the counter reaches
// gridDim.x * k. Thread 0 arrives with a gpu-scope release add and polls
// with gpu-scope acquire loads (no separate fences); the CTA barriers on
// both sides extend the ordering to the other threads of the block. `k`
// is the caller's barrier count (0 after the reset that precedes every
// launch). The poll gives up after gb.spin_limit tries or when
// another block has flagged an error, sets gb.err = 1 and returns false.
__device__ __forceinline__ bool grid_sync_ra(const GridBarrier& gb, unsigned& k) {
  __syncthreads();
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    ++k;
    const unsigned target = gridDim.x * k;
    unsigned v;
    asm volatile("atom.add.release.gpu.u32 %0, [%1], 1;" : "=r"(v) : "l"(gb.count) : "memory");
    int ok = 1;
    unsigned spins = 0;
    while (true) {
      asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(gb.count) : "memory");
      if ((int)(v - target) >= 0) break;
      if (++spins > gb.spin_limit || *(volatile int*)gb.err) {
        atomicExch(gb.err, 1);
        ok = 0;
        break;
      }
      __nanosleep(20);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ void red_release_add_u32(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(PFEM2_FULL_MASK, v, o);
  return v;
}

}  // namespace pfem2
