// project_noalloc.cu -- particle -> grid projection on caller-owned device
// buffers that allocates nothing.
//
// Some callers cannot let a library call cudaMalloc: a host code that owns
// every byte of device memory through its own pool or budget, or code that
// records its work into a CUDA graph, where allocation calls are not
// allowed. For them this entry point keeps its only scratch -- the per-cell
// partial sums of the projection -- in one file-scope device array of fixed
// size, PFEM2_NOALLOC_MAX_CELLS cells (16 MiB), which every GPU that loads
// the library holds until the process exits.
//
// The host code cannot use the array's name as a device address (in host
// code it is a stand-in symbol), so a call on a stream that is not being
// captured, with the device current, looks the address up with
// cudaGetSymbolAddress (again each time, so that a reloaded module after
// cudaDeviceReset is found) and caches it per device; a call made while its
// stream is being captured uses the cached address, so the first call on a
// device must come before any capture. All calls share the array: calls
// that overlap on the GPU (other streams, other threads) race on it and must
// be serialized by the caller. Every scratch entry a call reads has been
// written by the same call (incidences naming a cell outside [0, n_cells)
// are not read: the vertex gets NaN), so no clearing is needed between calls.
#include <mutex>

#include "common.cuh"
#include "ctx.h"

namespace pfem2 {

constexpr int kNoallocK = 32;  // doubles per cell: 2^dim vertices x (dim + 1) sums, 3D = 32

static __device__ __align__(256) double g_noalloc_partial[(size_t)PFEM2_NOALLOC_MAX_CELLS * kNoallocK];

static std::mutex g_noalloc_mu;
static double* g_noalloc_addr[256] = {};

template <int DIM>
__global__ void __launch_bounds__(256) k_noalloc_cells(int nc, const int* __restrict__ cell_start,
                                                       const double* __restrict__ xi, const double* __restrict__ u,
                                                       double* __restrict__ partial) {
  constexpr int NV = Dims<DIM>::NV;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  for (int c = blockIdx.x * wpb + warp; c < nc; c += gridDim.x * wpb) {
    const int b = cell_start[c], n = cell_start[c + 1] - b;
    double acc[NV][DIM + 1];
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int k = 0; k <= DIM; ++k) acc[v][k] = 0.0;
    for (int j = lane; j < n; j += 32) {
      double x[DIM], N[NV];
#pragma unroll
      for (int d = 0; d < DIM; ++d) x[d] = xi[(size_t)(b + j) * DIM + d];
      shape_values<DIM, double>(x, N);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
#pragma unroll
        for (int d = 0; d < DIM; ++d) acc[v][d] += N[v] * u[(size_t)(b + j) * DIM + d];
        acc[v][DIM] += N[v];
      }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int k = 0; k <= DIM; ++k) acc[v][k] = warp_sum(acc[v][k]);
    if (lane == 0)
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int k = 0; k <= DIM; ++k) partial[(size_t)c * kNoallocK + v * (DIM + 1) + k] = acc[v][k];
  }
}

// node sums over the incident cells' partials in incidence order; an
// incidence whose cell or local vertex index is out of range makes the
// vertex NaN instead of reading scratch that this call did not write; a
// vertex flagged in zero_flag (may be null) gets velocity 0, as the wall
// vertices after distribute_particle_velocities_to_grid
// (TurekBenchmarkCuda/pfem2particle.cu:866-869)
template <int DIM>
__global__ void __launch_bounds__(256) k_noalloc_nodes(int nv, int nc, const int* __restrict__ v2c_ptr,
                                                       const int* __restrict__ v2c_cell,
                                                       const int* __restrict__ v2c_local,
                                                       const unsigned char* __restrict__ zero_flag,
                                                       const double* __restrict__ partial,
                                                       double* __restrict__ node_u, double* __restrict__ node_w) {
  constexpr int NV = Dims<DIM>::NV;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    double s[DIM + 1];
#pragma unroll
    for (int k = 0; k <= DIM; ++k) s[k] = 0.0;
    bool bad = false;
    for (int k = v2c_ptr[v]; k < v2c_ptr[v + 1]; ++k) {
      const int c = v2c_cell[k], l = v2c_local[k];
      if (c < 0 || c >= nc || l < 0 || l >= NV) {
        bad = true;
        continue;
      }
      const double* pp = partial + (size_t)c * kNoallocK + l * (DIM + 1);
#pragma unroll
      for (int q = 0; q <= DIM; ++q) s[q] += pp[q];
    }
    const double w = bad ? nan("") : s[DIM];
    const bool zero = zero_flag != nullptr && zero_flag[v] != 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      node_u[(size_t)v * DIM + d] = bad ? w : ((w != 0.0 && !zero) ? s[d] / w : 0.0);
    node_w[v] = w;
  }
}

}  // namespace pfem2

using namespace pfem2;

extern "C" pfem2_status pfem2_project_noalloc(int32_t dim, int32_t n_cells, int32_t n_vertices,
                                              const int32_t* vertex_cell_ptr, const int32_t* vertex_cell,
                                              const int32_t* vertex_cell_local, const int32_t* cell_start,
                                              const double* xi, const double* u, const uint8_t* zero_flag,
                                              double* node_u, double* node_w, void* stream) {
  if (dim != 2 && dim != 3) {
    set_error("pfem2_project_noalloc: dim must be 2 or 3");
    return PFEM2_INVALID_ARG;
  }
  if (n_cells < 0 || n_vertices < 0) {
    set_error("pfem2_project_noalloc: negative size");
    return PFEM2_INVALID_ARG;
  }
  if (n_cells > PFEM2_NOALLOC_MAX_CELLS) {
    set_error("pfem2_project_noalloc: n_cells exceeds PFEM2_NOALLOC_MAX_CELLS (65536); use pfem2_project");
    return PFEM2_INVALID_ARG;
  }
  if (!vertex_cell_ptr || !vertex_cell || !vertex_cell_local || !cell_start || !xi || !u || !node_u || !node_w) {
    set_error("pfem2_project_noalloc: null buffer");
    return PFEM2_INVALID_ARG;
  }
  int dev = 0;
  PFEM2_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) {
    set_error("pfem2_project_noalloc: device ordinal out of range");
    return PFEM2_INVALID_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  PFEM2_CUDA(cudaStreamIsCapturing(st, &cap));
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (cap == cudaStreamCaptureStatusNone) {
      void* p = nullptr;
      PFEM2_CUDA(cudaGetSymbolAddress(&p, g_noalloc_partial));
      g_noalloc_addr[dev] = (double*)p;
    } else if (!g_noalloc_addr[dev]) {
      set_error("pfem2_project_noalloc: the first call on a device must come before any stream capture");
      return PFEM2_BAD_STATE;
    }
    scratch = g_noalloc_addr[dev];
  }
  if (n_cells == 0 && n_vertices == 0) return PFEM2_OK;
  const int cgrid = (int)std::min<long long>(((long long)n_cells * 32 + 255) / 256, 148LL * 16);
  const int vgrid = (int)std::min<long long>(((long long)n_vertices + 255) / 256, 148LL * 16);
  if (dim == 2) {
    if (n_cells) k_noalloc_cells<2><<<cgrid, 256, 0, st>>>(n_cells, cell_start, xi, u, scratch);
    if (n_vertices)
      k_noalloc_nodes<2><<<vgrid, 256, 0, st>>>(n_vertices, n_cells, vertex_cell_ptr, vertex_cell, vertex_cell_local,
                                               zero_flag, scratch, node_u, node_w);
  } else {
    if (n_cells) k_noalloc_cells<3><<<cgrid, 256, 0, st>>>(n_cells, cell_start, xi, u, scratch);
    if (n_vertices)
      k_noalloc_nodes<3><<<vgrid, 256, 0, st>>>(n_vertices, n_cells, vertex_cell_ptr, vertex_cell, vertex_cell_local,
                                               zero_flag, scratch, node_u, node_w);
  }
  PFEM2_CUDA(cudaGetLastError());
  return PFEM2_OK;
}
