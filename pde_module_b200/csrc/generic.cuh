// General-shape kernels: any eligible-axis pattern, any component count,
// order 2 or 4.  One thread per output float, grid-stride loops, coalesced
// along the contiguous component/Z direction.  They are the operators of
// record for 2D grids and odd shapes; 3D scalar/vector sweeps go through the
// TMA-staged streaming kernels (stream3d.cuh).
#pragma once
#include "common.cuh"

namespace pde {

// Device-side error word: set by bounds checks and bounded waits, read and
// cleared by pde_device_error().  Never traps.
__device__ int g_err = 0;

__device__ __forceinline__ void flag_error(int code) { atomicCAS(&g_err, 0, code); }

// Interior-cell decode: t -> flat cell index of the t-th interior cell
// (Z fastest), i.e. wp.tid() + dims_shift of FDM/kernel/laplacian.py:53-56.
__device__ __forceinline__ int64_t interior_cell(const Geo& G, int64_t t) {
  int64_t k = t % G.ext[2];
  int64_t r = t / G.ext[2];
  int64_t j = r % G.ext[1];
  int64_t i = r / G.ext[1];
  return (i + G.lo[0]) * G.cstride[0] + (j + G.lo[1]) * G.cstride[1] + (k + G.lo[2]);
}

// Laplacian, FDM/kernel/laplacian.py:34-59: acc = 0; for axis: for tap:
// acc += w[tap]*u[c + shift*e_axis]; out = alpha*acc.
template <int R>
__global__ void __launch_bounds__(256) lap_generic_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                          Geo G, int N, Weights W, float alpha, int64_t total) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t cell = t / N;
    int n = (int)(t - cell * N);
    int64_t c = interior_cell(G, cell);
    const float* p = in + c * N + n;
    float acc = 0.0f;
    for (int d = 0; d < G.ndims; ++d) {
      int64_t s = G.cstride[G.dims[d]] * N;
#pragma unroll
      for (int tap = 0; tap < 2 * R + 1; ++tap) acc = add(acc, mul(W.w[tap], __ldg(p + (tap - R) * s)));
    }
    out[c * N + n] = mul(alpha, acc);
  }
}

// Grad, FDM/kernel/grad.py:78-100: out[n][a] accumulates its own taps.
// The output column is the position of the axis among the eligible axes
// (the reference indexes by axis number, which coincides whenever the
// eligible axes are leading, the only layouts on which it is well defined).
template <int R>
__global__ void __launch_bounds__(256) grad_generic_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                           Geo G, int N, Weights W, float alpha, int64_t total) {
  const int D = G.ndims;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t q = t / D;
    int d = (int)(t - q * D);
    int64_t cell = q / N;
    int n = (int)(q - cell * N);
    int64_t c = interior_cell(G, cell);
    const float* p = in + c * N + n;
    int64_t s = G.cstride[G.dims[d]] * N;
    float acc = 0.0f;
#pragma unroll
    for (int tap = 0; tap < 2 * R + 1; ++tap) acc = add(acc, mul(W.w[tap], __ldg(p + (tap - R) * s)));
    out[(c * N + n) * D + d] = mul(alpha, acc);
  }
}

// Divergence, FDM/kernel/divergence.py:85-106: out[n] = alpha * sum over
// eligible axes (ascending) and taps of w*in[...][n][a].
template <int R>
__global__ void __launch_bounds__(256) div_generic_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                          Geo G, int N, Weights W, float alpha, int64_t total) {
  const int D = G.ndims;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t cell = t / N;
    int n = (int)(t - cell * N);
    int64_t c = interior_cell(G, cell);
    float acc = 0.0f;
    for (int d = 0; d < D; ++d) {
      int64_t s = G.cstride[G.dims[d]] * N * D;
      const float* p = in + (c * N + n) * D + d;
#pragma unroll
      for (int tap = 0; tap < 2 * R + 1; ++tap) acc = add(acc, mul(W.w[tap], __ldg(p + (tap - R) * s)));
    }
    out[c * N + n] = mul(alpha, acc);
  }
}

// Forward Euler, time_step/forwardEuler.py:70-79, 16-byte vectors.
__global__ void __launch_bounds__(256) euler_vec4_kernel(const float4* __restrict__ y, const float4* __restrict__ k,
                                                         float dt, float4* __restrict__ o, int64_t n4) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
    float4 a = y[i], b = k[i], r;
    r.x = add(a.x, mul(dt, b.x));
    r.y = add(a.y, mul(dt, b.y));
    r.z = add(a.z, mul(dt, b.z));
    r.w = add(a.w, mul(dt, b.w));
    o[i] = r;
  }
}

__global__ void euler_scalar_kernel(const float* __restrict__ y, const float* __restrict__ k, float dt,
                                    float* __restrict__ o, int64_t begin, int64_t n) {
  for (int64_t i = begin + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    o[i] = add(y[i], mul(dt, k[i]));
}

// Boundary value of one group at time t (boundary_functions.py:32-45, 77-92).
__device__ __forceinline__ float bc_value(int func, float value, float t_max, const float* t_dev) {
  if (func == PDE_BC_FUNC_RAMP) {
    float t = t_dev ? *t_dev : 0.0f;
    float ramp = fminf(__fdiv_rn(t, t_max), 1.0f);
    return mul(ramp, value);
  }
  return value;
}

// One boundary group, functional_boundary.py:357-400.  Reads only `in`
// (the pre-boundary field); `out` already holds the copy of `in`.
__global__ void bc_group_kernel(const float* __restrict__ in, float* __restrict__ out, Geo G, int N,
                                const int32_t* __restrict__ ids, int count, int type, uint32_t mask,
                                int func, float value, float t_max, const float* t_dev, float dx32) {
  int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= count) return;
  int64_t id = ids[tid];
  int64_t total = G.n[0] * G.n[1] * G.n[2];
  if (id < 0 || id >= total) { flag_error(PDE_ERR_SHAPE); return; }
  int64_t ijk[3];
  ijk[0] = id / (G.n[1] * G.n[2]);       // global_to_ijk_c, utils/warp_utils.py:17-30
  ijk[1] = (id / G.n[2]) % G.n[1];
  ijk[2] = id % G.n[2];
  const float v = bc_value(func, value, t_max, t_dev);
  if (type == PDE_BC_DIRICHLET) {
    for (int n = 0; n < N; ++n) out[id * N + n] = ((mask >> n) & 1u) ? v : in[id * N + n];
  }
  for (int d = 0; d < G.ndims; ++d) {
    int a = G.dims[d];
    int inc = 0;
    if (ijk[a] == G.g) inc = 1;                       // get_interior_vec, :343-352
    else if (ijk[a] == G.n[a] - 1 - G.g) inc = -1;
    if (inc == 0) continue;
    int64_t gidx = ijk[a] - inc, aidx = ijk[a] + inc;
    if (gidx < 0 || gidx >= G.n[a] || aidx < 0 || aidx >= G.n[a]) { flag_error(PDE_ERR_GHOST); continue; }
    int64_t ghost = id - inc * G.cstride[a];
    int64_t adj = id + inc * G.cstride[a];
    for (int n = 0; n < N; ++n) {
      if (!((mask >> n) & 1u)) continue;
      float cur = in[adj * N + n];
      float nv;
      if (type == PDE_BC_DIRICHLET) nv = sub(mul(2.0f, v), cur);
      else nv = add(mul(mul((float)(-2 * inc), dx32), v), cur);
      out[ghost * N + n] = nv;
    }
  }
}

// Periodic ghost fill along axis a (in place), over the full extent of the
// other axes.  Thread per (ghost-slab cell, component).
__global__ void periodic_axis_kernel(float* __restrict__ u, Geo G, int N, int a, int64_t total) {
  const int64_t g = G.g, na = G.n[a], M = na - 2 * g;
  // slab extents: along a there are 2g ghost indices, others are full.
  int64_t e[3] = {G.n[0], G.n[1], G.n[2]};
  e[a] = 2 * g;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t cell = t / N;
    int n = (int)(t - cell * N);
    int64_t c2 = cell % e[2], r = cell / e[2];
    int64_t c1 = r % e[1], c0 = r / e[1];
    int64_t ijk[3] = {c0, c1, c2};
    int64_t s = ijk[a];
    int64_t idx = s < g ? s : (na - 2 * g + s);  // ghost index in [0,g) or [n-g, n)
    int64_t src = g + (((idx - g) % M) + M) % M;
    ijk[a] = idx;
    int64_t dst_c = ijk[0] * G.cstride[0] + ijk[1] * G.cstride[1] + ijk[2];
    ijk[a] = src;
    int64_t src_c = ijk[0] * G.cstride[0] + ijk[1] * G.cstride[1] + ijk[2];
    u[dst_c * N + n] = u[src_c * N + n];
  }
}

}  // namespace pde
