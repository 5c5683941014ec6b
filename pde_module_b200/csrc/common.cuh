// Shared helpers for the sm_100a kernels of the finite-difference hot path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

#include "../../include/pde_b200.h"

namespace pde {

// 4-byte asynchronous global -> shared copy (cp.async); src-size 0 writes a
// zero instead of reading.  A thread's copies are all in flight at once, so a
// region load costs one memory latency, not one per cell it copies.
__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
// Asynchronous 8-byte global -> shared copy (both addresses 8-byte aligned).
__device__ __forceinline__ void cp_async8(float* dst, const float* src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}
// Wait for this thread's cp.async copies (the block still needs a barrier before others read them).
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start while the previous kernel of its stream runs.
// pdl_launch_dependents lets the next kernel be scheduled (it still waits);
// pdl_wait blocks until the previous kernel has completed and its writes are
// visible: every global access to data another launch reads or writes comes
// after it.  Both are no-ops for kernels launched without the attribute.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// Walk of a row-major (rows x W) rectangle by a block: cell c = tid, tid + nt, ...
// as (row, col), advanced without division.
struct RectWalk {
  int row, col, dq, dr, W;
  __device__ RectWalk(int W_, int nt) : W(max(W_, 1)) {
    dq = nt / W;
    dr = nt - dq * W;
    row = (int)threadIdx.x / W;
    col = (int)threadIdx.x - row * W;
  }
  __device__ void next() {
    row += dq;
    col += dr;
    if (col >= W) { col -= W; ++row; }
  }
};



// Geometry of one (X, Y, Z, N...) array, derived from PdeGrid.
struct Geo {
  int64_t n[3];        // array extents including ghosts
  int64_t lo[3];       // first interior index per axis (g on eligible axes, else 0)
  int64_t ext[3];      // interior extent per axis (n - 2g on eligible axes, else n)
  int64_t cstride[3];  // cell strides: Y*Z, Z, 1
  int ndims;           // number of eligible axes
  int dims[3];         // eligible axes, ascending
  int g;
  int order;
};

// Stencil weights rounded to fp32, largest stencil is 5 taps.
struct Weights {
  float w[5];
  double wd[5];  // the same weights before rounding to fp32
  int taps;  // 3 or 5
  int radius;
};

inline bool make_geo(const PdeGrid* grid, Geo* geo) {
  if (!grid) return false;
  if (grid->order != 2 && grid->order != 4) return false;
  if (grid->ghost_cells < 0) return false;
  geo->g = grid->ghost_cells;
  geo->order = grid->order;
  geo->ndims = 0;
  for (int a = 0; a < 3; ++a) {
    if (grid->shape[a] < 1) return false;
    geo->n[a] = grid->shape[a];
  }
  geo->cstride[2] = 1;
  geo->cstride[1] = geo->n[2];
  geo->cstride[0] = geo->n[1] * geo->n[2];
  for (int a = 0; a < 3; ++a) {
    if (geo->n[a] > 1) {
      geo->dims[geo->ndims++] = a;
      geo->lo[a] = geo->g;
      geo->ext[a] = geo->n[a] - 2 * (int64_t)geo->g;
      if (geo->ext[a] < 1) return false;
    } else {
      geo->lo[a] = 0;
      geo->ext[a] = geo->n[a];
    }
  }
  for (int k = geo->ndims; k < 3; ++k) geo->dims[k] = -1;
  return geo->ndims >= 1;
}

// Laplacian weights: order 2 (1,-2,1)/dx^2 (FDM/module/laplacian.py:33-35);
// order 4 (-1,16,-30,16,-1)/(12 dx^2).  Formed in double, rounded to fp32.
inline Weights lap_weights(int order, double dx) {
  Weights W{};
  if (order == 2) {
    double d2 = dx * dx;
    W.taps = 3; W.radius = 1;
    W.wd[0] = 1.0 / d2; W.wd[1] = -2.0 / d2; W.wd[2] = 1.0 / d2;
  } else {
    double d = 12.0 * dx * dx;
    W.taps = 5; W.radius = 2;
    W.wd[0] = -1.0 / d; W.wd[1] = 16.0 / d; W.wd[2] = -30.0 / d; W.wd[3] = 16.0 / d; W.wd[4] = -1.0 / d;
  }
  for (int t = 0; t < W.taps; ++t) W.w[t] = (float)W.wd[t];
  return W;
}

// First-derivative weights: order 2 (-1,0,1)/(2dx) (FDM/module/grad.py:37-39,
// divergence.py:37-39); order 4 (1,-8,0,8,-1)/(12 dx).
inline Weights d1_weights(int order, double dx) {
  Weights W{};
  if (order == 2) {
    W.taps = 3; W.radius = 1;
    W.wd[0] = -1.0 / (2 * dx); W.wd[1] = 0.0; W.wd[2] = 1.0 / (2 * dx);
  } else {
    double d = 12.0 * dx;
    W.taps = 5; W.radius = 2;
    W.wd[0] = 1.0 / d; W.wd[1] = -8.0 / d; W.wd[2] = 0.0; W.wd[3] = 8.0 / d; W.wd[4] = -1.0 / d;
  }
  for (int t = 0; t < W.taps; ++t) W.w[t] = (float)W.wd[t];
  return W;
}

// Correctly rounded fp32 operations that the compiler may not contract into FMA:
// every product and every sum of the reference is rounded on its own.
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }

// Packed pairs of fp32 (sm_100 f32x2 arithmetic): each lane is one IEEE
// round-to-nearest operation, exactly like the scalar mul/add above.
typedef unsigned long long f2;
__device__ __forceinline__ f2 pack2(float a, float b) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void unpack2(f2 r, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  f2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// Boundary time of rollout step n: t0 + n * tstep in double, each operation
// rounded on its own (as a host caller computes t0 + n*dt), then rounded to fp32.
__device__ __forceinline__ float step_time(double t0, double tstep, int n) {
  return __double2float_rn(__dadd_rn(t0, __dmul_rn((double)n, tstep)));
}

// Compile-time loop: f(std::integral_constant<int, I>) for I = I0 .. N-1.
template <int I, int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    static_for<I + 1, N>(f);
  }
}

// SMs of the current device (looked up once per process).
inline int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
  }
  return n;
}

// Launch with programmatic stream serialization: the kernel may be scheduled
// while the previous kernel of the stream runs; it calls pdl_wait before any
// global access to data another launch reads or writes.
template <typename... KArgs, typename... Args>
int launch_pdl(void (*kern)(KArgs...), int grid, int block, size_t smem, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, args...) == cudaSuccess ? PDE_OK : PDE_ERR_CUDA;
}

inline int grid_blocks(int64_t work, int threads, int64_t cap = 148LL * 64) {
  int64_t b = (work + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

}  // namespace pde

#define PDE_CUDA_CHECK(expr)                    \
  do {                                          \
    cudaError_t _e = (expr);                    \
    if (_e != cudaSuccess) return PDE_ERR_CUDA; \
  } while (0)
