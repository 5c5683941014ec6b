// Element-wise and absorbing-layer operators of the weakly compressible / ACM
// path: OuterProduct and scalarVectorMult (FDM/module/elementWiseOps.py:10-88),
// FarField (FDM/module/farfield.py, kernel FDM/kernel/farfield.py:50-77) and
// ViscousDampingLayer (FDM/module/viscousDampingLayer.py, kernel
// FDM/kernel/viscousDampingLayer.py:50-76).
//
// All are HBM streams with one rounding per operation, as the reference's
// kernels: M[i][j] = A[i] * B[j]; a[0] * b; and on the layer points
// out = -(scale * profile) * (u - u_far)  or  -(scale * profile) * du_dt.
// The layer's points and per-point profile (dx / L) ** exponent are set up once
// by the caller; a call reads each point's field value and writes its output.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace {

using namespace pde;

constexpr int kMaxCond = 16;  // far-field value: a vector or matrix of up to 16 floats
struct Cond {
  float v[kMaxCond];
};

__global__ void __launch_bounds__(256) outer_kernel(const float* __restrict__ a, const float* __restrict__ b,
                                                    float* __restrict__ out, int64_t total, int na, int nb) {
  const int nab = na * nb;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e / nab;
    const int r = (int)(e - c * nab);
    const int i = r / nb, j = r - i * nb;
    out[e] = mul(a[c * na + i], b[c * nb + j]);
  }
}

__global__ void __launch_bounds__(256) scalar_mult_kernel(const float* __restrict__ s, const float* __restrict__ b,
                                                          float* __restrict__ out, int64_t total, int nb) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    out[e] = mul(s[e / nb], b[e]);
}

template <bool FAR>
__global__ void __launch_bounds__(256) layer_kernel(const float* __restrict__ in, float* __restrict__ out, int ncomp,
                                                    const int64_t* __restrict__ cells,
                                                    const float* __restrict__ profile, int64_t total, float scale,
                                                    const Cond cond) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = e / ncomp;
    const int k = (int)(e - p * ncomp);
    const float damp = mul(scale, profile[p]);
    const int64_t i = cells[p] * ncomp + k;
    out[i] = FAR ? mul(-damp, sub(in[i], cond.v[k])) : mul(-damp, in[i]);
  }
}

}  // namespace

extern "C" {

int pde_outer(const float* a, const float* b, float* out, int64_t cells, int32_t na, int32_t nb, void* stream) {
  if (!a || !b || !out || cells < 0 || na < 1 || nb < 1) return PDE_ERR_ARG;
  const int64_t total = cells * na * nb;
  if (total == 0) return PDE_OK;
  outer_kernel<<<grid_blocks(total, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a, b, out, total, na, nb);
  return cudaGetLastError() == cudaSuccess ? PDE_OK : PDE_ERR_CUDA;
}

int pde_scalar_mult(const float* s, const float* b, float* out, int64_t cells, int32_t nb, void* stream) {
  if (!s || !b || !out || cells < 0 || nb < 1) return PDE_ERR_ARG;
  const int64_t total = cells * nb;
  if (total == 0) return PDE_OK;
  scalar_mult_kernel<<<grid_blocks(total, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(s, b, out, total,
                                                                                                   nb);
  return cudaGetLastError() == cudaSuccess ? PDE_OK : PDE_ERR_CUDA;
}

int pde_layer_apply(const float* in, float* out, int32_t ncomp, const int64_t* cells, const float* profile,
                    int64_t npoints, float scale, const float* cond_host, void* stream) {
  if (!in || !out || ncomp < 1 || npoints < 0 || (npoints > 0 && (!cells || !profile))) return PDE_ERR_ARG;
  if (cond_host && ncomp > kMaxCond) return PDE_ERR_ARG;
  Cond c{};
  if (cond_host)
    for (int k = 0; k < ncomp; ++k) c.v[k] = cond_host[k];
  const int64_t total = npoints * ncomp;
  if (total == 0) return PDE_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (cond_host)
    layer_kernel<true><<<grid_blocks(total, 256), 256, 0, st>>>(in, out, ncomp, cells, profile, total, scale, c);
  else
    layer_kernel<false><<<grid_blocks(total, 256), 256, 0, st>>>(in, out, ncomp, cells, profile, total, scale, c);
  return cudaGetLastError() == cudaSuccess ? PDE_OK : PDE_ERR_CUDA;
}

}  // extern "C"
