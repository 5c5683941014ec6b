// Allocation-free fused heat rollout.
//
// pde_heat_rollout needs a scratch field (the ping-pong buffer of its passes),
// which its callers allocate.  Some callers cannot: code that runs under a
// memory manager owning every device allocation of the process, real-time or
// latency-critical loops where cudaMalloc (which may synchronise the device and
// can fail under memory pressure) is not allowed, and foreign-language hosts
// that can only hand over the field buffers they already hold.  For them,
// pde_heat_rollout_noalloc takes its scratch from a fixed array in device
// memory that belongs to this library.
//
// The array is PDE_NOALLOC_MAX_FLOATS floats (16 MiB); every GPU that loads the
// library holds it until the process exits.  All calls share it: two calls whose
// work overlaps on the GPU (different streams, or threads without ordering)
// race on it and corrupt each other's results, so serialise them.  The array
// keeps the previous call's contents; nothing has to start at zero, because
// every pass of the rollout writes the whole scratch field before any pass
// reads it.
//
// The host side never names the array as a pointer (in host code its name is a
// host-side stand-in, not a device address): once per device, on the first call
// made with that device current, it asks the runtime for the array's device
// address with cudaGetSymbolAddress and keeps it.  Make that first call before
// any stream capture.
#include <cuda_runtime.h>
#include <mutex>

#include "../../include/pde_b200.h"

static __device__ __align__(256) float g_noalloc_scratch[PDE_NOALLOC_MAX_FLOATS];

namespace {

constexpr int kMaxDevices = 64;
float* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of the scratch array for the current device (looked up once).
int scratch_for_current_device(float** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return PDE_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return PDE_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return PDE_ERR_CUDA;
    g_scratch_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_scratch_ptr[dev];
  return PDE_OK;
}

}  // namespace

extern "C" int pde_heat_rollout_noalloc(const float* u_in, float* u_out, const PdeGrid* grid, int32_t ncomp,
                                        const PdeBCRules* rules, float alpha, float dt, int32_t nsteps,
                                        int32_t steps_per_pass, void* stream) {
  if (!u_in || !u_out || !grid || !rules || ncomp < 1) return PDE_ERR_ARG;
  for (int a = 0; a < 3; ++a)
    if (grid->shape[a] < 1) return PDE_ERR_SHAPE;
  const long double floats =
      (long double)grid->shape[0] * (long double)grid->shape[1] * (long double)grid->shape[2] * ncomp;
  if (floats > (long double)PDE_NOALLOC_MAX_FLOATS) return PDE_ERR_TOO_LARGE;
  float* scratch = nullptr;
  const int rc = scratch_for_current_device(&scratch);
  if (rc != PDE_OK) return rc;
  return pde_heat_rollout(u_in, u_out, scratch, grid, ncomp, rules, alpha, dt, nsteps, steps_per_pass, stream);
}
