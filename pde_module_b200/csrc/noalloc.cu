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
// host-side stand-in, not a device address): the first call made in a CUDA
// context (normally the device's primary context) asks the runtime for the
// array's device address with cudaGetSymbolAddress and keeps it, keyed by that
// context's unique id, so a context created later (another context, or the
// primary context again after cudaDeviceReset) looks the address up anew.
// Make the first call in a context before any stream capture.
#include <cuda.h>
#include <cuda_runtime.h>
#include <mutex>

#include "../../include/pde_b200.h"

static __device__ __align__(256) float g_noalloc_scratch[PDE_NOALLOC_MAX_FLOATS];

namespace {

// Driver entry points (resolved through the runtime: no link-time libcuda).
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

struct ScratchEntry {
  unsigned long long ctx_id;
  float* ptr;
};
constexpr int kMaxContexts = 64;
ScratchEntry g_scratch[kMaxContexts] = {};
int g_scratch_next = 0;
std::mutex g_scratch_mu;

// Unique id of the current context (0: unknown, the address is then looked up on every call).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    cudaDriverEntryPointQueryResult q1, q2;
    void* f1 = nullptr;
    void* f2 = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
      get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
      get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    resolved = true;
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the scratch array in the current context (looked up once per context).
int scratch_for_current_context(float** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return PDE_ERR_CUDA;  // makes the device's context current
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const unsigned long long id = current_context_id();
  if (id != 0)
    for (const ScratchEntry& e : g_scratch)
      if (e.ctx_id == id) {
        *out = e.ptr;
        return PDE_OK;
      }
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return PDE_ERR_CUDA;
  if (id != 0) {
    g_scratch[g_scratch_next] = ScratchEntry{id, static_cast<float*>(p)};
    g_scratch_next = (g_scratch_next + 1) % kMaxContexts;
  }
  *out = static_cast<float*>(p);
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
  const int rc = scratch_for_current_context(&scratch);
  if (rc != PDE_OK) return rc;
  return pde_heat_rollout(u_in, u_out, scratch, grid, ncomp, rules, alpha, dt, nsteps, steps_per_pass, stream);
}
