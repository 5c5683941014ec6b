// Host side of the 3D streaming heat rollout (heat3d.cuh): launch shape,
// X chunking and the dispatch over stencil radius, pass depth and component
// count.  Its own translation unit, so the kernel instantiations compile in
// parallel with the rest of the library.
#include <cuda_runtime.h>

#include "common.cuh"
#include "heat3d.cuh"

namespace pde {
namespace {

// Launch shape set by pde_set_launch_3d: tile sides (at most the compiled
// maxima) and the number of X chunks; 0 = each one chosen here.
int g_launch3d[3] = {0, 0, 0};

template <int R, int K, int N, int TYM, int TZM, int T>
int launch_heat3d_k(const float* src, float* dst, const Geo& G, const Weights& W, float alpha, float dt,
                    const PdeBCRules* rules, double t0, double tstep, int n0, cudaStream_t st) {
  using Cf = H3Cfg<R, K, N, TYM, TZM, T>;
  auto kern = heat3d_kernel<R, K, N, TYM, TZM, T>;
  static int occ = -1;
  if (occ < 0) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cf::SMEM) != cudaSuccess)
      return PDE_ERR_CUDA;
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, T, Cf::SMEM) != cudaSuccess || o < 1)
      return PDE_ERR_CUDA;
    occ = o;
  }
  H3Params P;
  P.X = (int)G.n[0]; P.Y = (int)G.n[1]; P.Z = (int)G.n[2]; P.g = G.g;
  const int ty = (g_launch3d[0] > 0 && g_launch3d[0] < TYM) ? g_launch3d[0] : TYM;
  const int tz = (g_launch3d[1] > 0 && g_launch3d[1] < TZM) ? g_launch3d[1] : TZM;
  P.ny_t = (P.Y + ty - 1) / ty;
  P.nz_t = (P.Z + tz - 1) / tz;
  P.ntiles = P.ny_t * P.nz_t;
  // X chunks (balanced, each at least min_chunk planes, which the ghost planes
  // at either end of X need).  The kernel is bound by instruction issue and
  // the items are dealt evenly, so the time is about the total planes streamed
  // (each item streams 2H extra) over the SMs, plus one item of granularity.
  const int H = Cf::H;
  const long long sms = sm_count();
  const long long slots = (long long)occ * sms;
  const int min_chunk = 2 * H + G.g + 8;
  const int max_n = P.X / min_chunk > 1 ? (P.X / min_chunk < 64 ? P.X / min_chunk : 64) : 1;
  int best_n = 1;
  if (g_launch3d[2] > 0) {
    best_n = g_launch3d[2] < max_n ? g_launch3d[2] : max_n;
  } else {
    double best = 1e300;
    for (int n = 1; n <= max_n; ++n) {
      const double per_item = (double)P.X / n + 2 * H;
      const double cost = (double)P.ntiles * n * per_item / (double)sms + per_item;
      if (cost < best - 1e-9) { best = cost; best_n = n; }
    }
  }
  P.nch = best_n;
  P.nitems = P.ntiles * P.nch;
  for (int t = 0; t < 5; ++t) P.w[t] = W.w[t];
  P.alpha = alpha; P.dt = dt;
  P.negzero = -0.0f;
  P.t0 = t0; P.tstep = tstep; P.n0 = n0;
  const long long blocks = slots < P.nitems ? slots : P.nitems;
  return launch_pdl(kern, (int)blocks, T, Cf::SMEM, st, src, dst, P, *rules);
}

}  // namespace

// Deepest temporal block of the 3D kernels per component count.
int heat3d_kmax(int ncomp) { return ncomp == 1 ? 4 : 2; }

int launch_heat3d(int ks, int R, int N, const float* src, float* dst, const Geo& G, const Weights& W, float alpha,
                  float dt, const PdeBCRules* rules, double t0, double tstep, int n0, cudaStream_t st) {
#define PDE_H3(RR, KK, NN, TY, TZ, TT) \
  return launch_heat3d_k<RR, KK, NN, TY, TZ, TT>(src, dst, G, W, alpha, dt, rules, t0, tstep, n0, st)
  // tile shapes: the region (tile + 2H per axis, rows rounded to 8, row pitch
  // to 8 floats) fills whole warp tiles of T/32 warps; registers bound T * C
  if (N == 1) {
    if (R == 1) {
      switch (ks) {
        case 1: PDE_H3(1, 1, 1, 44, 26, 256);
        case 2: PDE_H3(1, 2, 1, 42, 24, 256);
        case 3: PDE_H3(1, 3, 1, 40, 22, 384);
        default: PDE_H3(1, 4, 1, 38, 28, 480);
      }
    }
    switch (ks) {
      case 1: PDE_H3(2, 1, 1, 42, 24, 256);
      case 2: PDE_H3(2, 2, 1, 38, 28, 480);
      case 3: PDE_H3(2, 3, 1, 18, 16, 512);
      default: PDE_H3(2, 4, 1, 14, 12, 512);
    }
  }
  if (N == 2) {
    if (R == 1) { if (ks == 1) PDE_H3(1, 1, 2, 44, 11, 256); PDE_H3(1, 2, 2, 42, 9, 256); }
    if (ks == 1) PDE_H3(2, 1, 2, 42, 9, 256);
    PDE_H3(2, 2, 2, 38, 9, 480);
  }
  if (N == 3) {
    if (R == 1) { if (ks == 1) PDE_H3(1, 1, 3, 44, 6, 256); PDE_H3(1, 2, 3, 42, 6, 480); }
    if (ks == 1) PDE_H3(2, 1, 3, 42, 6, 480);
    PDE_H3(2, 2, 3, 38, 5, 384);
  }
  if (R == 1) { if (ks == 1) PDE_H3(1, 1, 4, 44, 3, 256); PDE_H3(1, 2, 4, 42, 3, 480); }
  if (ks == 1) PDE_H3(2, 1, 4, 42, 3, 480);
  PDE_H3(2, 2, 4, 38, 3, 448);
#undef PDE_H3
}

}  // namespace pde

extern "C" int pde_set_launch_3d(int32_t tile_y, int32_t tile_z, int32_t chunks) {
  if (tile_y < 0 || tile_z < 0 || chunks < 0 || chunks > 4096) return PDE_ERR_ARG;
  pde::g_launch3d[0] = tile_y;
  pde::g_launch3d[1] = tile_z;
  pde::g_launch3d[2] = chunks;
  return PDE_OK;
}
