// C-ABI entry points of the finite-difference hot path (include/pde_b200.h).
// One translation unit: every kernel header is included here so the library
// has a single device-side error word.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include "common.cuh"
#include "generic.cuh"
#include "stream3d.cuh"
#include "fused.cuh"
#include "ldc.cuh"
#include "wc.cuh"
#include "wave.cuh"
#include "batched.cuh"
#include "heat_adj.cuh"

using namespace pde;

namespace {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }


int launch_status() { return cudaGetLastError() == cudaSuccess ? PDE_OK : PDE_ERR_CUDA; }

// Launch shape of the temporally blocked 2D kernels set by pde_set_launch_2d
// (tile sides, threads per block); 0 = each entry point's own choice.
int g_tile2d[2] = {0, 0};
// Bound of every device-side wait (pde_set_wait_limit_ns).
uint64_t g_wait_ns = PDE_WAIT_LIMIT_DEFAULT_NS;
int g_threads2d = 0;

// A 2D tile count just above m x SMs (m = 1, 2) leaves a short tail wave in which
// a few SMs run a second tile while the rest wait: enlarge the tiles slightly
// (at most two fewer tiles per axis, sides up to 256) so the count drops to m x SMs.

void balance_tiles(int X, int Y, int* tbx, int* tby) {
  const long long sms = sm_count();
  const long long nx = (X + *tbx - 1) / *tbx, ny = (Y + *tby - 1) / *tby;
  for (long long m = 1; m <= 2; ++m) {
    const long long cap = m * sms;
    if (nx * ny <= cap) return;
    if (nx * ny * 4 > cap * 5) continue;
    long long bx = 0, by = 0;
    for (long long ax = nx - 2; ax <= nx; ++ax)
      for (long long ay = ny - 2; ay <= ny; ++ay)
        if (ax >= 1 && ay >= 1 && ax * ay <= cap && ax * ay > bx * by) {
          bx = ax;
          by = ay;
        }
    if (bx == 0) return;
    const int tx = (int)((X + bx - 1) / bx), ty = (int)((Y + by - 1) / by);
    if (tx > 256 || ty > 256) return;
    *tbx = tx;
    *tby = ty;
    return;
  }
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// ---- 3D streaming dispatch -------------------------------------------------
template <int R, int OP, int CIN, int TZ, int TY, int YPT, int PREF, int MAPK, int MODE>
int launch_stream3d_k(const float* in, float* out, const Geo& G, const Weights& Wt, double alpha_d, float alpha,
                      cudaStream_t st, float dt = 0.0f) {
  using C = S3Cfg<R, OP, CIN, TZ, TY, YPT, PREF, MAPK, MODE>;
  auto kern = stream3d_kernel<R, OP, CIN, TZ, TY, YPT, PREF, MAPK, MODE>;
  static int occ = -1;
  if (occ < 0) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM) != cudaSuccess)
      return PDE_ERR_CUDA;
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, C::THREADS, C::SMEM) != cudaSuccess || o < 1)
      return PDE_ERR_CUDA;
    occ = o;
  }
  const int64_t total = G.n[0] * G.n[1] * G.n[2] * CIN;
  S3Params P;
  P.X = (int)G.n[0]; P.Y = (int)G.n[1]; P.Z = (int)G.n[2]; P.g = G.g;
  P.ny_tiles = (int)((G.ext[1] + TY - 1) / TY);
  P.nz_tiles = (int)((G.ext[2] + TZ - 1) / TZ);
  P.pp = (int)((G.n[1] * G.n[2] * CIN) & 3);
  P.pr = (int)((G.n[2] * CIN) & 3);
  for (int t = 0; t < 5; ++t) P.w[t] = Wt.w[t];
  P.alpha = alpha;
  P.dt = dt;
  P.out = out;
  P.wait_ns = g_wait_ns;
  P.negzero = -0.0f;
  // Persistent grid over (chunk, tile) items in chunk-major order.  The chunk
  // count is chosen by a load model: the busiest SM runs ceil(blocks/SMs)
  // blocks of ceil(items/blocks) items each, against the ideal items/SMs, and
  // each item re-reads 2R planes at its ends; weighted by the share of resident
  // block slots the grid fills (a streaming block alone on an SM keeps too few
  // loads in flight: 384^3 with half the slots ran at 52% of DRAM bandwidth).
  P.ntiles = P.ny_tiles * P.nz_tiles;
  const int nx = (int)G.ext[0];
  const int sms = sm_count();
  const long long slots = (long long)occ * sms;
  int best_n = 1;
  double best = -1.0;
  for (int n = 1; n <= 64 && n <= nx; ++n) {
    const int ch = (nx + n - 1) / n;
    const int nn = (nx + ch - 1) / ch;
    const long long items = (long long)P.ntiles * nn;
    const long long B = items < slots ? items : slots;
    const long long per_block = (items + B - 1) / B;
    const long long per_sm = (B + sms - 1) / sms;
    const double eff =
        ((double)items / sms) / (double)(per_block * per_sm) * (double)ch / (ch + R) * ((double)B / (double)slots);
    if (eff > best + 1e-9) { best = eff; best_n = n; }
  }
  P.chunk = (nx + best_n - 1) / best_n;
  const int nchunks = (nx + P.chunk - 1) / P.chunk;
  P.nitems = P.ntiles * nchunks;
  long long blocks = slots < P.nitems ? slots : P.nitems;
  CUtensorMap m;
  if (MAPK == MAP_PAIRS) {
    const uint64_t zc = (uint64_t)G.n[2] * CIN;
    if (!encode_3d(&m, in, 2 * zc, (uint64_t)G.n[1] / 2, (uint64_t)G.n[0], 8 * zc, 4 * zc * (uint64_t)G.n[1],
                   (uint32_t)C::W, (uint32_t)(C::ROWS / 2)))
      return PDE_ERR_CUDA;
  } else if (!encode_1d(&m, in, (uint64_t)total, (uint32_t)C::W)) {
    return PDE_ERR_CUDA;
  }
  FastW FW{};
  if (MODE == MODE_FAST) {
    // folded weights from the double-precision stencil (Weights::wd)
    if (OP == OP_LAP) {
      for (int t = 0; t < R; ++t) FW.a[t] = (float)(alpha_d * Wt.wd[t]);
      FW.a[R] = (float)(alpha_d * 3.0 * Wt.wd[R]);
    } else {
      for (int t = R + 1; t < 2 * R + 1; ++t) FW.a[t - R - 1] = (float)(alpha_d * Wt.wd[t]);
    }
  }
  kern<<<(unsigned)blocks, C::THREADS, C::SMEM, st>>>(m, P, FW);
  return launch_status();
}

// Plane addressing for a grid: double-row boxes when the array's row pairs and
// planes have 16-byte multiple pitches and the tile rows start on even rows;
// else one copy per row (lead fixed across planes when the plane pitch is a
// multiple of 4 floats).
template <int CIN>
int pick_map(const Geo& G, int R) {
  const int64_t zc = G.n[2] * CIN;
  if ((G.n[1] % 2) == 0 && (zc % 2) == 0 && ((G.n[1] * zc) % 4) == 0 && ((G.g - R) % 2) == 0 &&
      G.n[1] / 2 < (1LL << 31) && 2 * zc < (1LL << 31))
    return MAP_PAIRS;
  return ((G.n[1] * zc) & 3) == 0 ? MAP_ROWS_PP0 : MAP_ROWS_GEN;
}

template <int R, int OP, int CIN, int TZ, int TY, int YPT, int PREF>
int launch_stream3d(const float* in, float* out, const Geo& G, const Weights& Wt, float alpha, int mode,
                    cudaStream_t st) {
  const int map = pick_map<CIN>(G, R);
  if (mode == PDE_MODE_FAST) {
    if (map == MAP_PAIRS)
      return launch_stream3d_k<R, OP, CIN, TZ, TY, YPT, PREF, MAP_PAIRS, MODE_FAST>(in, out, G, Wt, alpha, alpha, st);
    if (map == MAP_ROWS_PP0)
      return launch_stream3d_k<R, OP, CIN, TZ, TY, YPT, PREF, MAP_ROWS_PP0, MODE_FAST>(in, out, G, Wt, alpha, alpha, st);
    return launch_stream3d_k<R, OP, CIN, TZ, TY, YPT, PREF, MAP_ROWS_GEN, MODE_FAST>(in, out, G, Wt, alpha, alpha, st);
  }
  if (map == MAP_PAIRS)
    return launch_stream3d_k<R, OP, CIN, TZ, TY, YPT, PREF, MAP_PAIRS, MODE_EXACT>(in, out, G, Wt, alpha, alpha, st);
  if (map == MAP_ROWS_PP0)
    return launch_stream3d_k<R, OP, CIN, TZ, TY, YPT, PREF, MAP_ROWS_PP0, MODE_EXACT>(in, out, G, Wt, alpha, alpha, st);
  return launch_stream3d_k<R, OP, CIN, TZ, TY, YPT, PREF, MAP_ROWS_GEN, MODE_EXACT>(in, out, G, Wt, alpha, alpha, st);
}

// Tile configurations of the streaming kernels.  Candidate 0 is the default
// for every shape and mode; candidates 1-3 are compiled for double-row
// addressing (even Y and Z), exact arithmetic, and are picked per
// (operator, order) by pde_stream3d_select (the autotuner sweeps them).  The
// scalar Laplacian and the Grad at order 4 run z-pair consumers (two cells per
// lane), so their tiles hold twice the z cells per lane of the others.
enum { S3K_LAP1 = 0, S3K_LAP3 = 1, S3K_GRAD = 2, S3K_DIV = 3, S3K_KINDS = 4 };
// Defaults [kind][order 2, order 4]: the fastest candidates of a sweep at 512^3 on B200.
int g_s3_sel[S3K_KINDS][2] = {{2, 1}, {3, 3}, {1, 1}, {1, 1}};
constexpr int kS3Candidates = 4;

template <int R, int OP, int CIN>
int launch_candidate(int cand, const float* in, float* out, const Geo& G, const Weights& W, float alpha,
                     cudaStream_t st) {
  if constexpr (OP == OP_LAP && CIN == 1 && R == 2) {  // z-pair consumers (TZ/2 lanes per row group)
    switch (cand) {
      case 1: return launch_stream3d_k<R, OP, 1, 128, 16, 4, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      case 2: return launch_stream3d_k<R, OP, 1, 64, 32, 4, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      case 3: return launch_stream3d_k<R, OP, 1, 128, 8, 2, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      default: return launch_stream3d_k<R, OP, 1, 64, 32, 8, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
    }
  } else if constexpr (OP == OP_LAP && CIN == 1) {
    switch (cand) {
      case 1: return launch_stream3d_k<R, OP, 1, 64, 16, 4, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      case 2: return launch_stream3d_k<R, OP, 1, 128, 16, 8, 3, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      case 3: return launch_stream3d_k<R, OP, 1, 128, 8, 4, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      default: return launch_stream3d_k<R, OP, 1, 64, 32, 8, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
    }
  } else if constexpr (OP == OP_LAP) {
    switch (cand) {
      case 1: return launch_stream3d_k<R, OP, 3, 32, 16, 4, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      case 2: return launch_stream3d_k<R, OP, 3, 64, 8, 8, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      default: return launch_stream3d_k<R, OP, 3, 32, 32, 8, 2, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
    }
  } else if constexpr (OP == OP_GRAD && R == 2) {  // z-pair consumers
    switch (cand) {
      case 1: return launch_stream3d_k<R, OP, 1, 128, 8, 2, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      case 2: return launch_stream3d_k<R, OP, 1, 64, 16, 2, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      case 3: return launch_stream3d_k<R, OP, 1, 128, 8, 4, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      default: return launch_stream3d_k<R, OP, 1, 128, 8, 2, 6, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
    }
  } else if constexpr (OP == OP_GRAD) {
    switch (cand) {
      case 1: return launch_stream3d_k<R, OP, 1, 128, 16, 4, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      case 2: return launch_stream3d_k<R, OP, 1, 128, 8, 4, 6, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      case 3: return launch_stream3d_k<R, OP, 1, 128, 8, 4, 4, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      default: return launch_stream3d_k<R, OP, 1, 64, 16, 4, 6, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
    }
  } else {
    switch (cand) {
      case 1: return launch_stream3d_k<R, OP, 3, 64, 16, 4, 2, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      case 2: return launch_stream3d_k<R, OP, 3, 32, 16, 8, 3, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
      default: return launch_stream3d_k<R, OP, 3, 64, 32, 8, 1, MAP_PAIRS, MODE_EXACT>(in, out, G, W, alpha, alpha, st);
    }
  }
}

// Launch the selected candidate when it applies, else the default configuration.
template <int R, int OP, int CIN, int TZ, int TY, int YPT, int PREF>
int launch_selected(int kind, const float* in, float* out, const Geo& G, const Weights& W, float alpha, int mode,
                    cudaStream_t st) {
  const int cand = g_s3_sel[kind][R - 1];
  if (cand > 0 && mode == PDE_MODE_EXACT && pick_map<CIN>(G, R) == MAP_PAIRS)
    return launch_candidate<R, OP, CIN>(cand, in, out, G, W, alpha, st);
  return launch_stream3d<R, OP, CIN, TZ, TY, YPT, PREF>(in, out, G, W, alpha, mode, st);
}

// The flat 1D TMA view addresses floats with int32 coordinates, including rows
// up to one tile past the last interior row.
int g_dispatch = PDE_DISPATCH_AUTO;

bool stream3d_ok(const float* in, const Geo& G, int cin) {
  if (g_dispatch == PDE_DISPATCH_GENERIC) return false;
  if (G.ndims != 3) return false;
  if (!aligned16(in)) return false;
  const int64_t total = G.n[0] * G.n[1] * G.n[2] * cin;
  const int64_t slack = 64LL * G.n[2] * cin + 1024;
  return total + slack < (1LL << 31) && G.g >= G.order / 2;
}

int check_common(const void* in, const void* out, const PdeGrid* grid, int ncomp, Geo* G) {
  if (!in || !out || !grid) return PDE_ERR_ARG;
  if (ncomp < 1) return PDE_ERR_ARG;
  if (!make_geo(grid, G)) return PDE_ERR_SHAPE;
  if (G->g < G->order / 2) return PDE_ERR_GHOST;
  if (in == out) return PDE_ERR_ARG;
  return PDE_OK;
}

}  // namespace

extern "C" {

int pde_version(void) { return 100; }

int pde_stream3d_select(int32_t op, int32_t order, int32_t ncomp_in, int32_t candidate) {
  int kind;
  if (op == PDE_OP_LAPLACIAN && ncomp_in == 1) kind = S3K_LAP1;
  else if (op == PDE_OP_LAPLACIAN && ncomp_in == 3) kind = S3K_LAP3;
  else if (op == PDE_OP_GRAD && ncomp_in == 1) kind = S3K_GRAD;
  else if (op == PDE_OP_DIVERGENCE && ncomp_in == 3) kind = S3K_DIV;
  else return PDE_ERR_UNSUPPORTED;
  if (order != 2 && order != 4) return PDE_ERR_ARG;
  if (candidate < -1 || candidate >= kS3Candidates) return PDE_ERR_ARG;
  int& slot = g_s3_sel[kind][order / 2 - 1];
  const int prev = slot;
  if (candidate >= 0) slot = candidate;
  return prev;
}

int pde_set_dispatch(int mode) {
  const int prev = g_dispatch;
  if (mode == PDE_DISPATCH_AUTO || mode == PDE_DISPATCH_GENERIC) g_dispatch = mode;
  return prev;
}

const char* pde_strerror(int s) {
  switch (s) {
    case PDE_OK: return "ok";
    case PDE_ERR_ARG: return "invalid argument";
    case PDE_ERR_SHAPE: return "shape inconsistent with the operator";
    case PDE_ERR_GHOST: return "ghost width smaller than the stencil radius";
    case PDE_ERR_ALIGN: return "pointer alignment requirement not met";
    case PDE_ERR_CUDA: return "CUDA runtime call failed";
    case PDE_ERR_UNSUPPORTED: return "not supported by this build";
    case PDE_ERR_TIMEOUT: return "a bounded device wait gave up";
    case PDE_ERR_TOO_LARGE: return "size above the documented maximum";
    default: return "unknown status";
  }
}

uint64_t pde_set_wait_limit_ns(uint64_t ns) {
  const uint64_t prev = g_wait_ns;
  g_wait_ns = ns > 0 ? ns : PDE_WAIT_LIMIT_DEFAULT_NS;
  return prev;
}

int pde_wait_probe(const uint32_t* word, uint32_t target, void* stream) {
  if (!word) return PDE_ERR_ARG;
  wait_probe_kernel<<<1, 32, 0, as_stream(stream)>>>(word, target, g_wait_ns);
  return launch_status();
}

int pde_device_error(void* stream) {
  if (cudaStreamSynchronize(as_stream(stream)) != cudaSuccess) return PDE_ERR_CUDA;
  int v = 0, z = 0;
  if (cudaMemcpyFromSymbol(&v, g_err, sizeof(int)) != cudaSuccess) return PDE_ERR_CUDA;
  if (cudaMemcpyToSymbol(g_err, &z, sizeof(int)) != cudaSuccess) return PDE_ERR_CUDA;
  return v;
}

int pde_laplacian(const float* in, float* out, const PdeGrid* grid, int32_t ncomp, float alpha, void* stream) {
  return pde_laplacian_ex(in, out, grid, ncomp, alpha, PDE_MODE_EXACT, stream);
}

int pde_laplacian_ex(const float* in, float* out, const PdeGrid* grid, int32_t ncomp, float alpha, int32_t mode,
                     void* stream) {
  if (mode != PDE_MODE_EXACT && mode != PDE_MODE_FAST) return PDE_ERR_ARG;
  Geo G;
  int rc = check_common(in, out, grid, ncomp, &G);
  if (rc) return rc;
  const Weights W = lap_weights(G.order, grid->dx);
  cudaStream_t st = as_stream(stream);
  if ((ncomp == 1 || ncomp == 3) && stream3d_ok(in, G, ncomp)) {
    if (G.order == 2) {
      if (ncomp == 1) return launch_selected<1, OP_LAP, 1, 64, 32, 8, 4>(S3K_LAP1, in, out, G, W, alpha, mode, st);
      return launch_selected<1, OP_LAP, 3, 32, 16, 8, 4>(S3K_LAP3, in, out, G, W, alpha, mode, st);
    } else {
      if (ncomp == 1) return launch_selected<2, OP_LAP, 1, 64, 32, 8, 4>(S3K_LAP1, in, out, G, W, alpha, mode, st);
      return launch_selected<2, OP_LAP, 3, 32, 16, 8, 4>(S3K_LAP3, in, out, G, W, alpha, mode, st);
    }
  }
  const int64_t total = G.ext[0] * G.ext[1] * G.ext[2] * ncomp;
  const int blocks = grid_blocks(total, 256);
  if (G.order == 2) lap_generic_kernel<1><<<blocks, 256, 0, st>>>(in, out, G, ncomp, W, alpha, total);
  else lap_generic_kernel<2><<<blocks, 256, 0, st>>>(in, out, G, ncomp, W, alpha, total);
  return launch_status();
}

int pde_grad(const float* in, float* out, const PdeGrid* grid, int32_t ncomp, float alpha, void* stream) {
  return pde_grad_ex(in, out, grid, ncomp, alpha, PDE_MODE_EXACT, stream);
}

int pde_grad_ex(const float* in, float* out, const PdeGrid* grid, int32_t ncomp, float alpha, int32_t mode,
                void* stream) {
  if (mode != PDE_MODE_EXACT && mode != PDE_MODE_FAST) return PDE_ERR_ARG;
  Geo G;
  int rc = check_common(in, out, grid, ncomp, &G);
  if (rc) return rc;
  const Weights W = d1_weights(G.order, grid->dx);
  cudaStream_t st = as_stream(stream);
  if (ncomp == 1 && stream3d_ok(in, G, 1)) {
    // default tile (fast mode, and shapes without the double-row map): 128 x 8, 4 rows per thread
    if (G.order == 2) return launch_selected<1, OP_GRAD, 1, 128, 8, 4, 4>(S3K_GRAD, in, out, G, W, alpha, mode, st);
    return launch_selected<2, OP_GRAD, 1, 128, 8, 4, 4>(S3K_GRAD, in, out, G, W, alpha, mode, st);
  }
  const int64_t total = G.ext[0] * G.ext[1] * G.ext[2] * ncomp * G.ndims;
  const int blocks = grid_blocks(total, 256);
  if (G.order == 2) grad_generic_kernel<1><<<blocks, 256, 0, st>>>(in, out, G, ncomp, W, alpha, total);
  else grad_generic_kernel<2><<<blocks, 256, 0, st>>>(in, out, G, ncomp, W, alpha, total);
  return launch_status();
}

int pde_divergence(const float* in, float* out, const PdeGrid* grid, int32_t nrows, float alpha, void* stream) {
  return pde_divergence_ex(in, out, grid, nrows, alpha, PDE_MODE_EXACT, stream);
}

int pde_divergence_ex(const float* in, float* out, const PdeGrid* grid, int32_t nrows, float alpha, int32_t mode,
                      void* stream) {
  if (mode != PDE_MODE_EXACT && mode != PDE_MODE_FAST) return PDE_ERR_ARG;
  Geo G;
  int rc = check_common(in, out, grid, nrows, &G);
  if (rc) return rc;
  const Weights W = d1_weights(G.order, grid->dx);
  cudaStream_t st = as_stream(stream);
  if (nrows == 1 && stream3d_ok(in, G, 3)) {
    if (G.order == 2) return launch_selected<1, OP_DIV, 3, 64, 16, 8, 2>(S3K_DIV, in, out, G, W, alpha, mode, st);
    return launch_selected<2, OP_DIV, 3, 64, 16, 8, 2>(S3K_DIV, in, out, G, W, alpha, mode, st);
  }
  const int64_t total = G.ext[0] * G.ext[1] * G.ext[2] * nrows;
  const int blocks = grid_blocks(total, 256);
  if (G.order == 2) div_generic_kernel<1><<<blocks, 256, 0, st>>>(in, out, G, nrows, W, alpha, total);
  else div_generic_kernel<2><<<blocks, 256, 0, st>>>(in, out, G, nrows, W, alpha, total);
  return launch_status();
}

int pde_euler(const float* y, const float* k, float dt, float* out, int64_t count, void* stream) {
  if (!y || !k || !out || count < 0) return PDE_ERR_ARG;
  if (count == 0) return PDE_OK;
  cudaStream_t st = as_stream(stream);
  int64_t n4 = 0;
  if (aligned16(y) && aligned16(k) && aligned16(out)) {
    n4 = count / 4;
    if (n4 > 0)
      euler_vec4_kernel<<<grid_blocks(n4, 256), 256, 0, st>>>(reinterpret_cast<const float4*>(y),
                                                               reinterpret_cast<const float4*>(k), dt,
                                                               reinterpret_cast<float4*>(out), n4);
  }
  if (4 * n4 < count)
    euler_scalar_kernel<<<grid_blocks(count - 4 * n4, 256), 256, 0, st>>>(y, k, dt, out, 4 * n4, count);
  return launch_status();
}

int pde_bc_apply(const float* in, float* out, const PdeGrid* grid, int32_t ncomp, const PdeBCGroup* groups,
                 int32_t ngroups, const float* t_device, void* stream) {
  if (!in || !out || !grid || ncomp < 1 || ncomp > 32 || ngroups < 0 || (ngroups > 0 && !groups))
    return PDE_ERR_ARG;
  Geo G;
  if (!make_geo(grid, &G)) return PDE_ERR_SHAPE;
  cudaStream_t st = as_stream(stream);
  const size_t bytes = (size_t)(G.n[0] * G.n[1] * G.n[2]) * ncomp * sizeof(float);
  if (in != out) PDE_CUDA_CHECK(cudaMemcpyAsync(out, in, bytes, cudaMemcpyDeviceToDevice, st));
  const float dx32 = (float)grid->dx;
  for (int i = 0; i < ngroups; ++i) {
    const PdeBCGroup& B = groups[i];
    if (B.type != PDE_BC_DIRICHLET && B.type != PDE_BC_VON_NEUMANN) return PDE_ERR_ARG;
    if (B.func != PDE_BC_FUNC_CONSTANT && B.func != PDE_BC_FUNC_RAMP) return PDE_ERR_ARG;
    if (B.func == PDE_BC_FUNC_RAMP && !t_device) return PDE_ERR_ARG;
    if (B.count < 0 || (B.count > 0 && !B.node_ids)) return PDE_ERR_ARG;
    if (ncomp < 32 && (B.comp_mask >> ncomp) != 0) return PDE_ERR_ARG;
    if (B.count == 0) continue;
    bc_group_kernel<<<(B.count + 127) / 128, 128, 0, st>>>(in, out, G, ncomp, B.node_ids, B.count, B.type,
                                                           B.comp_mask, B.func, B.value, B.t_max, t_device, dx32);
  }
  return launch_status();
}

int pde_periodic_fill(float* u, const PdeGrid* grid, int32_t ncomp, int32_t axis_mask, void* stream) {
  if (!u || !grid || ncomp < 1) return PDE_ERR_ARG;
  Geo G;
  if (!make_geo(grid, &G)) return PDE_ERR_SHAPE;
  if (G.g < 1) return PDE_ERR_GHOST;
  cudaStream_t st = as_stream(stream);
  for (int a = 0; a < 3; ++a) {
    if (!((axis_mask >> a) & 1)) continue;
    if (G.n[a] == 1) return PDE_ERR_ARG;
    int64_t e[3] = {G.n[0], G.n[1], G.n[2]};
    e[a] = 2 * G.g;
    const int64_t total = e[0] * e[1] * e[2] * ncomp;
    periodic_axis_kernel<<<grid_blocks(total, 256), 256, 0, st>>>(u, G, ncomp, a, total);
  }
  return launch_status();
}

int pde_bc_compile(const PdeBCGroup* groups, int32_t ngroups, const PdeGrid* grid, int32_t ncomp,
                   PdeBCRules* rules) {
  if (!grid || !rules || ngroups < 0 || (ngroups > 0 && !groups)) return PDE_ERR_ARG;
  if (ngroups > PDE_MAX_GROUPS) return PDE_ERR_TOO_LARGE;
  if (ncomp < 1 || ncomp > PDE_FUSED_MAX_COMP) return PDE_ERR_UNSUPPORTED;
  Geo G;
  if (!make_geo(grid, &G)) return PDE_ERR_SHAPE;
  if (G.g < 1) return PDE_ERR_GHOST;
  memset(rules, 0, sizeof(*rules));
  rules->ncomp = ncomp;
  rules->ngroups = ngroups;
  rules->dx32 = (float)grid->dx;
  int elig_faces = 0;
  for (int a = 0; a < 3; ++a)
    if (G.n[a] > 1) elig_faces |= 3 << (2 * a);
  for (int i = 0; i < ngroups; ++i) {
    const PdeBCGroup& B = groups[i];
    if (B.face_mask == 0) return PDE_ERR_UNSUPPORTED;
    if (B.face_mask & ~elig_faces) return PDE_ERR_ARG;
    if (B.type != PDE_BC_DIRICHLET && B.type != PDE_BC_VON_NEUMANN) return PDE_ERR_ARG;
    if (B.func != PDE_BC_FUNC_CONSTANT && B.func != PDE_BC_FUNC_RAMP) return PDE_ERR_ARG;
    if ((B.comp_mask >> ncomp) != 0) return PDE_ERR_ARG;
    if (B.func == PDE_BC_FUNC_RAMP) rules->has_ramp = 1;
    rules->group[i].type = B.type;
    rules->group[i].comp_mask = B.comp_mask;
    rules->group[i].func = B.func;
    rules->group[i].value = B.value;
    rules->group[i].t_max = B.t_max;
  }
  for (int K = 0; K < 27; ++K) {
    const int k[3] = {K / 9, (K / 3) % 3, K % 3};
    int faces = 0;
    bool valid = true;
    for (int a = 0; a < 3; ++a) {
      if (G.n[a] == 1) {
        if (k[a] != 1) valid = false;
        continue;
      }
      if (k[a] == 0) faces |= 1 << (2 * a);
      if (k[a] == 2) faces |= 1 << (2 * a + 1);
    }
    rules->node_group[K] = -1;
    for (int a = 0; a < 3; ++a)
      for (int v = 0; v < PDE_FUSED_MAX_COMP; ++v) rules->ghost_group[K][a][v] = -1;
    if (!valid || faces == 0) continue;
    for (int i = 0; i < ngroups; ++i) {
      const PdeBCGroup& B = groups[i];
      if (!(B.face_mask & faces)) continue;  // node not in this group
      if (B.type == PDE_BC_DIRICHLET) rules->node_group[K] = (int8_t)i;
      for (int a = 0; a < 3; ++a) {
        if (G.n[a] == 1 || k[a] == 1) continue;  // no ghost along this axis
        for (int v = 0; v < ncomp; ++v)
          if ((B.comp_mask >> v) & 1u) rules->ghost_group[K][a][v] = (int8_t)i;
      }
    }
  }
  return PDE_OK;
}

// 3D streaming heat rollout (heat3d.cu)
extern "C++" {
namespace pde {
int heat3d_kmax(int ncomp);
int launch_heat3d(int ks, int R, int N, const float* src, float* dst, const Geo& G, const Weights& W, float alpha,
                  float dt, const PdeBCRules* rules, double t0, double tstep, int n0, cudaStream_t st);
}  // namespace pde
}

namespace {

// The streaming kernel takes 3D grids whose interior has at least 3 cells per
// axis, and whose planes index in 32 bits.
bool heat3d_ok(const Geo& G, int ncomp) {
  if (g_dispatch == PDE_DISPATCH_GENERIC) return false;
  if (G.ndims != 3 || ncomp < 1 || ncomp > 4) return false;
  for (int a = 0; a < 3; ++a)
    if (G.ext[a] < 3) return false;
  return G.n[1] * G.n[2] * ncomp < (1LL << 31);
}

// Host copy of generic.cuh bc_value for a ramp group at rollout step n: the
// same float operations (t / t_max rounded, min with 1, times the value).
float host_ramp_value(const PdeBCGroupParam& B, double t0, double tstep, long long n) {
  const double td = (double)n * tstep;
  const float t = (float)(t0 + td);
  const float q = t / B.t_max;
  const float r = q < 1.0f ? q : 1.0f;
  return r * B.value;
}

// One step per pass on the TMA streaming kernel (OP_HEAT) after a surface fill:
// scalar 3D fields whose shape takes the double-row map (even Y and Z, 16-byte
// plane pitch, even g - R) and whose index fits the 1D view.
bool heat_split_shape(const Geo& G, int ncomp) {
  if (g_dispatch == PDE_DISPATCH_GENERIC || G.ndims != 3 || ncomp != 1) return false;
  const int R = G.order / 2;
  const int64_t slack = 64LL * G.n[2] + 1024;
  return pick_map<1>(G, R) == MAP_PAIRS && G.n[0] * G.n[1] * G.n[2] + slack < (1LL << 31) && G.g >= R &&
         G.ext[0] >= 3 && G.ext[1] >= 3 && G.ext[2] >= 3;
}

// Steps per pass of the fused rollout for a request (0 = choose): 2D grids 8;
// 3D grids 1 where the one-step streaming path applies, else 2 for order 2 and 1
// for order 4 on the temporally blocked kernel (the fastest depths at 512^3 on
// B200), at most heat3d_kmax; other 3D grids 1.
int heat_depth(const Geo& G, int ncomp, int steps_per_pass) {
  const bool two_d = (G.ndims == 2 && G.n[2] == 1);
  if (two_d) return steps_per_pass > 0 ? steps_per_pass : 8;
  if (!heat3d_ok(G, ncomp)) return 1;
  const int k = steps_per_pass > 0 ? steps_per_pass : (heat_split_shape(G, ncomp) ? 1 : (G.order == 2 ? 2 : 1));
  return k > heat3d_kmax(ncomp) ? heat3d_kmax(ncomp) : k;
}

// The one-step streaming 3D rollout: per step a surface fill of the source
// buffer (ghosts into the source and the output, then nodes into the source)
// and the OP_HEAT streaming kernel over the stencil box.  The caller's input is
// first copied into a buffer of this call (the fill writes in place), chosen so
// the last step lands in u_out; with u_out == u_in the rollout runs in place.
// input_scratch: the caller lets the input be overwritten, so step 0 fills it
// in place and the steps alternate between work and u_out, ending in u_out.
int heat3d_split_run(const float* u_in, float* u_out, float* work, const Geo& G, const Weights& W,
                     const PdeBCRules* rules, float alpha, float dt, int32_t nsteps, double t0, double tstep,
                     int32_t n0, bool input_scratch, cudaStream_t st) {
  const size_t bytes = (size_t)(G.n[0] * G.n[1] * G.n[2]) * sizeof(float);
  float* src;
  float* dst;
  if (u_out == u_in) {
    src = u_out;
    dst = work;
  } else if (input_scratch) {
    src = const_cast<float*>(u_in);
    dst = (nsteps & 1) ? u_out : work;  // step s writes u_out when nsteps - 1 - s is even
  } else {
    float* first = (nsteps & 1) ? work : u_out;
    PDE_CUDA_CHECK(cudaMemcpyAsync(first, u_in, bytes, cudaMemcpyDeviceToDevice, st));
    src = first;
    dst = (first == work) ? u_out : work;
  }
  const int n[3] = {(int)G.n[0], (int)G.n[1], (int)G.n[2]};
  Shell gs, ns;
  gs.init(n, 0, G.g);
  ns.init(n, G.g, 1);
  const int sms = sm_count();
  auto blocks_for = [&](long long cells) {
    const long long b = (cells + 255) / 256;
    return (int)(b < 8LL * sms ? (b > 0 ? b : 1) : 8LL * sms);
  };
  PdeBCRules Rs = *rules;
  for (int s = 0; s < nsteps; ++s) {
    if (rules->has_ramp)
      for (int i = 0; i < rules->ngroups; ++i)
        if (rules->group[i].func == PDE_BC_FUNC_RAMP)
          Rs.group[i].value = host_ramp_value(rules->group[i], t0, tstep, (long long)n0 + s);
    heat_fill_ghosts_kernel<<<blocks_for(gs.off[6]), 256, 0, st>>>(src, (s == 0 || s == nsteps - 1) ? dst : nullptr,
                                                                    G, 1, Rs, gs);
    heat_fill_nodes_kernel<<<blocks_for(ns.off[6]), 256, 0, st>>>(src, G, 1, Rs, ns);
    int rc = launch_status();
    if (rc) return rc;
    if (G.order == 2)
      rc = launch_stream3d_k<1, OP_HEAT, 1, 128, 16, 8, 3, MAP_PAIRS, MODE_EXACT>(src, dst, G, W, alpha, alpha, st, dt);
    else
      rc = launch_stream3d_k<2, OP_HEAT, 1, 128, 16, 4, 4, MAP_PAIRS, MODE_EXACT>(src, dst, G, W, alpha, alpha, st, dt);
    if (rc) return rc;
    float* t = src;
    src = dst;
    dst = (input_scratch && t == u_in) ? (src == u_out ? work : u_out) : t;  // u_in only as the first source
  }
  if (src != u_out) PDE_CUDA_CHECK(cudaMemcpyAsync(u_out, src, bytes, cudaMemcpyDeviceToDevice, st));
  return PDE_OK;
}

// The fused rollout; time-dependent groups only when `allow_ramp`; step n of
// the call fills the boundary at fp32(t0 + (n0 + n) * tstep).
int heat_rollout_run(const float* u_in, float* u_out, float* work, const PdeGrid* grid, int32_t ncomp,
                     const PdeBCRules* rules, float alpha, float dt, int32_t nsteps, int32_t steps_per_pass,
                     bool allow_ramp, double t0, double tstep, int32_t n0, void* stream, bool input_scratch = false) {
  if (!u_in || !u_out || !work || !grid || !rules || nsteps < 0 || steps_per_pass < 0 || n0 < 0) return PDE_ERR_ARG;
  if (ncomp < 1 || ncomp > PDE_FUSED_MAX_COMP || rules->ncomp != ncomp) return PDE_ERR_ARG;
  if (rules->has_ramp && !allow_ramp) return PDE_ERR_UNSUPPORTED;
  if (rules->ngroups < 0 || rules->ngroups > PDE_MAX_GROUPS) return PDE_ERR_ARG;
  if (work == u_in || work == u_out) return PDE_ERR_ARG;
  Geo G;
  if (!make_geo(grid, &G)) return PDE_ERR_SHAPE;
  if (G.g < G.order / 2 || G.g < 1) return PDE_ERR_GHOST;
  cudaStream_t st = as_stream(stream);
  const size_t bytes = (size_t)(G.n[0] * G.n[1] * G.n[2]) * ncomp * sizeof(float);
  if (nsteps == 0) {
    if (u_out != u_in) PDE_CUDA_CHECK(cudaMemcpyAsync(u_out, u_in, bytes, cudaMemcpyDeviceToDevice, st));
    return PDE_OK;
  }
  const Weights W = lap_weights(G.order, grid->dx);
  const int R = W.radius;
  const bool two_d = (G.ndims == 2 && G.n[2] == 1);
  const bool s3d = !two_d && heat3d_ok(G, ncomp);
  int k = heat_depth(G, ncomp, steps_per_pass);
  if (k > nsteps) k = nsteps;
  if (s3d && k == 1 && heat_split_shape(G, ncomp) && aligned16(u_in) && aligned16(u_out) && aligned16(work))
    return heat3d_split_run(u_in, u_out, work, G, W, rules, alpha, dt, nsteps, t0, tstep, n0, input_scratch, st);
  const int npasses = (nsteps + k - 1) / k;
  // buffer sequence: the last pass writes u_out.
  const float* src = u_in;
  const bool alias = (u_out == u_in);
  bool need_copy = false;
  float* dst_first;
  if (alias) {
    dst_first = work;
    need_copy = (npasses % 2) == 1;
  } else {
    dst_first = (npasses % 2 == 1) ? u_out : work;
  }
  float* dst = dst_first;
  int done = 0;
  for (int p = 0; p < npasses; ++p) {
    const int ks = (nsteps - done < k) ? (nsteps - done) : k;
    if (two_d) {
      H2Params P;
      P.X = (int)G.n[0]; P.Y = (int)G.n[1]; P.g = G.g; P.N = ncomp; P.k = ks;
      const int H = k * R + 1;  // must match heat2d_tb_kernel
      // Automatic shape: square tiles of about one per SM (sides 16..64, balanced
      // against the SM count), 512 threads; 16x32 tiles when those regions would
      // not fit in shared memory.
      int threads = g_threads2d > 0 ? g_threads2d : 512;
      if (g_tile2d[0] > 0) {  // pde_set_launch_2d
        P.TBX = g_tile2d[0];
        P.TBY = g_tile2d[1];
      } else {
        int t = (int)ceil(sqrt((double)P.X * P.Y / sm_count()));
        t = t < 16 ? 16 : (t > 64 ? 64 : t);
        P.TBX = P.TBY = t;
        balance_tiles(P.X, P.Y, &P.TBX, &P.TBY);
        if ((size_t)2 * (P.TBX + 2 * H) * (P.TBY + 2 * H) * ncomp * sizeof(float) > 227 * 1024 - sizeof(PdeBCRules)) {
          P.TBX = 16;
          P.TBY = 32;
        }
      }
      P.RXM = P.TBX + 2 * H; P.RYM = P.TBY + 2 * H;
      P.tiles_y = (P.Y + P.TBY - 1) / P.TBY;
      const int tiles = ((P.X + P.TBX - 1) / P.TBX) * P.tiles_y;
      for (int t = 0; t < 5; ++t) P.w[t] = W.w[t];
      P.alpha = alpha; P.dt = dt;
      P.t0 = t0; P.tstep = tstep; P.n0 = n0 + done;
      const size_t smem = (size_t)2 * P.RXM * P.RYM * ncomp * sizeof(float);
      if (smem > 227 * 1024 - sizeof(PdeBCRules)) return PDE_ERR_TOO_LARGE;
      // one component and at most 8 region cells per thread: the register cell-list kernel
      const long long cap = (long long)P.RXM * P.RYM;
      const int cpt = (ncomp == 1 && cap < (1 << 16)) ? (cap <= 4LL * threads ? 4 : cap <= 8LL * threads ? 8 : 0) : 0;
      const size_t smem_c = (size_t)3 * cap * sizeof(float);
      if (cpt > 0 && smem_c <= 227 * 1024 - sizeof(PdeBCRules)) {
#define PDE_H2C(RR, CC)                                                                                    \
  do {                                                                                                     \
    auto kern = rules->has_ramp ? heat2d_cells_kernel<RR, CC, true> : heat2d_cells_kernel<RR, CC, false>;  \
    PDE_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_c)); \
    const int lrc = launch_pdl(kern, tiles, threads, smem_c, st, src, dst, P, *rules);                     \
    if (lrc) return lrc;                                                                                   \
  } while (0)
        if (R == 1) {
          if (cpt == 4) PDE_H2C(1, 4); else PDE_H2C(1, 8);
        } else {
          if (cpt == 4) PDE_H2C(2, 4); else PDE_H2C(2, 8);
        }
#undef PDE_H2C
      } else {
#define PDE_H2(RR, NN)                                                                                  \
  do {                                                                                                  \
    auto kern = rules->has_ramp ? heat2d_tb_kernel<RR, NN, true> : heat2d_tb_kernel<RR, NN, false>;      \
    PDE_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    kern<<<tiles, threads, smem, st>>>(src, dst, P, *rules);                                            \
  } while (0)
      if (R == 1) {
        switch (ncomp) {
          case 1: PDE_H2(1, 1); break;
          case 2: PDE_H2(1, 2); break;
          case 3: PDE_H2(1, 3); break;
          default: PDE_H2(1, 4); break;
        }
      } else {
        switch (ncomp) {
          case 1: PDE_H2(2, 1); break;
          case 2: PDE_H2(2, 2); break;
          case 3: PDE_H2(2, 3); break;
          default: PDE_H2(2, 4); break;
        }
      }
#undef PDE_H2
      }
    } else if (s3d) {
      const int lrc = launch_heat3d(ks, R, ncomp, src, dst, G, W, alpha, dt, rules, t0, tstep, n0 + done, st);
      if (lrc) return lrc;
    } else {
      const int64_t total = G.n[0] * G.n[1] * G.n[2] * ncomp;
      // one step per launch: time-dependent group values are set in a copy of the rules
      PdeBCRules Rs = *rules;
      if (rules->has_ramp)
        for (int i = 0; i < rules->ngroups; ++i)
          if (rules->group[i].func == PDE_BC_FUNC_RAMP) Rs.group[i].value = host_ramp_value(rules->group[i], t0, tstep, (long long)n0 + done);
      if (R == 1) heat_step_kernel<1><<<grid_blocks(total, 256), 256, 0, st>>>(src, dst, G, ncomp, W, alpha, dt, Rs, total);
      else heat_step_kernel<2><<<grid_blocks(total, 256), 256, 0, st>>>(src, dst, G, ncomp, W, alpha, dt, Rs, total);
    }
    int rc = launch_status();
    if (rc) return rc;
    done += ks;
    src = dst;
    dst = (dst == work) ? u_out : work;
  }
  if (need_copy) PDE_CUDA_CHECK(cudaMemcpyAsync(u_out, work, bytes, cudaMemcpyDeviceToDevice, st));
  return PDE_OK;
}

}  // namespace

int pde_heat_rollout(const float* u_in, float* u_out, float* work, const PdeGrid* grid, int32_t ncomp,
                     const PdeBCRules* rules, float alpha, float dt, int32_t nsteps, int32_t steps_per_pass,
                     void* stream) {
  return heat_rollout_run(u_in, u_out, work, grid, ncomp, rules, alpha, dt, nsteps, steps_per_pass, false, 0.0, 0.0,
                          0, stream);
}

int pde_heat_rollout_at(const float* u_in, float* u_out, float* work, const PdeGrid* grid, int32_t ncomp,
                        const PdeBCRules* rules, float alpha, float dt, int32_t nsteps, int32_t steps_per_pass,
                        double t0, double t_step, void* stream) {
  return heat_rollout_run(u_in, u_out, work, grid, ncomp, rules, alpha, dt, nsteps, steps_per_pass, true, t0, t_step,
                          0, stream);
}

int pde_heat_rollout_from(const float* u_in, float* u_out, float* work, const PdeGrid* grid, int32_t ncomp,
                          const PdeBCRules* rules, float alpha, float dt, int32_t nsteps, int32_t steps_per_pass,
                          double t0, double t_step, int32_t n0, void* stream) {
  return heat_rollout_run(u_in, u_out, work, grid, ncomp, rules, alpha, dt, nsteps, steps_per_pass, true, t0, t_step,
                          n0, stream, true);
}

int pde_heat_pass_depth(const PdeGrid* grid, int32_t ncomp, int32_t steps_per_pass) {
  if (!grid || ncomp < 1 || ncomp > PDE_FUSED_MAX_COMP || steps_per_pass < 0) return PDE_ERR_ARG;
  Geo G;
  if (!make_geo(grid, &G)) return PDE_ERR_SHAPE;
  return heat_depth(G, ncomp, steps_per_pass);
}

namespace {

// Output tile of the temporally blocked 2D kernels (differentiable heat, wave,
// cavity): the largest of 32x64, 32x32, 16x32 that still gives every SM a tile,
// balanced against the SM count, unless pde_set_launch_2d fixed one.

// Threads per block for the wave kernels: enough warps per SM to hide shared-
// memory latency when tiles are few (up to 1024), 256 when every SM has several.
int pick_threads_2d(long long tiles) {
  if (g_threads2d > 0) return g_threads2d;
  const double per_sm = (double)tiles / sm_count();
  if (per_sm <= 1.0) return 1024;
  if (per_sm <= 2.0) return 512;
  return 256;
}

void pick_tile_2d(int X, int Y, int* tbx, int* tby) {
  if (g_tile2d[0] > 0) {
    *tbx = g_tile2d[0];
    *tby = g_tile2d[1];
    return;
  }
  static const int cand[3][2] = {{32, 64}, {32, 32}, {16, 32}};
  for (int c = 0; c < 3; ++c) {
    const long long tiles = (long long)((X + cand[c][0] - 1) / cand[c][0]) * ((Y + cand[c][1] - 1) / cand[c][1]);
    if (tiles >= sm_count() || c == 2) {
      *tbx = cand[c][0];
      *tby = cand[c][1];
      balance_tiles(X, Y, tbx, tby);
      return;
    }
  }
}

// Shared checks and launch geometry of the differentiable heat entry points.
int heat_diff_setup(const PdeGrid* grid, const PdeBCRules* rules, int steps_per_pass, int nsteps, Geo* G,
                    HAParams* P, int* kk) {
  if (!make_geo(grid, G)) return PDE_ERR_SHAPE;
  if (G->ndims != 2 || G->n[2] != 1) return PDE_ERR_UNSUPPORTED;
  if (G->g < G->order / 2 || G->g < 1) return PDE_ERR_GHOST;
  if (rules->ncomp != 1) return PDE_ERR_ARG;
  if (G->n[0] < 2 * G->g + 3 || G->n[1] < 2 * G->g + 3) return PDE_ERR_SHAPE;
  const Weights W = lap_weights(G->order, grid->dx);
  memset(P, 0, sizeof(*P));
  P->X = (int)G->n[0];
  P->Y = (int)G->n[1];
  P->g = G->g;
  for (int t = 0; t < 5; ++t) P->w[t] = W.w[t];
  int k = steps_per_pass > 0 ? steps_per_pass : 8;
  if (k > nsteps) k = nsteps;
  if (k < 1) k = 1;
  *kk = k;
  pick_tile_2d(P->X, P->Y, &P->TBX, &P->TBY);
  P->tiles_y = (P->Y + P->TBY - 1) / P->TBY;
  P->cells = (long long)G->n[0] * G->n[1];
  return PDE_OK;
}

}  // namespace

namespace {
int heat_forward_run(const float* alpha, const float* u_in, float* u_out, float* work, const PdeGrid* grid,
                     const PdeBCRules* rules, float dt, int32_t nsteps, int32_t steps_per_pass, float* lstates,
                     double t0, double tstep, int n0, void* stream);
}  // namespace

extern "C" {

int pde_set_launch_2d(int32_t tile_x, int32_t tile_y, int32_t threads) {
  if (threads != 0 && threads != 256 && threads != 512 && threads != 1024) return PDE_ERR_ARG;
  if (!(tile_x == 0 && tile_y == 0) && (tile_x < 8 || tile_y < 8 || tile_x > 256 || tile_y > 256))
    return PDE_ERR_ARG;
  g_tile2d[0] = tile_x;
  g_tile2d[1] = tile_y;
  g_threads2d = threads;
  return PDE_OK;
}

int pde_heat_forward(const float* alpha, const float* u_in, float* u_out, float* work, const PdeGrid* grid,
                     const PdeBCRules* rules, float dt, int32_t nsteps, int32_t steps_per_pass, float* lstates,
                     void* stream) {
  if (rules && rules->has_ramp) return PDE_ERR_UNSUPPORTED;
  return heat_forward_run(alpha, u_in, u_out, work, grid, rules, dt, nsteps, steps_per_pass, lstates, 0.0, 0.0, 0,
                          stream);
}

int pde_heat_forward_at(const float* alpha, const float* u_in, float* u_out, float* work, const PdeGrid* grid,
                        const PdeBCRules* rules, float dt, int32_t nsteps, int32_t steps_per_pass, float* lstates,
                        double t0, double t_step, int32_t n0, void* stream) {
  if (n0 < 0) return PDE_ERR_ARG;
  return heat_forward_run(alpha, u_in, u_out, work, grid, rules, dt, nsteps, steps_per_pass, lstates, t0, t_step, n0,
                          stream);
}

}  // extern "C"

namespace {

int heat_forward_run(const float* alpha, const float* u_in, float* u_out, float* work, const PdeGrid* grid,
                     const PdeBCRules* rules, float dt, int32_t nsteps, int32_t steps_per_pass, float* lstates,
                     double t0, double tstep, int n0, void* stream) {
  if (!alpha || !u_in || !u_out || !work || !grid || !rules || nsteps < 0 || steps_per_pass < 0) return PDE_ERR_ARG;
  if (work == u_in || work == u_out) return PDE_ERR_ARG;
  Geo G;
  HAParams P;
  int k;
  int rc = heat_diff_setup(grid, rules, steps_per_pass, nsteps, &G, &P, &k);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  const size_t bytes = (size_t)P.cells * sizeof(float);
  if (nsteps == 0) {
    if (u_out != u_in) PDE_CUDA_CHECK(cudaMemcpyAsync(u_out, u_in, bytes, cudaMemcpyDeviceToDevice, st));
    return PDE_OK;
  }
  const int R = G.order / 2;
  const int H = k * R + 1;
  P.RC = (P.TBX + 2 * H) * (P.TBY + 2 * H);
  const size_t smem = (size_t)3 * P.RC * sizeof(float);
  if (smem > 227 * 1024) return PDE_ERR_TOO_LARGE;
  auto kern = R == 1 ? heat2d_field_fwd_kernel<1> : heat2d_field_fwd_kernel<2>;
  PDE_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int tiles = ((P.X + P.TBX - 1) / P.TBX) * P.tiles_y;
  const int threads = pick_threads_2d(tiles);
  P.alpha = alpha;
  P.dt = dt;
  P.ramp = rules->has_ramp ? 1 : 0;
  P.t0 = t0;
  P.tstep = tstep;
  const int npasses = (nsteps + k - 1) / k;
  const bool alias = (u_out == u_in);
  const float* src = u_in;
  float* dst = alias ? work : ((npasses % 2 == 1) ? u_out : work);
  int done = 0;
  for (int p = 0; p < npasses; ++p) {
    P.k = (nsteps - done < k) ? (nsteps - done) : k;
    P.lst = lstates ? lstates + (size_t)done * P.cells : nullptr;
    P.n0 = n0 + done;
    kern<<<tiles, threads, smem, st>>>(src, dst, P, *rules);
    rc = launch_status();
    if (rc) return rc;
    done += P.k;
    src = dst;
    dst = (dst == work) ? u_out : work;
  }
  if (src != u_out) PDE_CUDA_CHECK(cudaMemcpyAsync(u_out, src, bytes, cudaMemcpyDeviceToDevice, st));
  return PDE_OK;
}

}  // namespace

extern "C" {

int pde_heat_adjoint(const float* alpha, const float* lam_in, float* lam_out, const float* lstates,
                     float* grad_alpha, const PdeGrid* grid, const PdeBCRules* rules, float dt, int32_t nsteps,
                     int32_t steps_per_pass, float* work, void* stream) {
  if (!alpha || !lam_in || !lam_out || !lstates || !grad_alpha || !work || !grid || !rules || nsteps < 0 ||
      steps_per_pass < 0)
    return PDE_ERR_ARG;
  if (work == lam_in || work == lam_out) return PDE_ERR_ARG;
  Geo G;
  HAParams P;
  int k;
  int rc = heat_diff_setup(grid, rules, steps_per_pass, nsteps, &G, &P, &k);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  const size_t bytes = (size_t)P.cells * sizeof(float);
  if (nsteps == 0) {
    if (lam_out != lam_in) PDE_CUDA_CHECK(cudaMemcpyAsync(lam_out, lam_in, bytes, cudaMemcpyDeviceToDevice, st));
    return PDE_OK;
  }
  const int R = G.order / 2;
  const int H = k * R;
  P.RC = (P.TBX + 2 * H + 2 * (G.g + 2)) * (P.TBY + 2 * H + 2 * (G.g + 2));
  // four region fields, the boundary flags of the region, the tile's gradient and two S planes
  const size_t smem = ((size_t)5 * P.RC + (size_t)3 * P.TBX * P.TBY) * sizeof(float);
  if (smem > 227 * 1024) return PDE_ERR_TOO_LARGE;
  auto kern = R == 1 ? heat2d_adj_kernel<1> : heat2d_adj_kernel<2>;
  PDE_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int tiles = ((P.X + P.TBX - 1) / P.TBX) * P.tiles_y;
  const int threads = pick_threads_2d(tiles);
  P.alpha = alpha;
  P.dt = dt;
  P.lsts = lstates;
  P.galpha = grad_alpha;
  const int npasses = (nsteps + k - 1) / k;
  const bool alias = (lam_out == lam_in);
  const float* src = lam_in;
  float* dst = alias ? work : ((npasses % 2 == 1) ? lam_out : work);
  int done = 0;
  for (int p = 0; p < npasses; ++p) {
    P.k = (nsteps - done < k) ? (nsteps - done) : k;
    P.ntop = nsteps - 1 - done;
    kern<<<tiles, threads, smem, st>>>(src, dst, P, *rules);
    rc = launch_status();
    if (rc) return rc;
    done += P.k;
    src = dst;
    dst = (dst == work) ? lam_out : work;
  }
  if (src != lam_out) PDE_CUDA_CHECK(cudaMemcpyAsync(lam_out, src, bytes, cudaMemcpyDeviceToDevice, st));
  return PDE_OK;
}

}  // extern "C"

namespace {

bool wave_setup(const PdeGrid* grid, int steps_per_pass, int nsteps, Geo* G, WaveParams* P, int* kk, size_t* smem,
                int nbuf, int extra) {
  if (!make_geo(grid, G)) return false;
  if (G->ndims != 2 || G->n[2] != 1 || grid->order != 2 || G->g < 1) return false;
  const Weights WL = lap_weights(2, grid->dx);
  memset(P, 0, sizeof(*P));
  P->X = (int)G->n[0];
  P->Y = (int)G->n[1];
  P->g = G->g;
  for (int t = 0; t < 3; ++t) P->w[t] = WL.w[t];
  int k = steps_per_pass > 0 ? steps_per_pass : 8;
  if (k > nsteps) k = nsteps;
  if (k < 1) k = 1;
  *kk = k;
  pick_tile_2d(P->X, P->Y, &P->TBX, &P->TBY);
  P->tiles_y = (P->Y + P->TBY - 1) / P->TBY;
  P->RC = (P->TBX + 2 * k) * (P->TBY + 2 * k);
  P->cells = (long long)G->n[0] * G->n[1];
  P->srcx = -1;
  *smem = ((size_t)nbuf * P->RC + (size_t)extra * P->TBX * P->TBY) * sizeof(float);
  return *smem <= 227 * 1024;
}

// Register cell lists of the wave kernels: the region capacity bounds every
// block's rectangle, so MAXC (4, 6 or 8) cells per thread cover it; 0 = the
// general loop (rectangles beyond 8 cells per thread).
int wave_cells_per_thread(int rc, int threads) {
  if (rc <= 4 * threads) return 4;
  if (rc <= 6 * threads) return 6;
  if (rc <= 8 * threads) return 8;
  return 0;
}

}  // namespace

int pde_wave_forward(const float* K, const float* u_prev, const float* u_cur, float* out_prev, float* out_cur,
                     const float* src, int64_t src_cell, int32_t n0, int32_t nsteps, int32_t steps_per_pass,
                     float* lstates, float* work, const PdeGrid* grid, void* stream) {
  if (!K || !u_prev || !u_cur || !out_prev || !out_cur || !work || !grid || nsteps < 0 || n0 < 0) return PDE_ERR_ARG;
  if (src_cell >= 0 && !src) return PDE_ERR_ARG;
  Geo G;
  WaveParams P;
  int k;
  size_t smem;
  if (!wave_setup(grid, steps_per_pass, nsteps, &G, &P, &k, &smem, 3, 0)) return PDE_ERR_UNSUPPORTED;
  cudaStream_t st = as_stream(stream);
  const size_t bytes = sizeof(float) * (size_t)P.cells;
  if (nsteps == 0) {
    if (out_prev != u_prev) PDE_CUDA_CHECK(cudaMemcpyAsync(out_prev, u_prev, bytes, cudaMemcpyDeviceToDevice, st));
    if (out_cur != u_cur) PDE_CUDA_CHECK(cudaMemcpyAsync(out_cur, u_cur, bytes, cudaMemcpyDeviceToDevice, st));
    return PDE_OK;
  }
  if (src_cell >= P.cells) return PDE_ERR_ARG;
  if (src_cell >= 0) {
    P.srcx = (int)(src_cell / P.Y);
    P.srcy = (int)(src_cell % P.Y);
    P.src = src;
  }
  const int tiles = ((P.X + P.TBX - 1) / P.TBX) * P.tiles_y;
  const int threads = pick_threads_2d(tiles);
  const int cpt = wave_cells_per_thread(P.RC, threads);
  auto kern = cpt == 4 ? wave_fwd_tb_kernel<4> : cpt == 6 ? wave_fwd_tb_kernel<6> : cpt == 8 ? wave_fwd_tb_kernel<8> : wave_fwd_tb_kernel<0>;
  PDE_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int npasses = (nsteps + k - 1) / k;
  float* w0 = work;
  float* w1 = work + P.cells;
  const bool alias = out_prev == u_prev || out_cur == u_cur || out_prev == u_cur || out_cur == u_prev;
  bool to_out = alias ? false : (npasses % 2 == 1);
  const float* a = u_prev;
  const float* b = u_cur;
  int done = 0;
  for (int p = 0; p < npasses; ++p) {
    P.k = (nsteps - done < k) ? (nsteps - done) : k;
    P.n0 = n0 + done;
    P.lst = lstates ? lstates + (size_t)done * P.cells : nullptr;
    float* da = to_out ? out_prev : w0;
    float* db = to_out ? out_cur : w1;
    kern<<<tiles, threads, smem, st>>>(a, b, K, da, db, P);
    const int rc = launch_status();
    if (rc) return rc;
    a = da;
    b = db;
    done += P.k;
    to_out = !to_out;
  }
  if (a != out_prev) {
    PDE_CUDA_CHECK(cudaMemcpyAsync(out_prev, a, bytes, cudaMemcpyDeviceToDevice, st));
    PDE_CUDA_CHECK(cudaMemcpyAsync(out_cur, b, bytes, cudaMemcpyDeviceToDevice, st));
  }
  return PDE_OK;
}

int pde_wave_pair(const float* K, const float* u_prev, const float* u_cur, int32_t n0, int32_t nsteps_fwd,
                  float* lstates_fwd, const float* mu_next, const float* mu_next2, float* mu_out, float* mu_out_next,
                  const float* lstates_adj, float* grad_K, int32_t nsteps_adj, const float* src, int64_t src_cell,
                  int32_t steps_per_pass, float* work, const PdeGrid* grid, void* stream) {
  if (!K || !work || !grid || nsteps_fwd < 0 || nsteps_adj < 0 || n0 < 0 || steps_per_pass < 0) return PDE_ERR_ARG;
  if (nsteps_fwd > 0 && (!u_prev || !u_cur || !lstates_fwd)) return PDE_ERR_ARG;
  if (nsteps_adj > 0 && (!mu_next || !mu_next2 || !mu_out || !mu_out_next || !lstates_adj || !grad_K))
    return PDE_ERR_ARG;
  if (src_cell >= 0 && !src) return PDE_ERR_ARG;
  const int nmax = nsteps_fwd > nsteps_adj ? nsteps_fwd : nsteps_adj;
  if (nmax == 0) return PDE_OK;
  Geo G;
  WaveParams Pa;
  int k;
  size_t smem;
  // results do not depend on the pass depth: take the deepest one (up to the
  // requested) whose seven interleaved region floats per cell fit in shared memory
  bool ok = false;
  for (int kk = steps_per_pass > 0 ? steps_per_pass : 8; kk >= 1 && !ok; --kk)
    ok = wave_setup(grid, kk, nmax, &G, &Pa, &k, &smem, 7, 1);
  if (!ok) return PDE_ERR_UNSUPPORTED;
  if (src_cell >= Pa.cells) return PDE_ERR_ARG;
  WaveParams Pf = Pa;
  if (src_cell >= 0) {
    Pf.srcx = (int)(src_cell / Pf.Y);
    Pf.srcy = (int)(src_cell % Pf.Y);
    Pf.src = src;
  }
  Pa.lsts = lstates_adj;
  Pa.gK = grad_K;
  cudaStream_t st = as_stream(stream);
  const size_t bytes = sizeof(float) * (size_t)Pa.cells;
  const int tiles = ((Pa.X + Pa.TBX - 1) / Pa.TBX) * Pa.tiles_y;
  const int threads = pick_threads_2d(tiles);
  const int cpt = wave_cells_per_thread(Pa.RC, threads);
  // register lists: the packed kernel (two cells per slot, cpt/2 slots); beyond 8
  // cells per thread the general loop
  auto kern = cpt == 4 ? wave_pair2_tb_kernel<2> : cpt == 6 ? wave_pair2_tb_kernel<3> : wave_pair2_tb_kernel<4>;
  auto kern0 = wave_pair_tb_kernel;
  if (cpt > 0) PDE_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  else PDE_CUDA_CHECK(cudaFuncSetAttribute(kern0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  float* w[6];
  for (int i = 0; i < 6; ++i) w[i] = work + (size_t)i * Pa.cells;
  // forward part: (u_prev, u_cur) -> (w0, w1) -> (w2, w3) -> (w0, w1) ...; the inputs are never written
  const float* fa = u_prev;
  const float* fb = u_cur;
  int fslot = 0;
  // adjoint part: alternate (w4, w5) and the outputs so that its last pass writes the outputs
  const int npa = (nsteps_adj + k - 1) / k;
  const bool alias = mu_out == mu_next || mu_out_next == mu_next2 || mu_out == mu_next2 || mu_out_next == mu_next;
  bool to_out = alias ? false : (npa % 2 == 1);
  const float* ma = mu_next;
  const float* mb = mu_next2;
  for (int done = 0; done < nmax; done += k) {
    Pf.k = nsteps_fwd - done < k ? (nsteps_fwd - done > 0 ? nsteps_fwd - done : 0) : k;
    Pa.k = nsteps_adj - done < k ? (nsteps_adj - done > 0 ? nsteps_adj - done : 0) : k;
    Pf.n0 = n0 + done;
    Pf.lst = Pf.k > 0 ? lstates_fwd + (size_t)done * Pf.cells : nullptr;
    Pa.ntop = nsteps_adj - 1 - done;
    float* fo_a = w[2 * fslot];
    float* fo_b = w[2 * fslot + 1];
    float* mo_a = to_out ? mu_out : w[4];
    float* mo_b = to_out ? mu_out_next : w[5];
    if (cpt > 0) kern<<<tiles, threads, smem, st>>>(fa, fb, fo_a, fo_b, ma, mb, mo_a, mo_b, K, Pf, Pa, -0.0f);
    else kern0<<<tiles, threads, smem, st>>>(fa, fb, fo_a, fo_b, ma, mb, mo_a, mo_b, K, Pf, Pa);
    const int rc = launch_status();
    if (rc) return rc;
    if (Pf.k > 0) {
      fa = fo_a;
      fb = fo_b;
      fslot ^= 1;
    }
    if (Pa.k > 0) {
      ma = mo_a;
      mb = mo_b;
      to_out = !to_out;
    }
  }
  if (nsteps_adj > 0 && ma != mu_out) {
    PDE_CUDA_CHECK(cudaMemcpyAsync(mu_out, ma, bytes, cudaMemcpyDeviceToDevice, st));
    PDE_CUDA_CHECK(cudaMemcpyAsync(mu_out_next, mb, bytes, cudaMemcpyDeviceToDevice, st));
  }
  return PDE_OK;
}

int pde_wave_adjoint(const float* K, const float* mu_next, const float* mu_next2, float* mu_out, float* mu_out_next,
                     const float* lstates, float* grad_K, int32_t nsteps, int32_t steps_per_pass, float* work,
                     const PdeGrid* grid, void* stream) {
  if (!K || !mu_next || !mu_next2 || !mu_out || !mu_out_next || !lstates || !grad_K || !work || !grid ||
      nsteps < 1)
    return PDE_ERR_ARG;
  Geo G;
  WaveParams P;
  int k;
  size_t smem;
  if (!wave_setup(grid, steps_per_pass, nsteps, &G, &P, &k, &smem, 5, 1)) return PDE_ERR_UNSUPPORTED;

  cudaStream_t st = as_stream(stream);
  const size_t bytes = sizeof(float) * (size_t)P.cells;
  const int tiles = ((P.X + P.TBX - 1) / P.TBX) * P.tiles_y;
  const int threads = pick_threads_2d(tiles);
  const int cpt = wave_cells_per_thread(P.RC, threads);
  auto kern = cpt == 4 ? wave_adj_tb_kernel<4> : cpt == 6 ? wave_adj_tb_kernel<6> : cpt == 8 ? wave_adj_tb_kernel<8> : wave_adj_tb_kernel<0>;
  PDE_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int npasses = (nsteps + k - 1) / k;
  float* w0 = work;
  float* w1 = work + P.cells;
  const bool alias = mu_out == mu_next || mu_out_next == mu_next2 || mu_out == mu_next2 || mu_out_next == mu_next;
  bool to_out = alias ? false : (npasses % 2 == 1);
  const float* a = mu_next;
  const float* b = mu_next2;
  P.lsts = lstates;  // lstates[n] = L(u^n), steps numbered from 0 within the segment
  P.gK = grad_K;
  int done = 0;
  for (int p = 0; p < npasses; ++p) {
    P.k = (nsteps - done < k) ? (nsteps - done) : k;
    P.ntop = nsteps - 1 - done;
    float* da = to_out ? mu_out : w0;
    float* db = to_out ? mu_out_next : w1;
    kern<<<tiles, threads, smem, st>>>(a, b, K, da, db, P);
    const int rc = launch_status();
    if (rc) return rc;
    a = da;
    b = db;
    done += P.k;
    to_out = !to_out;
  }
  if (a != mu_out) {
    PDE_CUDA_CHECK(cudaMemcpyAsync(mu_out, a, bytes, cudaMemcpyDeviceToDevice, st));
    PDE_CUDA_CHECK(cudaMemcpyAsync(mu_out_next, b, bytes, cudaMemcpyDeviceToDevice, st));
  }
  return PDE_OK;
}

}  // extern "C"

namespace {

// Checks and constants shared by the cavity entry points; G describes the whole domain.
int ldc_setup(const PdeGrid* grid, const PdeBCRules* u_rules, const PdeBCRules* p_rules, const PdeLDCParams* prm,
              Geo* G, LdcConst* K, bool allow_ramp = false) {
  if (!grid || !u_rules || !p_rules || !prm) return PDE_ERR_ARG;
  if (u_rules->ncomp != 2 || p_rules->ncomp != 1) return PDE_ERR_ARG;
  if (!allow_ramp && (u_rules->has_ramp || p_rules->has_ramp)) return PDE_ERR_UNSUPPORTED;
  if (prm->jacobi_iters < 0 || prm->jacobi_per_pass < 0) return PDE_ERR_ARG;
  if (!make_geo(grid, G)) return PDE_ERR_SHAPE;
  if (G->ndims != 2 || G->n[2] != 1 || grid->order != 2) return PDE_ERR_UNSUPPORTED;
  if (G->g < 1) return PDE_ERR_GHOST;
  if (G->n[0] * G->n[1] >= (1LL << 30) || G->n[0] > 65535) return PDE_ERR_TOO_LARGE;  // 32-bit cells, grid rows
  const Weights WL = lap_weights(2, grid->dx), WD = d1_weights(2, grid->dx);
  for (int t = 0; t < 3; ++t) { K->wl[t] = WL.w[t]; K->wd[t] = WD.w[t]; }
  K->nu = prm->nu;
  K->dt = prm->dt;
  K->inv_dt = (float)(1.0 / (double)prm->dt);
  K->h2 = (float)(grid->dx * grid->dx);
  return PDE_OK;
}

// Jacobi launch geometry for k sweeps per pass over owned rows [own_lo, own_hi)
// of arrays holding rows [held_lo, held_hi) of a domain of G.n[0] rows.
struct JacobiLaunch {
  int tiles, threads, cpt;  // cpt: register cells per thread (0: the flat-walk kernel)
  size_t smem;
};

int jacobi_setup(const Geo& G, float h2, int k, int own_lo, int own_hi, int held_lo, int held_hi, J2Params* JP,
                 JacobiLaunch* L) {
  JP->X = (int)G.n[0]; JP->Y = (int)G.n[1]; JP->g = G.g;
  JP->own_lo = own_lo; JP->own_hi = own_hi; JP->held_lo = held_lo; JP->held_hi = held_hi;
  bool placed = false;
  if (g_tile2d[0] == 0 && g_threads2d == 0) {
    // automatic shape on grids that fill the SMs: one near-square tile per SM,
    // 1024 threads (the register cell-list kernel, at most 12 cells per thread)
    const int rows = own_hi - own_lo, sms = (int)sm_count();
    int nx = (int)lround(sqrt((double)sms * rows / JP->Y));
    nx = nx < 1 ? 1 : (nx > sms ? sms : nx);
    const int ny = sms / nx > 0 ? sms / nx : 1;
    const int tx = (rows + nx - 1) / nx, ty = (JP->Y + ny - 1) / ny;
    const long long capb = (long long)(tx + 2 * (k + 1)) * (ty + 2 * (k + 1));
    if (tx >= 32 && ty >= 32 && tx <= 256 && ty <= 256 && capb <= 12LL * 1024 && capb < (1 << 16)) {
      JP->TBX = tx;
      JP->TBY = ty;
      L->threads = 1024;
      placed = true;
    }
  }
  if (!placed) {
    pick_tile_2d(JP->X, JP->Y, &JP->TBX, &JP->TBY);
    L->threads = g_threads2d > 0 ? g_threads2d : 256;
  }
  JP->tiles_y = (JP->Y + JP->TBY - 1) / JP->TBY;
  JP->RXM = JP->TBX + 2 * (k + 1);
  JP->RYM = JP->TBY + 2 * (k + 1);
  JP->h2 = h2;
  L->tiles = ((own_hi - own_lo + JP->TBX - 1) / JP->TBX) * JP->tiles_y;
  // the register cell lists cover every block's stencil rows x RY <= RXM x RYM
  const long long cap = (long long)JP->RXM * JP->RYM;
  L->cpt = cap <= 4LL * L->threads ? 4 : cap <= 6LL * L->threads ? 6 : cap <= 8LL * L->threads ? 8
         : cap <= 12LL * L->threads ? 12 : 0;
  L->smem = (size_t)3 * cap * sizeof(float);  // both kernels: two levels and the rhs per cell
  if (L->smem > 227 * 1024) return PDE_ERR_TOO_LARGE;
  if (cap >= (1 << 16)) L->cpt = 0;  // the cell lists pack region indices in 16 bits
  const void* kern = L->cpt == 4 ? (const void*)jacobi2d_cells_kernel<4>
                   : L->cpt == 6 ? (const void*)jacobi2d_cells_kernel<6>
                   : L->cpt == 8 ? (const void*)jacobi2d_cells_kernel<8>
                   : L->cpt == 12 ? (const void*)jacobi2d_cells_kernel<12>
                                  : (const void*)jacobi2d_tb_kernel;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->smem) != cudaSuccess)
    return PDE_ERR_CUDA;
  return PDE_OK;
}

int launch_jacobi(const JacobiLaunch& L, cudaStream_t st, const float* pin, float* pout, const float* rhs,
                  float* resid, const J2Params& JP, const PdeBCRules& R) {
  switch (L.cpt) {
    case 4: return launch_pdl(jacobi2d_cells_kernel<4>, L.tiles, L.threads, L.smem, st, pin, pout, rhs, resid, JP, R);
    case 6: return launch_pdl(jacobi2d_cells_kernel<6>, L.tiles, L.threads, L.smem, st, pin, pout, rhs, resid, JP, R);
    case 8: return launch_pdl(jacobi2d_cells_kernel<8>, L.tiles, L.threads, L.smem, st, pin, pout, rhs, resid, JP, R);
    case 12:
      return launch_pdl(jacobi2d_cells_kernel<12>, L.tiles, L.threads, L.smem, st, pin, pout, rhs, resid, JP, R);
    default:
      jacobi2d_tb_kernel<<<L.tiles, L.threads, L.smem, st>>>(pin, pout, rhs, resid, JP, R);
      return launch_status();
  }
}

}  // namespace

namespace {

// The rules of step n: ramp groups take their value at fp32(t0 + n * tstep).
PdeBCRules rules_at(const PdeBCRules& R, double t0, double tstep, long long n) {
  PdeBCRules out = R;
  if (R.has_ramp)
    for (int i = 0; i < R.ngroups; ++i)
      if (R.group[i].func == PDE_BC_FUNC_RAMP) out.group[i].value = host_ramp_value(R.group[i], t0, tstep, n);
  return out;
}

int ldc_rollout_run(float* u, float* p, float* u_star, float* p_tmp, float* rhs, float* resid, const PdeGrid* grid,
                    const PdeBCRules* u_rules_in, const PdeBCRules* p_rules_in, const PdeLDCParams* prm,
                    int32_t nsteps, bool allow_ramp, double t0, double tstep, void* stream) {
  if (!u || !p || !u_star || !p_tmp || !rhs || nsteps < 0) return PDE_ERR_ARG;
  Geo G;
  LdcConst K;
  int rc = ldc_setup(grid, u_rules_in, p_rules_in, prm, &G, &K, allow_ramp);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  const int64_t cells = G.n[0] * G.n[1];
  const int X = (int)G.n[0];
  const dim3 grid2((unsigned)((G.n[1] + 255) / 256), (unsigned)X);
  if (resid && nsteps > 0) PDE_CUDA_CHECK(cudaMemsetAsync(resid, 0, sizeof(float) * nsteps, st));
  const int iters = prm->jacobi_iters;
  int k = prm->jacobi_per_pass > 0 ? prm->jacobi_per_pass : 10;
  if (k > iters && iters > 0) k = iters;
  J2Params JP;
  JacobiLaunch JL;
  rc = jacobi_setup(G, K.h2, k, 0, X, 0, X, &JP, &JL);
  if (rc) return rc;
  for (int step = 0; step < nsteps; ++step) {
    // time-dependent groups: step n fills every boundary at t0 + n * tstep
    const PdeBCRules ur = rules_at(*u_rules_in, t0, tstep, step), pr = rules_at(*p_rules_in, t0, tstep, step);
    const PdeBCRules* u_rules = &ur;
    const PdeBCRules* p_rules = &pr;
    ldc_predictor_kernel<<<grid2, 256, 0, st>>>(u, u_star, G, *u_rules, K, 0);
    ldc_divergence_kernel<<<grid2, 256, 0, st>>>(u_star, rhs, G, *u_rules, K, 0);
    float* src = p;
    float* dst = p_tmp;
    for (int done = 0; done < iters;) {
      JP.k = (iters - done < k) ? (iters - done) : k;
      done += JP.k;
      JP.last = (done == iters);
      rc = launch_jacobi(JL, st, src, dst, rhs, resid ? resid + step : nullptr, JP, *p_rules);
      if (rc) return rc;
      float* t = src;
      src = dst;
      dst = t;
    }
    if (src != p) PDE_CUDA_CHECK(cudaMemcpyAsync(p, src, sizeof(float) * cells, cudaMemcpyDeviceToDevice, st));
    ldc_project_kernel<<<grid2, 256, 0, st>>>(u_star, p, u, G, *u_rules, *p_rules, K, 0);
    rc = launch_status();
    if (rc) return rc;
  }
  return PDE_OK;
}

}  // namespace

extern "C" {

int pde_ldc_rollout(float* u, float* p, float* u_star, float* p_tmp, float* rhs, float* resid, const PdeGrid* grid,
                    const PdeBCRules* u_rules, const PdeBCRules* p_rules, const PdeLDCParams* prm, int32_t nsteps,
                    void* stream) {
  return ldc_rollout_run(u, p, u_star, p_tmp, rhs, resid, grid, u_rules, p_rules, prm, nsteps, false, 0.0, 0.0,
                         stream);
}

int pde_ldc_rollout_at(float* u, float* p, float* u_star, float* p_tmp, float* rhs, float* resid,
                       const PdeGrid* grid, const PdeBCRules* u_rules, const PdeBCRules* p_rules,
                       const PdeLDCParams* prm, int32_t nsteps, double t0, double t_step, void* stream) {
  return ldc_rollout_run(u, p, u_star, p_tmp, rhs, resid, grid, u_rules, p_rules, prm, nsteps, true, t0, t_step,
                         stream);
}


int pde_wc_rk2(const float* m_in, const float* rho_in, float* m_out, float* rho_out, const PdeGrid* grid,
               const PdeBCRules* u_rules, const PdeBCRules* rho_rules, const PdeWCParams* prm, int32_t nsteps,
               float* work, void* stream) {
  if (!m_in || !rho_in || !m_out || !rho_out || !grid || !u_rules || !rho_rules || !prm || !work || nsteps < 0)
    return PDE_ERR_ARG;
  if (work == m_in || work == m_out || work == rho_in || work == rho_out) return PDE_ERR_ARG;
  Geo G;
  if (!make_geo(grid, &G)) return PDE_ERR_SHAPE;
  if (G.ndims != 2 || G.n[2] != 1 || grid->order != 2 || G.g < 1) return PDE_ERR_UNSUPPORTED;
  if (G.n[0] < 2 * G.g + 3 || G.n[1] < 2 * G.g + 3) return PDE_ERR_SHAPE;
  if (u_rules->ncomp != 2 || rho_rules->ncomp != 1 || u_rules->has_ramp || rho_rules->has_ramp) return PDE_ERR_ARG;
  cudaStream_t st = as_stream(stream);
  const size_t cells = (size_t)G.n[0] * G.n[1];
  if (nsteps == 0) {
    if (m_out != m_in) PDE_CUDA_CHECK(cudaMemcpyAsync(m_out, m_in, 2 * cells * 4, cudaMemcpyDeviceToDevice, st));
    if (rho_out != rho_in) PDE_CUDA_CHECK(cudaMemcpyAsync(rho_out, rho_in, cells * 4, cudaMemcpyDeviceToDevice, st));
    return PDE_OK;
  }
  WCParams P;
  memset(&P, 0, sizeof(P));
  P.X = (int)G.n[0];
  P.Y = (int)G.n[1];
  P.g = G.g;
  // automatic shape: 32x32 tiles; 16x16 when those leave SMs idle, 64x32 when
  // there are several per SM (fewer halo cells per tile cell)
  const long long t32 = (long long)((P.X + 31) / 32) * ((P.Y + 31) / 32);
  P.TBX = P.TBY = 32;
  if (t32 < sm_count()) P.TBX = P.TBY = 16;
  else if (t32 >= 4LL * sm_count()) P.TBX = 64;
  if (g_tile2d[0] > 0) {  // pde_set_launch_2d
    P.TBX = g_tile2d[0];
    P.TBY = g_tile2d[1];
  }
  const int threads = (g_threads2d == 256 || g_threads2d == 512) ? g_threads2d : 512;
  P.tiles_y = (P.Y + P.TBY - 1) / P.TBY;
  P.RC = (P.TBX + 2 * WC_HALO) * (P.TBY + 2 * WC_HALO);
  const size_t smem = (size_t)10 * P.RC * sizeof(float);
  if (smem > 227 * 1024) return PDE_ERR_TOO_LARGE;
  const Weights WL = lap_weights(2, grid->dx), WD = d1_weights(2, grid->dx);
  for (int i = 0; i < 3; ++i) {
    P.wl[i] = WL.w[i];
    P.wd[i] = WD.w[i];
  }
  P.nu = (float)prm->nu;
  P.eps = (float)prm->eps;
  P.c2 = (float)prm->c2;
  P.rho0 = (float)prm->rho0;
  P.dt_half = (float)(prm->dt / 2);
  P.dt = (float)prm->dt;
  PDE_CUDA_CHECK(cudaFuncSetAttribute(wc_rk2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int tiles = ((P.X + P.TBX - 1) / P.TBX) * P.tiles_y;
  float* wm = work;
  float* wr = work + 2 * cells;
  const bool alias = m_out == m_in || rho_out == rho_in;
  bool to_out = alias ? false : (nsteps % 2 == 1);
  const float* sm_ = m_in;
  const float* sr = rho_in;
  for (int s = 0; s < nsteps; ++s) {
    float* dm = to_out ? m_out : wm;
    float* dr = to_out ? rho_out : wr;
    wc_rk2_kernel<<<tiles, threads, smem, st>>>(sm_, sr, dm, dr, P, *u_rules, *rho_rules);
    const int rc = launch_status();
    if (rc) return rc;
    sm_ = dm;
    sr = dr;
    to_out = !to_out;
  }
  if (sm_ != m_out) {
    PDE_CUDA_CHECK(cudaMemcpyAsync(m_out, sm_, 2 * cells * 4, cudaMemcpyDeviceToDevice, st));
    PDE_CUDA_CHECK(cudaMemcpyAsync(rho_out, sr, cells * 4, cudaMemcpyDeviceToDevice, st));
  }
  return PDE_OK;
}

int pde_ldc_slab_step(int32_t phase, float* u, float* u_star, const float* p_in, float* p_out, float* rhs,
                      float* resid, const PdeGrid* grid, const PdeSlab* slab, const PdeBCRules* u_rules,
                      const PdeBCRules* p_rules, const PdeLDCParams* prm, int32_t nsweeps, int32_t last,
                      void* stream) {
  if (!grid || !slab) return PDE_ERR_ARG;
  // the whole domain's geometry; the arrays hold rows [x_offset, x_offset + grid->shape[0])
  PdeGrid whole = *grid;
  whole.shape[0] = slab->x_global;
  Geo G;
  LdcConst K;
  int rc = ldc_setup(&whole, u_rules, p_rules, prm, &G, &K);
  if (rc) return rc;
  const int64_t Xg = slab->x_global, off = slab->x_offset, nloc = grid->shape[0];
  const int64_t lo = slab->own_lo, hi = slab->own_hi;
  if (grid->shape[1] != whole.shape[1] || off < 0 || nloc < 1 || off + nloc > Xg || lo < off || hi > off + nloc ||
      lo >= hi)
    return PDE_ERR_SHAPE;
  const int64_t Y = G.n[1];
  cudaStream_t st = as_stream(stream);
  // pointers addressed by global row: local row r is global row off + r
  auto gl = [&](const float* q, int ncomp) { return q ? q - off * Y * ncomp : nullptr; };
  const dim3 grid2((unsigned)((Y + 255) / 256), (unsigned)(hi - lo));
  // rows one beyond the owned range on a cut side must be held (halo)
  const bool cut_lo = lo > 0, cut_hi = hi < Xg;
  // a ghost row's fill reads the row two steps inward: a slab with a physical
  // side and a cut side must own rows beyond that partner
  if ((!cut_lo && cut_hi && hi < G.g + 2) || (!cut_hi && cut_lo && lo > Xg - G.g - 2)) return PDE_ERR_SHAPE;
  if (phase == PDE_LDC_PREDICT || phase == PDE_LDC_DIVERGENCE || phase == PDE_LDC_PROJECT) {
    if ((cut_lo && lo - 1 < off) || (cut_hi && hi + 1 > off + nloc)) return PDE_ERR_SHAPE;
  }
  switch (phase) {
    case PDE_LDC_PREDICT:
      if (!u || !u_star) return PDE_ERR_ARG;
      ldc_predictor_kernel<<<grid2, 256, 0, st>>>(gl(u, 2), const_cast<float*>(gl(u_star, 2)), G, *u_rules, K,
                                                  (int)lo);
      break;
    case PDE_LDC_DIVERGENCE:
      if (!u_star || !rhs) return PDE_ERR_ARG;
      ldc_divergence_kernel<<<grid2, 256, 0, st>>>(gl(u_star, 2), const_cast<float*>(gl(rhs, 1)), G, *u_rules, K,
                                                   (int)lo);
      break;
    case PDE_LDC_PROJECT:
      if (!u || !u_star || !p_in) return PDE_ERR_ARG;
      ldc_project_kernel<<<grid2, 256, 0, st>>>(gl(u_star, 2), gl(p_in, 1), const_cast<float*>(gl(u, 2)), G,
                                                *u_rules, *p_rules, K, (int)lo);
      break;
    case PDE_LDC_JACOBI: {
      if (!p_in || !p_out || !rhs || nsweeps < 1 || p_in == p_out) return PDE_ERR_ARG;
      // k sweeps invalidate k + 1 rows inward from a cut side of the held rows
      if ((cut_lo && lo - (nsweeps + 1) < off) || (cut_hi && hi + nsweeps + 1 > off + nloc)) return PDE_ERR_SHAPE;
      J2Params JP;
      JacobiLaunch JL;
      rc = jacobi_setup(G, K.h2, nsweeps, (int)lo, (int)hi, (int)off, (int)(off + nloc), &JP, &JL);
      if (rc) return rc;
      JP.k = nsweeps;
      JP.last = last ? 1 : 0;
      rc = launch_jacobi(JL, st, gl(p_in, 1), const_cast<float*>(gl(p_out, 1)), gl(rhs, 1), resid, JP, *p_rules);
      if (rc) return rc;
      break;
    }
    default:
      return PDE_ERR_ARG;
  }
  return launch_status();
}

}  // extern "C"

// ---- batched rollouts --------------------------------------------------------
namespace {

constexpr int BATCH_TILE_X = 32, BATCH_TILE_Y = 64, BATCH_K = 8;
constexpr size_t BATCH_QUEUE_OFF_ALIGN = 256;

size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// work layout: [descriptor table][queue counter, 256 B][progress: u32 per tile]
bool batch_layout(const PdeBatchGrid* grids, int ngrids, int tx, int ty, int64_t* total_tiles, size_t* table_bytes,
                  size_t* bytes) {
  int64_t tiles = 0;
  for (int i = 0; i < ngrids; ++i) {
    const int64_t X = grids[i].shape[0], Y = grids[i].shape[1];
    if (X < 1 || Y < 1 || X > (1 << 30) || Y > (1 << 30)) return false;
    tiles += ((X + tx - 1) / tx) * ((Y + ty - 1) / ty);
  }
  if (tiles <= 0 || tiles > (1LL << 30)) return false;
  *total_tiles = tiles;
  *table_bytes = round_up((size_t)ngrids * sizeof(BatchGridDev), BATCH_QUEUE_OFF_ALIGN);
  *bytes = *table_bytes + BATCH_QUEUE_OFF_ALIGN + (size_t)tiles * sizeof(unsigned);
  return true;
}

int batch_halo(int kind, int order, int k) { return kind == PDE_BATCH_HEAT ? k * (order / 2) + 1 : k; }

template <int OP, int R>
int batch_occupancy(int smem, int* occ) {
  auto kern = batched_kernel<OP, R>;
  PDE_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int o = 0;
  PDE_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, 256, smem));
  if (o < 1) return PDE_ERR_TOO_LARGE;
  *occ = o;
  return PDE_OK;
}

}  // namespace

namespace {
int batch_rollout_run(const PdeBatchPlan* plan, int32_t nsteps, double t0, void* stream);
}  // namespace

extern "C" {

int pde_batch_work_bytes(const PdeBatchGrid* grids, int32_t ngrids, int32_t tile_x, int32_t tile_y,
                         uint64_t* bytes) {
  if (!grids || ngrids < 1 || !bytes || tile_x < 0 || tile_y < 0) return PDE_ERR_ARG;
  const int tx = tile_x > 0 ? tile_x : BATCH_TILE_X, ty = tile_y > 0 ? tile_y : BATCH_TILE_Y;
  int64_t tiles;
  size_t tb, b;
  if (!batch_layout(grids, ngrids, tx, ty, &tiles, &tb, &b)) return PDE_ERR_SHAPE;
  *bytes = b;
  return PDE_OK;
}

int pde_batch_plan(int32_t kind, const PdeBatchGrid* grids, int32_t ngrids, int32_t ghost_cells, int32_t order,
                   const PdeBCRules* rules, int32_t tile_x, int32_t tile_y, int32_t steps_per_pass, void* work,
                   uint64_t work_bytes, PdeBatchPlan* plan, void* stream) {
  if (!grids || ngrids < 1 || !work || !plan || tile_x < 0 || tile_y < 0 || steps_per_pass < 0) return PDE_ERR_ARG;
  if (kind != PDE_BATCH_HEAT && kind != PDE_BATCH_WAVE) return PDE_ERR_ARG;
  if (order != 2 && order != 4) return PDE_ERR_ARG;
  if (kind == PDE_BATCH_WAVE && order != 2) return PDE_ERR_UNSUPPORTED;
  if (ghost_cells < order / 2 || ghost_cells < 1) return PDE_ERR_GHOST;
  if (kind == PDE_BATCH_HEAT) {
    if (!rules) return PDE_ERR_ARG;
    if (rules->ncomp != 1) return PDE_ERR_ARG;
  }
  if ((reinterpret_cast<uintptr_t>(work) & (BATCH_QUEUE_OFF_ALIGN - 1)) != 0) return PDE_ERR_ALIGN;
  const int tx = tile_x > 0 ? tile_x : BATCH_TILE_X, ty = tile_y > 0 ? tile_y : BATCH_TILE_Y;
  const int k = steps_per_pass > 0 ? steps_per_pass : BATCH_K;
  const int H = batch_halo(kind, order, k);
  if (H > tx || H > ty || tx > 4096 || ty > 4096) return PDE_ERR_ARG;
  int64_t tiles;
  size_t table_bytes, bytes;
  if (!batch_layout(grids, ngrids, tx, ty, &tiles, &table_bytes, &bytes)) return PDE_ERR_SHAPE;
  if (work_bytes < bytes) return PDE_ERR_TOO_LARGE;
  const int nbuf = kind == PDE_BATCH_HEAT ? 2 : 3;
  const size_t smem = (size_t)nbuf * (tx + 2 * H) * (ty + 2 * H) * sizeof(float);
  if (smem > 227 * 1024) return PDE_ERR_TOO_LARGE;
  BatchGridDev* host = new BatchGridDev[ngrids];
  int64_t base = 0;
  for (int i = 0; i < ngrids; ++i) {
    const PdeBatchGrid& B = grids[i];
    const int64_t X = B.shape[0], Y = B.shape[1];
    const bool ok = B.field && B.scratch && (kind == PDE_BATCH_HEAT || B.field_prev) && B.dx > 0.0 &&
                    X > 2 * ghost_cells + 1 && Y > 2 * ghost_cells + 1 && B.field != B.scratch &&
                    B.field_prev != B.field;
    if (!ok) {
      delete[] host;
      return X > 2 * ghost_cells + 1 && Y > 2 * ghost_cells + 1 ? PDE_ERR_ARG : PDE_ERR_SHAPE;
    }
    BatchGridDev& D = host[i];
    memset(&D, 0, sizeof(D));
    const size_t cells = (size_t)X * Y;
    D.a0 = B.field;
    D.a1 = kind == PDE_BATCH_WAVE ? B.field_prev : nullptr;
    D.b0 = B.scratch;
    D.b1 = kind == PDE_BATCH_WAVE ? B.scratch + cells : nullptr;
    D.X = (int)X;
    D.Y = (int)Y;
    D.tiles_y = (int)((Y + ty - 1) / ty);
    D.ntiles = (int)(((X + tx - 1) / tx) * D.tiles_y);
    D.tile_base = (int)base;
    base += D.ntiles;
    D.coef = B.coef;
    D.dt = B.dt;
    D.dx32 = (float)B.dx;
    const Weights W = lap_weights(order, B.dx);
    for (int t = 0; t < 5; ++t) D.w[t] = W.w[t];
  }
  cudaStream_t st = as_stream(stream);
  const cudaError_t ce = cudaMemcpyAsync(work, host, (size_t)ngrids * sizeof(BatchGridDev), cudaMemcpyHostToDevice, st);
  delete[] host;
  if (ce != cudaSuccess) return PDE_ERR_CUDA;
  int occ = 0, rc;
  if (kind == PDE_BATCH_HEAT)
    rc = order == 2 ? batch_occupancy<BATCH_HEAT, 1>((int)smem, &occ) : batch_occupancy<BATCH_HEAT, 2>((int)smem, &occ);
  else
    rc = batch_occupancy<BATCH_WAVE, 1>((int)smem, &occ);
  if (rc) return rc;
  memset(plan, 0, sizeof(*plan));
  plan->table = work;
  plan->kind = kind;
  plan->ngrids = ngrids;
  plan->total_tiles = (int32_t)tiles;
  plan->ghost_cells = ghost_cells;
  plan->order = order;
  plan->tile_x = tx;
  plan->tile_y = ty;
  plan->steps_per_pass = k;
  plan->blocks = occ * sm_count();
  plan->smem_bytes = (int32_t)smem;
  if (kind == PDE_BATCH_HEAT) plan->rules = *rules;
  return PDE_OK;
}

int pde_batch_rollout(const PdeBatchPlan* plan, int32_t nsteps, void* stream) {
  if (plan && plan->kind == PDE_BATCH_HEAT && plan->rules.has_ramp) return PDE_ERR_UNSUPPORTED;
  return batch_rollout_run(plan, nsteps, 0.0, stream);
}

int pde_batch_rollout_at(const PdeBatchPlan* plan, int32_t nsteps, double t0, void* stream) {
  return batch_rollout_run(plan, nsteps, t0, stream);
}

}  // extern "C"

namespace {

int batch_rollout_run(const PdeBatchPlan* plan, int32_t nsteps, double t0, void* stream) {
  if (!plan || !plan->table || nsteps < 0 || plan->steps_per_pass < 1 || plan->total_tiles < 1) return PDE_ERR_ARG;
  if (nsteps == 0) return PDE_OK;
  const int k = plan->steps_per_pass;
  int ntb = (nsteps + k - 1) / k;
  ntb += ntb & 1;  // even: the last block writes the parity-0 buffers (the caller's fields)
  if ((int64_t)ntb * plan->total_tiles >= (1LL << 31) - (int64_t)plan->blocks) return PDE_ERR_TOO_LARGE;
  const int kmax = (nsteps + ntb - 1) / ntb;
  size_t table_bytes = round_up((size_t)plan->ngrids * sizeof(BatchGridDev), BATCH_QUEUE_OFF_ALIGN);
  char* base = static_cast<char*>(plan->table);
  BatchParams P;
  P.grids = reinterpret_cast<const BatchGridDev*>(base);
  P.ngrids = plan->ngrids;
  P.total_tiles = plan->total_tiles;
  P.ntb = ntb;
  P.nsteps = nsteps;
  P.H = batch_halo(plan->kind, plan->order, kmax);
  P.TBX = plan->tile_x;
  P.TBY = plan->tile_y;
  const int Hp = batch_halo(plan->kind, plan->order, k);
  P.RC = (plan->tile_x + 2 * Hp) * (plan->tile_y + 2 * Hp);
  P.g = plan->ghost_cells;
  P.counter = reinterpret_cast<unsigned*>(base + table_bytes);
  P.progress = reinterpret_cast<unsigned*>(base + table_bytes + BATCH_QUEUE_OFF_ALIGN);
  P.wait_ns = g_wait_ns;
  P.ramp = (plan->kind == PDE_BATCH_HEAT && plan->rules.has_ramp) ? 1 : 0;
  P.t0 = t0;
  cudaStream_t st = as_stream(stream);
  PDE_CUDA_CHECK(cudaMemsetAsync(P.counter, 0, BATCH_QUEUE_OFF_ALIGN + (size_t)plan->total_tiles * sizeof(unsigned), st));
  const int64_t items = (int64_t)ntb * plan->total_tiles;
  const int blocks = (int)(items < plan->blocks ? items : plan->blocks);
  const size_t smem = (size_t)plan->smem_bytes;
  if (plan->kind == PDE_BATCH_HEAT) {
    if (plan->order == 2) batched_kernel<BATCH_HEAT, 1><<<blocks, 256, smem, st>>>(P, plan->rules);
    else batched_kernel<BATCH_HEAT, 2><<<blocks, 256, smem, st>>>(P, plan->rules);
  } else {
    batched_kernel<BATCH_WAVE, 1><<<blocks, 256, smem, st>>>(P, plan->rules);
  }
  return launch_status();
}

}  // namespace
