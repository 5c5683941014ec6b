// Immersed boundary: solid regions inside the grid with a staircase boundary
// (FDM/boundary/immersedBoundary.py).
//
// Geometry.  finalize() (immersedBoundary.py:57-66) classifies every cell of an
// int8 bitmask (nonzero = solid): a solid cell with a fluid (0) neighbour along an
// eligible axis is a boundary cell (locate_boundary, :406-438), the other solids
// are interior; fluid cells next to a solid are the fluid boundary (:110-131,
// :344-378); each boundary cell keeps the bitmask at -1 / +1 along each eligible
// axis (:133-151, :381-403).  The reference lists the cells with np.nonzero and
// np.unique, i.e. in C order.  Here the grid is cut into tiles of 2048
// consecutive cells (C order): a count pass gives each tile its number of cells of
// each class, one block scans the tile counts into offsets, and a scatter pass
// writes each tile's cells at its offset in order (a block-wide prefix over its
// threads' 8 consecutive cells), so the lists come out in C order without a sort.
//
// Boundary fill.  forward(u, fill) (:176-205, kernels :207-298): every boundary
// cell and component, Dirichlet -> the value; von Neumann -> the running mean
// avg += (c - avg) / n over the fluid neighbours, axes ascending, low side
// first, of c = u_f - (s * value) * dx (s = -1, +1), each operation rounded on its
// own; then interior solids take `fill` in every component.  The fill reads only
// fluid cells and writes only solid ones, so one launch does both and the field
// may be updated in place.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace {

using namespace pde;

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;  // consecutive cells per tile
constexpr int kBits = 21;                 // packed per-class counts (up to 2048 each)
constexpr uint64_t kMask = (1ull << kBits) - 1;
enum { C_SB = 0, C_IS = 1, C_FB = 2, C_EDGE = 3 };

struct IBGeo {
  int64_t n[3], st[3];
  int nd, dims[3];
  int64_t cells, ntiles;
};

bool ib_geo(const PdeGrid* grid, IBGeo* G) {
  Geo g;
  if (!make_geo(grid, &g)) return false;
  G->nd = g.ndims;
  for (int a = 0; a < 3; ++a) {
    G->n[a] = g.n[a];
    G->st[a] = g.cstride[a];
    G->dims[a] = g.dims[a];
  }
  G->cells = g.n[0] * g.n[1] * g.n[2];
  G->ntiles = (G->cells + kTile - 1) / kTile;
  return true;
}

// Work buffer layout: per-class tile counts (int32), per-class tile offsets
// (int64), per-class totals (int64), error word.
struct IBWork {
  int32_t* counts;
  int64_t* offsets;
  int64_t* totals;
  int32_t* err;
};

size_t ib_work_bytes(int64_t ntiles) {
  return (size_t)3 * ntiles * sizeof(int32_t) + (size_t)3 * ntiles * sizeof(int64_t) + 3 * sizeof(int64_t) + 64;
}

IBWork ib_work(void* w, int64_t ntiles) {
  char* p = static_cast<char*>(w);
  IBWork k;
  k.offsets = reinterpret_cast<int64_t*>(p);
  k.totals = k.offsets + 3 * ntiles;
  k.err = reinterpret_cast<int32_t*>(k.totals + 3);
  k.counts = k.err + 16;
  return k;
}

// Class of cell c (C_SB, C_IS, C_FB, C_EDGE: a solid on the outer layer), -1 for
// a fluid cell with no solid neighbour; nb receives a boundary cell's neighbours.
__device__ __forceinline__ int ib_class(const int8_t* __restrict__ bm, const IBGeo& G, int64_t c, int8_t* nb) {
  const int64_t q0 = c / G.st[0];
  const int64_t r = c - q0 * G.st[0];
  const int64_t q1 = r / G.st[1];
  const int64_t q[3] = {q0, q1, r - q1 * G.st[1]};
  if (bm[c] != 0) {
    for (int d = 0; d < G.nd; ++d) {
      const int a = G.dims[d];
      if (q[a] == 0 || q[a] == G.n[a] - 1) return C_EDGE;
    }
    bool b = false;
    for (int d = 0; d < G.nd; ++d) {
      const int a = G.dims[d];
      const int8_t lo = bm[c - G.st[a]], hi = bm[c + G.st[a]];
      if (nb) {
        nb[2 * d] = lo;
        nb[2 * d + 1] = hi;
      }
      b = b || lo == 0 || hi == 0;
    }
    return b ? C_SB : C_IS;
  }
  for (int d = 0; d < G.nd; ++d) {
    const int a = G.dims[d];
    if (q[a] > 0 && bm[c - G.st[a]] != 0) return C_FB;
    if (q[a] < G.n[a] - 1 && bm[c + G.st[a]] != 0) return C_FB;
  }
  return -1;
}

// Packed (SB, IS, FB) counts of this thread's kItems consecutive cells of tile t.
__device__ __forceinline__ uint64_t thread_counts(const int8_t* __restrict__ bm, const IBGeo& G, int64_t t,
                                                  bool* edge) {
  uint64_t cnt = 0;
  const int64_t c0 = t * kTile + (int64_t)threadIdx.x * kItems;
  for (int j = 0; j < kItems; ++j) {
    const int64_t c = c0 + j;
    if (c >= G.cells) break;
    const int k = ib_class(bm, G, c, nullptr);
    if (k == C_EDGE) *edge = true;
    else if (k >= 0) cnt += 1ull << (kBits * k);
  }
  return cnt;
}

// Exclusive prefix of v over the block's threads (kThreads), and the block total.
__device__ __forceinline__ uint64_t block_exclusive(uint64_t v, uint64_t* total) {
  __shared__ uint64_t warp_sum[kThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sum[w] = x;
  __syncthreads();
  if (w == 0) {
    uint64_t s = lane < kThreads / 32 ? warp_sum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kThreads / 32) warp_sum[lane] = s;  // inclusive over warps
  }
  __syncthreads();
  const uint64_t before = (w > 0 ? warp_sum[w - 1] : 0) + x - v;
  *total = warp_sum[kThreads / 32 - 1];
  __syncthreads();  // warp_sum is reused by the next call
  return before;
}

__global__ void __launch_bounds__(kThreads) ib_count_kernel(const int8_t* __restrict__ bm, const IBGeo G,
                                                            IBWork W) {
  for (int64_t t = blockIdx.x; t < G.ntiles; t += gridDim.x) {
    bool edge = false;
    const uint64_t cnt = thread_counts(bm, G, t, &edge);
    if (edge) atomicOr(W.err, 1);
    uint64_t total;
    block_exclusive(cnt, &total);
    if (threadIdx.x < 3) W.counts[threadIdx.x * G.ntiles + t] = (int32_t)((total >> (kBits * threadIdx.x)) & kMask);
  }
}

// One block: exclusive scan of each class's tile counts into offsets, and totals.
__global__ void __launch_bounds__(1024) ib_scan_kernel(const IBGeo G, IBWork W) {
  __shared__ int64_t part[1024];
  const int nt = (int)blockDim.x, tid = (int)threadIdx.x;
  const int64_t per = (G.ntiles + nt - 1) / nt;
  const int64_t lo = tid * per, hi = min(G.ntiles, lo + per);
  for (int k = 0; k < 3; ++k) {
    const int32_t* cnt = W.counts + k * G.ntiles;
    int64_t s = 0;
    for (int64_t t = lo; t < hi; ++t) s += cnt[t];
    part[tid] = s;
    __syncthreads();
    for (int o = 1; o < nt; o <<= 1) {  // inclusive Hillis-Steele scan over the threads' sums
      const int64_t y = tid >= o ? part[tid - o] : 0;
      __syncthreads();
      part[tid] += y;
      __syncthreads();
    }
    int64_t run = part[tid] - s;
    int64_t* off = W.offsets + k * G.ntiles;
    for (int64_t t = lo; t < hi; ++t) {
      off[t] = run;
      run += cnt[t];
    }
    if (tid == nt - 1) W.totals[k] = part[tid];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads) ib_scatter_kernel(const int8_t* __restrict__ bm, const IBGeo G,
                                                              IBWork W, int32_t* __restrict__ sb,
                                                              int8_t* __restrict__ fnb, int32_t* __restrict__ is,
                                                              int32_t* __restrict__ fb) {
  for (int64_t t = blockIdx.x; t < G.ntiles; t += gridDim.x) {
    bool edge = false;
    const uint64_t cnt = thread_counts(bm, G, t, &edge);
    uint64_t total;
    const uint64_t before = block_exclusive(cnt, &total);
    int64_t pos[3];
    for (int k = 0; k < 3; ++k) pos[k] = W.offsets[k * G.ntiles + t] + (int64_t)((before >> (kBits * k)) & kMask);
    const int64_t c0 = t * kTile + (int64_t)threadIdx.x * kItems;
    for (int j = 0; j < kItems; ++j) {
      const int64_t c = c0 + j;
      if (c >= G.cells) break;
      int8_t nb[6];
      const int k = ib_class(bm, G, c, nb);
      if (k < 0 || k == C_EDGE) continue;
      const int64_t q0 = c / G.st[0];
      const int64_t r = c - q0 * G.st[0];
      const int64_t q1 = r / G.st[1];
      int32_t* dst = k == C_SB ? sb : k == C_IS ? is : fb;
      const int64_t p = pos[k]++;
      dst[3 * p] = (int32_t)q0;
      dst[3 * p + 1] = (int32_t)q1;
      dst[3 * p + 2] = (int32_t)(r - q1 * G.st[1]);
      if (k == C_SB)
        for (int e = 0; e < 2 * G.nd; ++e) fnb[2 * G.nd * p + e] = nb[e];
    }
  }
}

// `in` and `out` may be the same array (no cell is both read and written).
__global__ void __launch_bounds__(256) ib_apply_kernel(const float* in, float* out,
                                                       const IBGeo G, int N, const int32_t* __restrict__ sb,
                                                       const int8_t* __restrict__ fnb, const int8_t* __restrict__ bt,
                                                       const float* __restrict__ bv, int64_t nsb,
                                                       const int32_t* __restrict__ is, int64_t nis, float fill,
                                                       float dx32) {
  const int64_t nb_items = nsb * N, total = nb_items + nis * N;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    if (i >= nb_items) {  // interior solid: the fill value in every component (:207-231)
      const int64_t j = i - nb_items, cell = j / N;
      const int v = (int)(j - cell * N);
      const int64_t c = is[3 * cell] * G.st[0] + is[3 * cell + 1] * G.st[1] + is[3 * cell + 2];
      out[c * N + v] = fill;
      continue;
    }
    const int64_t tid = i / N;
    const int var = (int)(i - tid * N);
    const int64_t c = sb[3 * tid] * G.st[0] + sb[3 * tid + 1] * G.st[1] + sb[3 * tid + 2];
    const float val = bv[i];
    const int8_t type = bt[i];
    if (type == PDE_BC_DIRICHLET) {
      out[c * N + var] = val;
    } else if (type == PDE_BC_VON_NEUMANN) {
      float avg = 0.0f, n = 1.0f;
      for (int d = 0; d < G.nd; ++d) {
        const int a = G.dims[d];
        for (int side = 0; side < 2; ++side) {
          if (fnb[2 * G.nd * tid + 2 * d + side] != 0) continue;  // not a fluid cell
          const int s = side ? 1 : -1;
          const float cv = sub(in[(c + s * G.st[a]) * N + var], mul(mul((float)s, val), dx32));
          avg = add(avg, __fdiv_rn(sub(cv, avg), n));
          n = add(n, 1.0f);
        }
      }
      out[c * N + var] = avg;
    }
  }
}

}  // namespace

extern "C" {

int64_t pde_ib_work_bytes(const PdeGrid* grid) {
  IBGeo G;
  if (!ib_geo(grid, &G)) return -1;
  return (int64_t)ib_work_bytes(G.ntiles);
}

int pde_ib_maps(const int8_t* bitmask, const PdeGrid* grid, int32_t* solid_boundary, int8_t* fluid_neighbors,
                int32_t* interior_solids, int32_t* fluid_boundary, int64_t* counts, void* work, int64_t work_bytes,
                void* stream) {
  if (!bitmask || !grid || !counts || !work) return PDE_ERR_ARG;
  IBGeo G;
  if (!ib_geo(grid, &G)) return PDE_ERR_SHAPE;
  if (G.cells > INT32_MAX || work_bytes < (int64_t)ib_work_bytes(G.ntiles)) return PDE_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  IBWork W = ib_work(work, G.ntiles);
  PDE_CUDA_CHECK(cudaMemsetAsync(W.err, 0, sizeof(int32_t), st));
  const int blocks = (int)(G.ntiles < 148LL * 16 ? G.ntiles : 148LL * 16);
  ib_count_kernel<<<blocks, kThreads, 0, st>>>(bitmask, G, W);
  PDE_CUDA_CHECK(cudaGetLastError());
  ib_scan_kernel<<<1, 1024, 0, st>>>(G, W);
  PDE_CUDA_CHECK(cudaGetLastError());
  int64_t host[4];
  PDE_CUDA_CHECK(cudaMemcpyAsync(host, W.totals, 3 * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  int32_t err = 0;
  PDE_CUDA_CHECK(cudaMemcpyAsync(&err, W.err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  PDE_CUDA_CHECK(cudaStreamSynchronize(st));
  if (err) return PDE_ERR_ARG;  // a solid cell on the array's outer layer
  for (int k = 0; k < 3; ++k) counts[k] = host[k];
  if (!solid_boundary) return PDE_OK;  // counts only
  if ((host[0] > 0 && !fluid_neighbors) || (host[1] > 0 && !interior_solids) || (host[2] > 0 && !fluid_boundary))
    return PDE_ERR_ARG;
  ib_scatter_kernel<<<blocks, kThreads, 0, st>>>(bitmask, G, W, solid_boundary, fluid_neighbors, interior_solids,
                                                  fluid_boundary);
  PDE_CUDA_CHECK(cudaGetLastError());
  return PDE_OK;
}

int pde_ib_apply(const float* in, float* out, const PdeGrid* grid, int32_t ncomp, const int32_t* solid_boundary,
                 const int8_t* fluid_neighbors, const int8_t* bc_type, const float* bc_value, int64_t n_boundary,
                 const int32_t* interior_solids, int64_t n_interior, float fill_value, void* stream) {
  if (!in || !out || !grid || ncomp < 1 || n_boundary < 0 || n_interior < 0) return PDE_ERR_ARG;
  if (n_boundary > 0 && (!solid_boundary || !fluid_neighbors || !bc_type || !bc_value)) return PDE_ERR_ARG;
  if (n_interior > 0 && !interior_solids) return PDE_ERR_ARG;
  IBGeo G;
  if (!ib_geo(grid, &G)) return PDE_ERR_SHAPE;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (out != in)
    PDE_CUDA_CHECK(cudaMemcpyAsync(out, in, (size_t)G.cells * ncomp * sizeof(float), cudaMemcpyDeviceToDevice, st));
  const int64_t items = (n_boundary + n_interior) * ncomp;
  if (items == 0) return PDE_OK;
  ib_apply_kernel<<<grid_blocks(items, 256), 256, 0, st>>>(in, out, G, ncomp, solid_boundary, fluid_neighbors,
                                                            bc_type, bc_value, n_boundary, interior_solids, n_interior,
                                                            fill_value, (float)grid->dx);
  return cudaGetLastError() == cudaSuccess ? PDE_OK : PDE_ERR_CUDA;
}

}  // extern "C"
