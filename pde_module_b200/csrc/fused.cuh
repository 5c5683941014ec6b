// Fused explicit steps: ghost/boundary fill + Laplacian + forward Euler in one
// pass, with the boundary groups compiled into a PdeBCRules table.
//
// The per-cell boundary semantics are those of functional_boundary.py:357-400
// applied group by group: a boundary node takes the vector of the last
// Dirichlet group that contains it (input vector with that group's components
// replaced); the ghost one step outside a node along an axis takes, per
// component, the formula of the last group containing the node that sets the
// component, evaluated on the pre-boundary field at the interior neighbour
// (adj = node + inc).  All other cells keep the input value.
#pragma once
#include <type_traits>

#include "common.cuh"
#include "generic.cuh"

namespace pde {

__device__ __forceinline__ int node_class_axis(int64_t i, int64_t n, int g, bool elig) {
  if (!elig) return 1;
  if (i == g) return 0;
  if (i == n - 1 - g) return 2;
  return 1;
}

// Value written into a ghost component by group `gi` from the pre-boundary
// neighbour value `a` (inc = +1 for a low-side node, -1 for a high-side node).
__device__ __forceinline__ float ghost_value(const PdeBCRules& Rl, int gi, int inc, float a, float dx32) {
  const PdeBCGroupParam& G = Rl.group[gi];
  const float v = G.value;  // constant groups only on fused paths
  if (G.type == PDE_BC_DIRICHLET) return sub(mul(2.0f, v), a);
  return add(mul(mul((float)(-2 * inc), dx32), v), a);
}

__device__ __forceinline__ float ghost_value(const PdeBCRules& Rl, int gi, int inc, float a) {
  return ghost_value(Rl, gi, inc, a, Rl.dx32);
}

// Boundary-filled value u2 at cell (c0,c1,c2), component v, of the field
// `u` (pre-boundary), read through accessor U(i,j,k,v).
template <class Acc>
__device__ __forceinline__ float bc_eval(const Geo& G, const PdeBCRules& Rl, const Acc& U, int64_t c0, int64_t c1,
                                         int64_t c2, int v) {
  const int64_t c[3] = {c0, c1, c2};
  int ghost_axis = -1, nghost = 0;
  bool deep = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (G.n[a] == 1) continue;
    if (c[a] < G.g || c[a] > G.n[a] - 1 - G.g) {
      if (c[a] == G.g - 1 || c[a] == G.n[a] - G.g) { ghost_axis = a; ++nghost; }
      else deep = true;
    }
  }
  if (deep || nghost > 1) return U(c0, c1, c2, v);
  if (nghost == 1) {
    const int a = ghost_axis;
    const int inc = (c[a] == G.g - 1) ? 1 : -1;
    int64_t p[3] = {c0, c1, c2};
    p[a] += inc;  // partner node
    const int K = node_class_axis(p[0], G.n[0], G.g, G.n[0] > 1) * 9 +
                  node_class_axis(p[1], G.n[1], G.g, G.n[1] > 1) * 3 +
                  node_class_axis(p[2], G.n[2], G.g, G.n[2] > 1);
    const int gi = Rl.ghost_group[K][a][v];
    if (gi < 0) return U(c0, c1, c2, v);
    p[a] += inc;  // adj = node + inc
    return ghost_value(Rl, gi, inc, U(p[0], p[1], p[2], v));
  }
  const int K = node_class_axis(c0, G.n[0], G.g, G.n[0] > 1) * 9 + node_class_axis(c1, G.n[1], G.g, G.n[1] > 1) * 3 +
                node_class_axis(c2, G.n[2], G.g, G.n[2] > 1);
  if (K != 13) {
    const int gi = Rl.node_group[K];
    if (gi >= 0 && ((Rl.group[gi].comp_mask >> v) & 1u)) return Rl.group[gi].value;
  }
  return U(c0, c1, c2, v);
}

// u2 at a cell of a 2D grid: cells strictly inside the node ring are neither
// boundary nodes nor ghosts, so their boundary-filled value is the input value.
template <class Acc>
__device__ __forceinline__ float bc_eval2d(const Geo& G, const PdeBCRules& Rl, const Acc& U, int64_t i, int64_t j,
                                           int v) {
  if (i > G.g && i < G.n[0] - 1 - G.g && j > G.g && j < G.n[1] - 1 - G.g) return U(i, j, 0, v);
  return bc_eval(G, Rl, U, i, j, 0, v);
}

struct GlobalAcc {
  const float* u;
  int64_t s0, s1;  // cell strides
  int N;
  __device__ __forceinline__ float operator()(int64_t i, int64_t j, int64_t k, int v) const {
    return __ldg(u + (i * s0 + j * s1 + k) * N + v);
  }
};

// Cells of a box shell: the cells of [b, n-b)^3 with some coordinate in the
// t layers at either end of its axis ([b, b+t) or [n-b-t, n-b)).  Block (a, s)
// holds the layers of axis a on side s; axes before a range over their inner
// part [b+t, n-b-t) (their layers are earlier blocks), axes after a over
// [b, n-b), so every shell cell is in exactly one block.  Flat index ->
// (block, layer, the two other coordinates) with two integer divisions.
struct Shell {
  int n[3];
  int b, t;
  long long off[7];  // block (a, s) = 2a + s starts at off[2a + s]; off[6] = cells
  __host__ __device__ void init(const int* nn, int b_, int t_) {
    b = b_;
    t = t_;
    n[0] = nn[0]; n[1] = nn[1]; n[2] = nn[2];
    off[0] = 0;
    for (int a = 0; a < 3; ++a) {
      long long m = t;
      for (int q = 0; q < 3; ++q)
        if (q != a) m *= (q < a) ? (n[q] - 2 * b - 2 * t) : (n[q] - 2 * b);
      if (m < 0) m = 0;
      off[2 * a + 1] = off[2 * a] + m;
      off[2 * a + 2] = off[2 * a + 1] + m;
    }
  }
  __device__ void cell(long long i, int* c) const {
    int blk = 0;
    while (blk < 5 && i >= off[blk + 1]) ++blk;
    const int a = blk >> 1, s = blk & 1;
    long long r = i - off[blk];
    const int q0 = a == 0 ? 1 : 0, q1 = a == 2 ? 1 : 2;  // the other axes, ascending
    const int lo0 = (q0 < a) ? b + t : b, len0 = (q0 < a) ? n[q0] - 2 * b - 2 * t : n[q0] - 2 * b;
    const int lo1 = (q1 < a) ? b + t : b, len1 = (q1 < a) ? n[q1] - 2 * b - 2 * t : n[q1] - 2 * b;
    const long long per_layer = (long long)len0 * len1;
    const int l = (int)(r / per_layer);
    r -= (long long)l * per_layer;
    const int u = (int)(r / len1);
    c[a] = s ? n[a] - 1 - b - l : b + l;
    c[q0] = lo0 + u;
    c[q1] = lo1 + (int)(r - (long long)u * len1);
  }
};

// Surface fill of the one-step 3D heat rollout, first pass: every cell outside
// the stencil box [g, n-g)^3 takes its boundary-filled value u2 (bc_eval) in u
// (in place: a ghost's value reads its partner two cells inward, never another
// ghost cell, and deeper ghosts keep their value) and, when out is set, in the
// step's output (the first step seeds the constant deeper ghosts there; the last
// leaves the result's ghosts; steps between skip it, their output's ghosts
// being recomputed before anything reads them).
__global__ void __launch_bounds__(256) heat_fill_ghosts_kernel(float* __restrict__ u, float* __restrict__ out, Geo G,
                                                               int N, const PdeBCRules Rl, Shell S) {
  GlobalAcc U{u, G.cstride[0], G.cstride[1], N};
  const long long total = S.off[6] * N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / N;
    const int v = (int)(t - i * N);
    int c[3];
    S.cell(i, c);
    const float u2 = bc_eval(G, Rl, U, c[0], c[1], c[2], v);
    const long long k = ((long long)c[0] * G.n[1] + c[1]) * G.n[2] + c[2];
    u[k * N + v] = u2;
    if (out) out[k * N + v] = u2;
  }
}

// Second pass: the node layers (coordinate g or n-1-g inside the stencil box)
// take their Dirichlet values in u, after every ghost has read its partner's
// pre-boundary value.
__global__ void __launch_bounds__(256) heat_fill_nodes_kernel(float* __restrict__ u, Geo G, int N,
                                                              const PdeBCRules Rl, Shell S) {
  GlobalAcc U{u, G.cstride[0], G.cstride[1], N};
  const long long total = S.off[6] * N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / N;
    const int v = (int)(t - i * N);
    int c[3];
    S.cell(i, c);
    const float u2 = bc_eval(G, Rl, U, c[0], c[1], c[2], v);
    u[(((long long)c[0] * G.n[1] + c[1]) * G.n[2] + c[2]) * N + v] = u2;
  }
}

// One fused step over the whole array (any number of eligible axes), thread
// per (cell, component): stencil cells get u2 + dt*(alpha*L(u2)); every other
// cell gets u2 (its boundary-filled value).
template <int R>
__global__ void __launch_bounds__(256) heat_step_kernel(const float* __restrict__ in, float* __restrict__ out, Geo G,
                                                        int N, Weights W, float alpha, float dt, const PdeBCRules Rl,
                                                        int64_t total) {
  GlobalAcc U{in, G.cstride[0], G.cstride[1], N};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t cell = t / N;
    const int v = (int)(t - cell * N);
    const int64_t c2 = cell % G.n[2];
    const int64_t r = cell / G.n[2];
    const int64_t c1 = r % G.n[1];
    const int64_t c0 = r / G.n[1];
    const float u2 = bc_eval(G, Rl, U, c0, c1, c2, v);
    bool st = true;
    const int64_t c[3] = {c0, c1, c2};
#pragma unroll
    for (int a = 0; a < 3; ++a)
      if (G.n[a] > 1 && (c[a] < G.g || c[a] >= G.n[a] - G.g)) st = false;
    float res = u2;
    if (st) {
      float acc = 0.0f;
      for (int d = 0; d < G.ndims; ++d) {
        const int a = G.dims[d];
#pragma unroll
        for (int tp = 0; tp < 2 * R + 1; ++tp) {
          int64_t q[3] = {c0, c1, c2};
          q[a] += tp - R;
          acc = add(acc, mul(W.w[tp], bc_eval(G, Rl, U, q[0], q[1], q[2], v)));
        }
      }
      res = add(u2, mul(dt, mul(alpha, acc)));
    }
    out[cell * N + v] = res;
  }
}

// ---- 2D temporal blocking -------------------------------------------------
struct H2Params {
  int X, Y, g, N;
  int k;           // steps in this pass
  int TBX, TBY;    // output tile (array coordinates, ghosts included)
  int tiles_y;
  int RXM, RYM;    // smem region capacity (cells)
  float w[5];
  float alpha, dt;
  // time-dependent groups: step n of the rollout fills the boundary at
  // fp32(t0 + n * tstep), n = n0 + the step within this pass
  double t0, tstep;
  int n0;
};


// Boundary fill of the smem region (array rectangle [rx0,rx0+RX) x [ry0,ry0+RY)),
// in place: ghosts first (they read pre-boundary interior values), then nodes.
// S: floats per region cell (N for a dense field; more when the field's values
// are interleaved with other data, A pointing at the field's first value).
template <int N, int S = N>
__device__ __forceinline__ void bc_fill_region(float* A, const H2Params& P, const PdeBCRules& Rl, int rx0, int RX,
                                               int ry0, int RY, float dx32) {
  const int g = P.g, X = P.X, Y = P.Y;
  // A region without ghost or node cells (x, y in [g+1, n-g-2] throughout) has
  // nothing to fill; the test is the same for every thread of the block, so
  // the barriers below are skipped by all or by none.
  if (rx0 > g && rx0 + RX < X - g && ry0 > g && ry0 + RY < Y - g) return;
  const int nthr = blockDim.x, tid = threadIdx.x;
  // ghost strips: x = g-1 (low), x = X-g (high), partner rows y in [g, Y-g)
  const int ylo = max(g, ry0), yhi = min(Y - g, ry0 + RY);
  const int xlo = max(g, rx0), xhi = min(X - g, rx0 + RX);
  const int ny = max(0, yhi - ylo), nx = max(0, xhi - xlo);
  const int total = 2 * ny + 2 * nx;
  for (int e = tid; e < total; e += nthr) {
    int gx, gy, ax, inc;
    if (e < 2 * ny) {
      const int side = e / ny;
      gy = ylo + (e - side * ny);
      gx = side == 0 ? g - 1 : X - g;
      inc = side == 0 ? 1 : -1;
      ax = 0;
    } else {
      const int e2 = e - 2 * ny;
      const int side = e2 / nx;
      gx = xlo + (e2 - side * nx);
      gy = side == 0 ? g - 1 : Y - g;
      inc = side == 0 ? 1 : -1;
      ax = 1;
    }
    const int px = gx + (ax == 0 ? inc : 0), py = gy + (ax == 1 ? inc : 0);
    const int qx = px + (ax == 0 ? inc : 0), qy = py + (ax == 1 ? inc : 0);
    if (gx < rx0 || gx >= rx0 + RX || gy < ry0 || gy >= ry0 + RY) continue;
    if (qx < rx0 || qx >= rx0 + RX || qy < ry0 || qy >= ry0 + RY) continue;
    const int K = node_class_axis(px, X, g, true) * 9 + node_class_axis(py, Y, g, true) * 3 + 1;
#pragma unroll
    for (int v = 0; v < N; ++v) {
      const int gi = Rl.ghost_group[K][ax][v];
      if (gi < 0) continue;
      const float a = A[((qx - rx0) * RY + (qy - ry0)) * S + v];
      A[((gx - rx0) * RY + (gy - ry0)) * S + v] = ghost_value(Rl, gi, inc, a, dx32);
    }
  }
  __syncthreads();
  // node strips: x in {g, X-g-1} (y in [g,Y-g)), y in {g, Y-g-1} (x in [g,X-g))
  for (int e = tid; e < total; e += nthr) {
    int x, y;
    if (e < 2 * ny) {
      const int side = e / ny;
      y = ylo + (e - side * ny);
      x = side == 0 ? g : X - g - 1;
    } else {
      const int e2 = e - 2 * ny;
      const int side = e2 / nx;
      x = xlo + (e2 - side * nx);
      y = side == 0 ? g : Y - g - 1;
    }
    if (x < rx0 || x >= rx0 + RX || y < ry0 || y >= ry0 + RY) continue;
    const int K = node_class_axis(x, X, g, true) * 9 + node_class_axis(y, Y, g, true) * 3 + 1;
    const int gi = Rl.node_group[K];
    if (gi < 0) continue;
    const uint32_t m = Rl.group[gi].comp_mask;
    const float val = Rl.group[gi].value;
#pragma unroll
    for (int v = 0; v < N; ++v)
      if ((m >> v) & 1u) A[((x - rx0) * RY + (y - ry0)) * S + v] = val;
  }
  __syncthreads();
}

// The boundary-fill work of one thread for a region fixed over many fills (a
// launch, or a batched item): up to E ghost cells (region index, the partner two
// cells inward, boundary class, axis, side) and up to E node cells (region index,
// class), found once with the enumeration of bc_fill_region, so a fill needs no
// index arithmetic.  Region indices are packed in 16 bits; regions of 2^16 cells
// or more, or with more strip cells than E per thread, use bc_fill_region.
template <int E>
struct BcPlan {
  unsigned gh[E];  // ghost | partner << 16; ~0u: none
  int gm[E];       // class K | axis << 5 | (side low ? 1 : 0) << 6
  unsigned nd[E];  // node | K << 16; ~0u: none
  int mode;        // 0: nothing to fill, 1: planned, 2: bc_fill_region (block-uniform)
};

template <int E>
__device__ __forceinline__ void bc_plan(BcPlan<E>& pl, const H2Params& P, int rx0, int RX, int ry0, int RY) {
  const int g = P.g, X = P.X, Y = P.Y;
#pragma unroll
  for (int i = 0; i < E; ++i) {
    pl.gh[i] = ~0u;
    pl.gm[i] = 0;
    pl.nd[i] = ~0u;
  }
  pl.mode = 0;
  if (rx0 > g && rx0 + RX < X - g && ry0 > g && ry0 + RY < Y - g) return;
  const int nthr = blockDim.x, tid = threadIdx.x;
  const int ylo = max(g, ry0), yhi = min(Y - g, ry0 + RY);
  const int xlo = max(g, rx0), xhi = min(X - g, rx0 + RX);
  const int ny = max(0, yhi - ylo), nx = max(0, xhi - xlo);
  const int total = 2 * ny + 2 * nx;
  if (total > E * nthr || RX * RY >= (1 << 16) - 1) {
    pl.mode = 2;
    return;
  }
  pl.mode = 1;
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int e = tid + i * nthr;
    if (e >= total) continue;
    int gx, gy, ax, inc, x, y;  // ghost (gx, gy) and node (x, y) of strip element e
    if (e < 2 * ny) {
      const int side = e / ny;
      gy = ylo + (e - side * ny);
      gx = side == 0 ? g - 1 : X - g;
      inc = side == 0 ? 1 : -1;
      ax = 0;
      y = gy;
      x = side == 0 ? g : X - g - 1;
    } else {
      const int e2 = e - 2 * ny;
      const int side = e2 / nx;
      gx = xlo + (e2 - side * nx);
      gy = side == 0 ? g - 1 : Y - g;
      inc = side == 0 ? 1 : -1;
      ax = 1;
      x = gx;
      y = side == 0 ? g : Y - g - 1;
    }
    const int px = gx + (ax == 0 ? inc : 0), py = gy + (ax == 1 ? inc : 0);
    const int qx = px + (ax == 0 ? inc : 0), qy = py + (ax == 1 ? inc : 0);
    if (!(gx < rx0 || gx >= rx0 + RX || gy < ry0 || gy >= ry0 + RY) &&
        !(qx < rx0 || qx >= rx0 + RX || qy < ry0 || qy >= ry0 + RY)) {
      const int K = node_class_axis(px, X, g, true) * 9 + node_class_axis(py, Y, g, true) * 3 + 1;
      pl.gh[i] = (unsigned)((gx - rx0) * RY + (gy - ry0)) | ((unsigned)((qx - rx0) * RY + (qy - ry0)) << 16);
      pl.gm[i] = K | (ax << 5) | ((inc > 0 ? 1 : 0) << 6);
    }
    if (!(x < rx0 || x >= rx0 + RX || y < ry0 || y >= ry0 + RY)) {
      const int K = node_class_axis(x, X, g, true) * 9 + node_class_axis(y, Y, g, true) * 3 + 1;
      pl.nd[i] = (unsigned)((x - rx0) * RY + (y - ry0)) | ((unsigned)K << 16);
    }
  }
}

// bc_fill_region by a plan: the same cells, values and order (ghosts, barrier,
// nodes, barrier).
template <int N, int S, int E>
__device__ __forceinline__ void bc_fill_planned(float* A, const BcPlan<E>& pl, const H2Params& P,
                                                const PdeBCRules& Rl, int rx0, int RX, int ry0, int RY, float dx32) {
  if (pl.mode == 0) return;
  if (pl.mode == 2) {
    bc_fill_region<N, S>(A, P, Rl, rx0, RX, ry0, RY, dx32);
    return;
  }
#pragma unroll
  for (int i = 0; i < E; ++i) {
    if (pl.gh[i] == ~0u) continue;
    const int dst = (int)(pl.gh[i] & 0xffffu), src = (int)(pl.gh[i] >> 16);
    const int K = pl.gm[i] & 31, ax = (pl.gm[i] >> 5) & 1, inc = ((pl.gm[i] >> 6) & 1) ? 1 : -1;
#pragma unroll
    for (int v = 0; v < N; ++v) {
      const int gi = Rl.ghost_group[K][ax][v];
      if (gi < 0) continue;
      const float a = A[src * S + v];
      A[dst * S + v] = ghost_value(Rl, gi, inc, a, dx32);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < E; ++i) {
    if (pl.nd[i] == ~0u) continue;
    const int dst = (int)(pl.nd[i] & 0xffffu), K = (int)(pl.nd[i] >> 16);
    const int gi = Rl.node_group[K];
    if (gi < 0) continue;
    const uint32_t m = Rl.group[gi].comp_mask;
    const float val = Rl.group[gi].value;
#pragma unroll
    for (int v = 0; v < N; ++v)
      if ((m >> v) & 1u) A[dst * S + v] = val;
  }
  __syncthreads();
}

// k fused steps on a 2D grid (X, Y, 1, N) per pass.  Tiles cover the whole
// array (ghosts included); the smem region is the tile grown by H = k*R + 1
// cells on each side (clipped to the array).  Values invalidated by the
// region's cut edges move inward R cells per step; the extra cell covers the
// output ghost cells, whose last boundary fill reads the cell two steps
// inward (adj) at the previous step.
// RAMP: some groups take time-dependent values; the block keeps the rules in
// shared memory and sets those groups' values for each step before its fill.
template <int R, int N, bool RAMP>
__global__ void __launch_bounds__(1024) heat2d_tb_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                         const H2Params P, const PdeBCRules Rl) {
  extern __shared__ __align__(16) float sm[];
  __shared__ PdeBCRules SR;  // RAMP only: the rules with the current step's group values
  if (RAMP && threadIdx.x == 0) SR = Rl;
  const int tx = blockIdx.x / P.tiles_y, ty = blockIdx.x % P.tiles_y;
  const int bx0 = tx * P.TBX, by0 = ty * P.TBY;
  const int H = P.k * R + 1;
  const int rx0 = max(bx0 - H, 0), rx1 = min(bx0 + P.TBX + H, P.X);
  const int ry0 = max(by0 - H, 0), ry1 = min(by0 + P.TBY + H, P.Y);
  const int RX = rx1 - rx0, RY = ry1 - ry0;
  float* A = sm;
  float* B = sm + P.RXM * P.RYM * N;
  const int nrow = RY * N;  // floats per region row
  const int nt = (int)blockDim.x, RF = RX * nrow;
  // flat walk over the region's floats (rows of nrow contiguous floats): consecutive
  // threads take consecutive floats, every thread has the same share
  {
    RectWalk wk(nrow, nt);
    for (int i = threadIdx.x; i < RF; i += nt, wk.next())
      cp_async4(A + i, in + ((size_t)(rx0 + wk.row) * P.Y + ry0) * N + wk.col, true);
  }
  cp_async_wait_all();
  __syncthreads();
  const int g = P.g;
  // stencil cells whose R neighbours along both axes are inside the region
  const int sx0 = max(g, rx0 + R) - rx0, sx1 = min(P.X - g, rx0 + RX - R) - rx0;
  const int sy0 = max(g, ry0 + R) - ry0, sy1 = min(P.Y - g, ry0 + RY - R) - ry0;
  const int ox1 = min(bx0 + P.TBX, P.X), oy1 = min(by0 + P.TBY, P.Y);
  // the tile in region coordinates (inclusive bounds)
  const int tlx0 = bx0 - rx0, tlx1 = ox1 - 1 - rx0, tly0 = by0 - ry0, tly1 = oy1 - 1 - ry0;
  for (int s = 0; s < P.k; ++s) {
    if constexpr (RAMP) {
      // every read of SR's values in the previous step came before its last barrier
      const int gi = (int)threadIdx.x;
      if (gi < Rl.ngroups && Rl.group[gi].func == PDE_BC_FUNC_RAMP) {
        const float t = step_time(P.t0, P.tstep, P.n0 + s);
        SR.group[gi].value = bc_value(PDE_BC_FUNC_RAMP, Rl.group[gi].value, Rl.group[gi].t_max, &t);
      }
      __syncthreads();
      bc_fill_region<N>(A, P, SR, rx0, RX, ry0, RY, Rl.dx32);
    } else {
      bc_fill_region<N>(A, P, Rl, rx0, RX, ry0, RY, Rl.dx32);
    }
    // Only the box of cells within R (k - 1 - s) + 1 of the tile can reach the
    // tile's result (the boundary fills read inward, never farther out): the
    // step walks that box; the cells outside it keep stale values nobody reads.
    const int reach = R * (P.k - 1 - s) + 1;
    const int bx_lo = max(tlx0 - reach, 0), bx_hi = min(tlx1 + reach, RX - 1);
    const int by_lo = max(tly0 - reach, 0), by_hi = min(tly1 + reach, RY - 1);
    const int bw = (by_hi - by_lo + 1) * N, bcount = (bx_hi - bx_lo + 1) * bw;
    RectWalk wk(bw, nt);
    for (int q = threadIdx.x; q < bcount; q += nt, wk.next()) {
      const int lx = bx_lo + wk.row, lf = by_lo * N + wk.col, ly = lf / N;
      const int idx = lx * nrow + lf;
      const float u2 = A[idx];
      float res = u2;
      if (lx >= sx0 && lx < sx1 && ly >= sy0 && ly < sy1) {
        float acc = 0.0f;
#pragma unroll
        for (int t = 0; t < 2 * R + 1; ++t) acc = add(acc, mul(P.w[t], A[idx + (t - R) * nrow]));
#pragma unroll
        for (int t = 0; t < 2 * R + 1; ++t) acc = add(acc, mul(P.w[t], A[idx + (t - R) * N]));
        res = add(u2, mul(P.dt, mul(P.alpha, acc)));
      }
      B[idx] = res;
    }
    __syncthreads();
    float* tmp = A;
    A = B;
    B = tmp;
  }
  // The ghost cells of the result hold the last step's boundary-filled values
  // (non-stencil cells copy their filled value through).
  const int onrow = (oy1 - by0) * N;
  RectWalk wo(onrow, nt);
  for (int i = threadIdx.x; i < (ox1 - bx0) * onrow; i += nt, wo.next())
    out[((size_t)(bx0 + wo.row) * P.Y + by0) * N + wo.col] = A[(bx0 + wo.row - rx0) * nrow + (by0 - ry0) * N + wo.col];
}

// The same passes for a one-component field with register cell lists (as the
// wave and Jacobi kernels): the region interleaves the two levels (3 floats per
// cell, an odd stride: no bank conflicts), each thread's region cells are fixed
// for the pass (slots q = threadIdx.x + c * blockDim.x over the region's rows),
// each with one packed word (region index in the low 16 bits, distance from the
// tile above) and a bit for "stencil cell".  Step s reads level s & 1, writes the
// other, and updates the cells within R (k - 1 - s) + 1 of the tile: stencil
// cells by the reference's sum, the others (ghosts, cut edges) copied through.
// Same arithmetic and order per cell as heat2d_tb_kernel<R, 1, RAMP>; needs
// RXM x RYM <= MAXC * blockDim.x and < 2^16.
template <int R, int MAXC, bool RAMP>
__global__ void __launch_bounds__(1024) heat2d_cells_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                            const H2Params P, const PdeBCRules Rl) {
  pdl_launch_dependents();  // the next pass may be scheduled; it waits for this one
  extern __shared__ __align__(16) float sm[];
  __shared__ PdeBCRules SR;  // RAMP only: the rules with the current step's group values
  if (RAMP && threadIdx.x == 0) SR = Rl;
  constexpr int NB = 3;  // per region cell: level 0, level 1, (unused)
  const int tx = blockIdx.x / P.tiles_y, ty = blockIdx.x % P.tiles_y;
  const int bx0 = tx * P.TBX, by0 = ty * P.TBY;
  const int H = P.k * R + 1;
  const int rx0 = max(bx0 - H, 0), rx1 = min(bx0 + P.TBX + H, P.X);
  const int ry0 = max(by0 - H, 0), ry1 = min(by0 + P.TBY + H, P.Y);
  const int RX = rx1 - rx0, RY = ry1 - ry0, RC = RX * RY;
  const int nt = (int)blockDim.x;
  const int g = P.g;
  // stencil cells whose R neighbours along both axes are inside the region
  const int sx0 = max(g, rx0 + R) - rx0, sx1 = min(P.X - g, rx0 + RX - R) - rx0;
  const int sy0 = max(g, ry0 + R) - ry0, sy1 = min(P.Y - g, ry0 + RY - R) - ry0;
  const int ox1 = min(bx0 + P.TBX, P.X), oy1 = min(by0 + P.TBY, P.Y);
  // the tile in region coordinates (inclusive bounds)
  const int tlx0 = bx0 - rx0, tlx1 = ox1 - 1 - rx0, tly0 = by0 - ry0, tly1 = oy1 - 1 - ry0;
  int key[MAXC];      // region index | distance from the tile << 16; idle slots: INT_MAX
  unsigned sten = 0;  // bit c: slot c is a stencil cell
  {
    RectWalk wk(RY, nt);
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      key[c] = 0x7fffffff;
      if ((int)threadIdx.x + c * nt < RC) {
        const int lx = wk.row, ly = wk.col;
        const int d = max(max(max(tlx0 - lx, lx - tlx1), max(tly0 - ly, ly - tly1)), 0);
        key[c] = (lx * RY + ly) | (d << 16);
        if (lx >= sx0 && lx < sx1 && ly >= sy0 && ly < sy1) sten |= 1u << c;
      }
      wk.next();
    }
  }
  const int rs = NB * RY;
  BcPlan<1> bp;
  bc_plan(bp, P, rx0, RX, ry0, RY);
  pdl_wait();  // the previous pass's output (this pass's input) is complete
  {
    RectWalk wk(RY, nt);
    for (int i = threadIdx.x; i < RC; i += nt, wk.next())
      cp_async4(sm + NB * i, in + (size_t)(rx0 + wk.row) * P.Y + ry0 + wk.col, true);
  }
  cp_async_wait_all();
  __syncthreads();
  auto step = [&](auto PAR, int s) {
    constexpr int p = decltype(PAR)::value;  // reads level p, writes level 1 - p
    if constexpr (RAMP) {
      // every read of SR's values in the previous step came before its last barrier
      const int gi = (int)threadIdx.x;
      if (gi < Rl.ngroups && Rl.group[gi].func == PDE_BC_FUNC_RAMP) {
        const float t = step_time(P.t0, P.tstep, P.n0 + s);
        SR.group[gi].value = bc_value(PDE_BC_FUNC_RAMP, Rl.group[gi].value, Rl.group[gi].t_max, &t);
      }
      __syncthreads();
      bc_fill_planned<1, NB>(sm + p, bp, P, SR, rx0, RX, ry0, RY, Rl.dx32);
    } else {
      bc_fill_planned<1, NB>(sm + p, bp, P, Rl, rx0, RX, ry0, RY, Rl.dx32);
    }
    // Only the cells within R (k - 1 - s) + 1 of the tile can reach the tile's
    // result (the boundary fills read inward, never farther out).
    const int lim = (R * (P.k - 1 - s) + 2) << 16;  // dist <= reach  <=>  key < lim
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      if (key[c] >= lim) continue;
      float* pc = sm + NB * (key[c] & 0xffff) + p;
      const float u2 = pc[0];
      float res = u2;
      if ((sten >> c) & 1u) {
        float acc = 0.0f;
#pragma unroll
        for (int t = 0; t < 2 * R + 1; ++t) acc = add(acc, mul(P.w[t], pc[(t - R) * rs]));
#pragma unroll
        for (int t = 0; t < 2 * R + 1; ++t) acc = add(acc, mul(P.w[t], pc[(t - R) * NB]));
        res = add(u2, mul(P.dt, mul(P.alpha, acc)));
      }
      pc[1 - 2 * p] = res;  // the other level of the same cell
    }
    __syncthreads();
  };
  for (int s = 0; s < P.k; s += 2) {
    step(std::integral_constant<int, 0>{}, s);
    if (s + 1 < P.k) step(std::integral_constant<int, 1>{}, s + 1);
  }
  // The ghost cells of the result hold the last step's boundary-filled values
  // (non-stencil cells copy their filled value through).
  const int nw = P.k & 1;  // the level the last step wrote
  const int OX = ox1 - bx0, OY = oy1 - by0;
  RectWalk wo(OY, nt);
  for (int i = threadIdx.x; i < OX * OY; i += nt, wo.next())
    out[(size_t)(bx0 + wo.row) * P.Y + by0 + wo.col] = sm[NB * ((tlx0 + wo.row) * RY + tly0 + wo.col) + nw];
}

}  // namespace pde
