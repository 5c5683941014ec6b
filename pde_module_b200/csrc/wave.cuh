// Differentiable 2D wave equation (new: the reference's wave examples step a
// first-order (u, v) pair with forward Euler, tests/FDM/test_WaveStanding.py:71-76).
//
// State on the cells strictly inside the Dirichlet node ring (x, y in
// [g+1, n-g-2]); nodes and ghosts stay 0.  With K = dt^2 c^2 (a field) and L the
// reference's 5-point Laplacian (FDM/kernel/laplacian.py:40-46 order, alpha 1):
//
//   forward  u^{n+1} = 2 u^n - u^{n-1} + K o L(u^n) + s^n e_src
//   adjoint  mu^n    = 2 mu^{n+1} - mu^{n+2} + L(K o mu^{n+1})      (mu^{N+1} = 0)
//   gradient dJ/dK  += mu^{n+1} o L(u^n)      for n = N-1 .. 0, one add per step
//
// Both directions advance k steps per launch out of shared-memory tiles
// (halo k cells; cells outside the node ring are constant zeros, so only the
// region's cut edges lose one valid cell per step).  Every product and sum is
// rounded on its own.  The forward can store L(u^n), the Laplacian it has just
// formed, for the adjoint's gradient term; the adjoint keeps K o mu in shared
// memory (each product formed once per cell and step, the same value every
// neighbour reads) and accumulates dJ/dK of its tile in shared memory, in the
// order n = N-1 .. 0, so the result does not depend on k or the tile.
#pragma once
#include "common.cuh"

namespace pde {

struct WaveParams {
  int X, Y, g;
  int k;                 // steps in this pass
  int TBX, TBY, tiles_y;
  int RC;                // region capacity (cells)
  float w[3];            // Laplacian weights
  int srcx, srcy;        // source cell (forward), -1 for none
  const float* src;      // per-step source amplitude s^n (forward)
  int n0;                // forward: index n of u^n (the input "current" field)
  float* lst;            // forward: if set, L(u^{n0+s}) is stored at lst + s*cells
  long long cells;       // X*Y
  const float* lsts;     // adjoint: L(u^n) at lsts + n*cells
  int ntop;              // adjoint: the pass handles n = ntop, ntop-1, ..., ntop-k+1
  float* gK;             // adjoint: dJ/dK accumulated in place
};

__device__ __forceinline__ bool wave_inside(const WaveParams& P, int x, int y) {
  return x > P.g && x < P.X - 1 - P.g && y > P.g && y < P.Y - 1 - P.g;
}

// Laplacian at region index i of a region with row length RY (alpha 1).
__device__ __forceinline__ float lap5(const float* B, int i, int RY, const float* w) {
  float acc = 0.0f;
  acc = add(acc, mul(w[0], B[i - RY]));
  acc = add(acc, mul(w[1], B[i]));
  acc = add(acc, mul(w[2], B[i + RY]));
  acc = add(acc, mul(w[0], B[i - 1]));
  acc = add(acc, mul(w[1], B[i]));
  acc = add(acc, mul(w[2], B[i + 1]));
  return acc;
}

// Region of a tile: the tile grown by the halo H, clipped to the array.
struct WaveRegion {
  int bx0, by0, rx0, ry0, RX, RY, OX, OY;
  __device__ WaveRegion(const WaveParams& P, int H) {
    const int tx = blockIdx.x / P.tiles_y, ty = blockIdx.x % P.tiles_y;
    bx0 = tx * P.TBX;
    by0 = ty * P.TBY;
    rx0 = max(bx0 - H, 0);
    ry0 = max(by0 - H, 0);
    RX = min(bx0 + P.TBX + H, P.X) - rx0;
    RY = min(by0 + P.TBY + H, P.Y) - ry0;
    OX = min(P.TBX, P.X - bx0);
    OY = min(P.TBY, P.Y - by0);
  }
  __device__ int tile_to_region(int i) const {  // tile cell i (row-major OX x OY) -> region index
    const int lx = i / OY, ly = i - lx * OY;
    return (bx0 - rx0 + lx) * RY + (by0 - ry0 + ly);
  }
  __device__ size_t tile_to_global(int i, int Y) const {
    const int lx = i / OY, ly = i - lx * OY;
    return (size_t)(bx0 + lx) * Y + by0 + ly;
  }
};

__global__ void __launch_bounds__(256) wave_fwd_tb_kernel(const float* __restrict__ um_in,
                                                           const float* __restrict__ u0_in,
                                                           const float* __restrict__ Kf, float* __restrict__ um_out,
                                                           float* __restrict__ u0_out, const WaveParams P) {
  extern __shared__ __align__(16) float sm[];
  const WaveRegion Rg(P, P.k);
  const int RX = Rg.RX, RY = Rg.RY, RC = RX * RY, rx0 = Rg.rx0, ry0 = Rg.ry0;
  float* Bm = sm;
  float* B0 = sm + P.RC;
  float* Bp = sm + 2 * P.RC;
  float* Kt = sm + 3 * P.RC;
  for (int i = threadIdx.x; i < RC; i += blockDim.x) {
    const int lx = i / RY, ly = i - lx * RY;
    const size_t gi = (size_t)(rx0 + lx) * P.Y + ry0 + ly;
    const bool in = wave_inside(P, rx0 + lx, ry0 + ly);  // the state is zero outside the node ring
    Bm[i] = in ? __ldg(um_in + gi) : 0.0f;
    B0[i] = in ? __ldg(u0_in + gi) : 0.0f;
    Kt[i] = __ldg(Kf + gi);
  }
  __syncthreads();
  const int dq = (int)blockDim.x / RY, dr = (int)blockDim.x - dq * RY;
  const int lxs = (int)threadIdx.x / RY, lys = (int)threadIdx.x - lxs * RY;
  const int ox1 = Rg.bx0 + Rg.OX, oy1 = Rg.by0 + Rg.OY;
  for (int s = 0; s < P.k; ++s) {
    const float sn = (P.srcx >= 0) ? P.src[P.n0 + s] : 0.0f;
    float* Ls = P.lst ? P.lst + (size_t)s * P.cells : nullptr;
    int lx = lxs, ly = lys;
    for (int i = threadIdx.x; i < RC; i += blockDim.x) {
      const int x = rx0 + lx, y = ry0 + ly;
      float v = 0.0f, lap = 0.0f;
      if (wave_inside(P, x, y)) {
        if (lx >= 1 && lx < RX - 1 && ly >= 1 && ly < RY - 1) {
          lap = lap5(B0, i, RY, P.w);
          v = sub(mul(2.0f, B0[i]), Bm[i]);
          v = add(v, mul(Kt[i], lap));
          if (x == P.srcx && y == P.srcy) v = add(v, sn);
        } else {
          v = B0[i];  // cut edge: not valid after this step, never output
        }
      }
      Bp[i] = v;
      if (Ls && x >= Rg.bx0 && x < ox1 && y >= Rg.by0 && y < oy1) Ls[(size_t)x * P.Y + y] = lap;
      lx += dq;
      ly += dr;
      if (ly >= RY) { ly -= RY; ++lx; }
    }
    __syncthreads();
    float* t = Bm;
    Bm = B0;
    B0 = Bp;
    Bp = t;
  }
  for (int i = threadIdx.x; i < Rg.OX * Rg.OY; i += blockDim.x) {
    const size_t gi = Rg.tile_to_global(i, P.Y);
    const int ri = Rg.tile_to_region(i);
    um_out[gi] = Bm[ri];
    u0_out[gi] = B0[ri];
  }
}

__global__ void __launch_bounds__(256) wave_adj_tb_kernel(const float* __restrict__ m1_in,
                                                           const float* __restrict__ m2_in,
                                                           const float* __restrict__ Kf, float* __restrict__ m1_out,
                                                           float* __restrict__ m2_out, const WaveParams P) {
  extern __shared__ __align__(16) float sm[];
  const WaveRegion Rg(P, P.k);
  const int RX = Rg.RX, RY = Rg.RY, RC = RX * RY, rx0 = Rg.rx0, ry0 = Rg.ry0;
  float* M2 = sm;
  float* M1 = sm + P.RC;
  float* M0 = sm + 2 * P.RC;
  float* KM1 = sm + 3 * P.RC;  // K o mu^{n+1}
  float* KM0 = sm + 4 * P.RC;  // K o mu^{n}, formed with mu^n
  float* Kt = sm + 5 * P.RC;
  float* GA = sm + 6 * P.RC;   // dJ/dK of the tile (OX x OY)
  for (int i = threadIdx.x; i < RC; i += blockDim.x) {
    const int lx = i / RY, ly = i - lx * RY;
    const size_t gi = (size_t)(rx0 + lx) * P.Y + ry0 + ly;
    const bool in = wave_inside(P, rx0 + lx, ry0 + ly);
    const float m1 = in ? __ldg(m1_in + gi) : 0.0f, kk = __ldg(Kf + gi);
    M2[i] = in ? __ldg(m2_in + gi) : 0.0f;
    M1[i] = m1;
    Kt[i] = kk;
    KM1[i] = mul(kk, m1);
  }
  for (int i = threadIdx.x; i < Rg.OX * Rg.OY; i += blockDim.x) GA[i] = P.gK[Rg.tile_to_global(i, P.Y)];
  __syncthreads();
  const int dq = (int)blockDim.x / RY, dr = (int)blockDim.x - dq * RY;
  const int lxs = (int)threadIdx.x / RY, lys = (int)threadIdx.x - lxs * RY;
  const int ox1 = Rg.bx0 + Rg.OX, oy1 = Rg.by0 + Rg.OY;
  for (int s = 0; s < P.k; ++s) {
    const float* Ln = P.lsts + (size_t)(P.ntop - s) * P.cells;
    int lx = lxs, ly = lys;
    for (int i = threadIdx.x; i < RC; i += blockDim.x) {
      const int x = rx0 + lx, y = ry0 + ly;
      float v = 0.0f;
      if (wave_inside(P, x, y)) {
        if (lx >= 1 && lx < RX - 1 && ly >= 1 && ly < RY - 1) {
          // L(K o mu^{n+1})
          float acc = 0.0f;
          acc = add(acc, mul(P.w[0], KM1[i - RY]));
          acc = add(acc, mul(P.w[1], KM1[i]));
          acc = add(acc, mul(P.w[2], KM1[i + RY]));
          acc = add(acc, mul(P.w[0], KM1[i - 1]));
          acc = add(acc, mul(P.w[1], KM1[i]));
          acc = add(acc, mul(P.w[2], KM1[i + 1]));
          v = add(sub(mul(2.0f, M1[i]), M2[i]), acc);
        } else {
          v = M1[i];
        }
        // gradient term of step n on the tile: dJ/dK += mu^{n+1} o L(u^n)
        if (x >= Rg.bx0 && x < ox1 && y >= Rg.by0 && y < oy1) {
          const int t = (x - Rg.bx0) * Rg.OY + (y - Rg.by0);
          GA[t] = add(GA[t], mul(M1[i], __ldg(Ln + (size_t)x * P.Y + y)));
        }
      }
      M0[i] = v;
      KM0[i] = mul(Kt[i], v);
      lx += dq;
      ly += dr;
      if (ly >= RY) { ly -= RY; ++lx; }
    }
    __syncthreads();
    float* t = M2;
    M2 = M1;
    M1 = M0;
    M0 = t;
    t = KM1;
    KM1 = KM0;
    KM0 = t;
  }
  for (int i = threadIdx.x; i < Rg.OX * Rg.OY; i += blockDim.x) {
    const size_t gi = Rg.tile_to_global(i, P.Y);
    const int ri = Rg.tile_to_region(i);
    m1_out[gi] = M1[ri];
    m2_out[gi] = M2[ri];
    P.gK[gi] = GA[i];
  }
}

}  // namespace pde
