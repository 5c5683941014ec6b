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
// rounded on its own; the gradient is read-modified-written in global memory
// once per step in the order n = N-1 .. 0, so it does not depend on k.
#pragma once
#include "common.cuh"

namespace pde {

// Output tile of the wave kernels (the adjoint keeps per-thread gradient
// registers for it: 256 threads = 8 rows of 32 lanes).
constexpr int WAVE_TBX = 32, WAVE_TBY = 64;

struct WaveParams {
  int X, Y, g;
  int k;                 // steps in this pass
  int TBX, TBY, tiles_y;
  int RXM, RYM;          // region capacity (cells)
  float w[3];            // Laplacian weights
  int srcx, srcy;        // source cell (forward), -1 for none
  const float* src;      // per-step source amplitude s^n (forward)
  int n0;                // forward: index n of u^n (the input "current" field)
  float* states;         // forward: if set, u^{n0+1+s} is stored at states + s*cells
  long long cells;       // X*Y
  // adjoint
  const float* ustates;  // u^n for the pass's steps: u^{n} at ustates + (n - ubase)*cells
  int ubase;
  int ntop;              // adjoint: the pass handles n = ntop, ntop-1, ..., ntop-k+1
  float* gK;             // adjoint: dJ/dK accumulated in place
};

__device__ __forceinline__ bool wave_inside(const WaveParams& P, int x, int y) {
  return x > P.g && x < P.X - 1 - P.g && y > P.g && y < P.Y - 1 - P.g;
}

// Laplacian at region index idx of a region with row length RY (alpha 1).
__device__ __forceinline__ float lap5(const float* B, int idx, int RY, const float* w) {
  float acc = 0.0f;
  acc = add(acc, mul(w[0], B[idx - RY]));
  acc = add(acc, mul(w[1], B[idx]));
  acc = add(acc, mul(w[2], B[idx + RY]));
  acc = add(acc, mul(w[0], B[idx - 1]));
  acc = add(acc, mul(w[1], B[idx]));
  acc = add(acc, mul(w[2], B[idx + 1]));
  return acc;
}

__global__ void __launch_bounds__(256) wave_fwd_tb_kernel(const float* __restrict__ um_in,
                                                           const float* __restrict__ u0_in,
                                                           const float* __restrict__ Kf, float* __restrict__ um_out,
                                                           float* __restrict__ u0_out, const WaveParams P) {
  extern __shared__ __align__(16) float sm[];
  const int tx = blockIdx.x / P.tiles_y, ty = blockIdx.x % P.tiles_y;
  const int bx0 = tx * P.TBX, by0 = ty * P.TBY;
  const int H = P.k;
  const int rx0 = max(bx0 - H, 0), rx1 = min(bx0 + P.TBX + H, P.X);
  const int ry0 = max(by0 - H, 0), ry1 = min(by0 + P.TBY + H, P.Y);
  const int RX = rx1 - rx0, RY = ry1 - ry0;
  const int cap = P.RXM * P.RYM;
  float* Bm = sm;
  float* B0 = sm + cap;
  float* Bp = sm + 2 * cap;
  float* Kt = sm + 3 * cap;
  const int ly0 = threadIdx.x & 31, lx0 = threadIdx.x >> 5, nrows = blockDim.x >> 5;
  for (int lx = lx0; lx < RX; lx += nrows)
    for (int ly = ly0; ly < RY; ly += 32) {
      const size_t gi = (size_t)(rx0 + lx) * P.Y + ry0 + ly;
      const bool in = wave_inside(P, rx0 + lx, ry0 + ly);  // the state is zero outside the node ring
      Bm[lx * RY + ly] = in ? __ldg(um_in + gi) : 0.0f;
      B0[lx * RY + ly] = in ? __ldg(u0_in + gi) : 0.0f;
      Kt[lx * RY + ly] = __ldg(Kf + gi);
    }
  __syncthreads();
  for (int s = 0; s < P.k; ++s) {
    const float sn = (P.srcx >= 0) ? P.src[P.n0 + s] : 0.0f;
    for (int lx = lx0; lx < RX; lx += nrows)
      for (int ly = ly0; ly < RY; ly += 32) {
        const int idx = lx * RY + ly;
        const int x = rx0 + lx, y = ry0 + ly;
        float v = 0.0f;
        if (wave_inside(P, x, y)) {
          if (lx >= 1 && lx < RX - 1 && ly >= 1 && ly < RY - 1) {
            v = sub(mul(2.0f, B0[idx]), Bm[idx]);
            v = add(v, mul(Kt[idx], lap5(B0, idx, RY, P.w)));
            if (x == P.srcx && y == P.srcy) v = add(v, sn);
          } else {
            v = B0[idx];  // cut edge: not valid after this step, never output
          }
        }
        Bp[idx] = v;
      }
    __syncthreads();
    float* t = Bm;
    Bm = B0;
    B0 = Bp;
    Bp = t;
    if (P.states) {
      float* st = P.states + (size_t)s * P.cells;
      for (int lx = lx0; lx < min(P.TBX, P.X - bx0); lx += nrows)
        for (int ly = ly0; ly < min(P.TBY, P.Y - by0); ly += 32)
          st[(size_t)(bx0 + lx) * P.Y + by0 + ly] = B0[(bx0 + lx - rx0) * RY + (by0 + ly - ry0)];
    }
  }
  for (int lx = lx0; lx < min(P.TBX, P.X - bx0); lx += nrows)
    for (int ly = ly0; ly < min(P.TBY, P.Y - by0); ly += 32) {
      const size_t gi = (size_t)(bx0 + lx) * P.Y + by0 + ly;
      const int ri = (bx0 + lx - rx0) * RY + (by0 + ly - ry0);
      um_out[gi] = Bm[ri];
      u0_out[gi] = B0[ri];
    }
}

__global__ void __launch_bounds__(256) wave_adj_tb_kernel(const float* __restrict__ m1_in,
                                                           const float* __restrict__ m2_in,
                                                           const float* __restrict__ Kf, float* __restrict__ m1_out,
                                                           float* __restrict__ m2_out, const WaveParams P) {
  extern __shared__ __align__(16) float sm[];
  const int tx = blockIdx.x / P.tiles_y, ty = blockIdx.x % P.tiles_y;
  const int bx0 = tx * P.TBX, by0 = ty * P.TBY;
  const int H = P.k;
  const int rx0 = max(bx0 - H, 0), rx1 = min(bx0 + P.TBX + H, P.X);
  const int ry0 = max(by0 - H, 0), ry1 = min(by0 + P.TBY + H, P.Y);
  const int RX = rx1 - rx0, RY = ry1 - ry0;
  const int cap = P.RXM * P.RYM;
  float* M2 = sm;
  float* M1 = sm + cap;
  float* M0 = sm + 2 * cap;
  float* Kt = sm + 3 * cap;
  const int ly0 = threadIdx.x & 31, lx0 = threadIdx.x >> 5, nrows = blockDim.x >> 5;
  for (int lx = lx0; lx < RX; lx += nrows)
    for (int ly = ly0; ly < RY; ly += 32) {
      const size_t gi = (size_t)(rx0 + lx) * P.Y + ry0 + ly;
      const bool in = wave_inside(P, rx0 + lx, ry0 + ly);
      M2[lx * RY + ly] = in ? __ldg(m2_in + gi) : 0.0f;
      M1[lx * RY + ly] = in ? __ldg(m1_in + gi) : 0.0f;
      Kt[lx * RY + ly] = __ldg(Kf + gi);
    }
  __syncthreads();
  const int tw = min(P.TBX, P.X - bx0), th = min(P.TBY, P.Y - by0);
  // Each thread owns the same tile cells in every step: their running dJ/dK
  // stays in registers between steps (still one add per step, in step order).
  constexpr int GX = WAVE_TBX / 8, GY = WAVE_TBY / 32;
  float gk[GX][GY];
#pragma unroll
  for (int a = 0; a < GX; ++a)
#pragma unroll
    for (int b = 0; b < GY; ++b) {
      const int x = bx0 + lx0 + 8 * a, y = by0 + ly0 + 32 * b;
      gk[a][b] = (lx0 + 8 * a < tw && ly0 + 32 * b < th) ? P.gK[(size_t)x * P.Y + y] : 0.0f;
    }
  for (int s = 0; s < P.k; ++s) {
    const int n = P.ntop - s;
    // gradient term of step n on the tile: dJ/dK += mu^{n+1} o L(u^n)
    const float* un = P.ustates + (size_t)(n - P.ubase) * P.cells;
#pragma unroll
    for (int a = 0; a < GX; ++a)
#pragma unroll
      for (int b = 0; b < GY; ++b) {
        const int lx = lx0 + 8 * a, ly = ly0 + 32 * b;
        const int x = bx0 + lx, y = by0 + ly;
        if (lx >= tw || ly >= th || !wave_inside(P, x, y)) continue;
        const size_t gi = (size_t)x * P.Y + y;
        float acc = 0.0f;
        acc = add(acc, mul(P.w[0], __ldg(un + gi - P.Y)));
        acc = add(acc, mul(P.w[1], __ldg(un + gi)));
        acc = add(acc, mul(P.w[2], __ldg(un + gi + P.Y)));
        acc = add(acc, mul(P.w[0], __ldg(un + gi - 1)));
        acc = add(acc, mul(P.w[1], __ldg(un + gi)));
        acc = add(acc, mul(P.w[2], __ldg(un + gi + 1)));
        gk[a][b] = add(gk[a][b], mul(M1[(x - rx0) * RY + (y - ry0)], acc));
      }
    for (int lx = lx0; lx < RX; lx += nrows)
      for (int ly = ly0; ly < RY; ly += 32) {
        const int idx = lx * RY + ly;
        const int x = rx0 + lx, y = ry0 + ly;
        float v = 0.0f;
        if (wave_inside(P, x, y)) {
          if (lx >= 1 && lx < RX - 1 && ly >= 1 && ly < RY - 1) {
            // L(K o mu^{n+1}) with the products formed per neighbour
            const float kc = mul(Kt[idx], M1[idx]);
            float acc = 0.0f;
            acc = add(acc, mul(P.w[0], mul(Kt[idx - RY], M1[idx - RY])));
            acc = add(acc, mul(P.w[1], kc));
            acc = add(acc, mul(P.w[2], mul(Kt[idx + RY], M1[idx + RY])));
            acc = add(acc, mul(P.w[0], mul(Kt[idx - 1], M1[idx - 1])));
            acc = add(acc, mul(P.w[1], kc));
            acc = add(acc, mul(P.w[2], mul(Kt[idx + 1], M1[idx + 1])));
            v = add(sub(mul(2.0f, M1[idx]), M2[idx]), acc);
          } else {
            v = M1[idx];
          }
        }
        M0[idx] = v;
      }
    __syncthreads();
    float* t = M2;
    M2 = M1;
    M1 = M0;
    M0 = t;
  }
  for (int lx = lx0; lx < tw; lx += nrows)
    for (int ly = ly0; ly < th; ly += 32) {
      const size_t gi = (size_t)(bx0 + lx) * P.Y + by0 + ly;
      const int ri = (bx0 + lx - rx0) * RY + (by0 + ly - ry0);
      m1_out[gi] = M1[ri];
      m2_out[gi] = M2[ri];
    }
#pragma unroll
  for (int a = 0; a < GX; ++a)
#pragma unroll
    for (int b = 0; b < GY; ++b) {
      const int lx = lx0 + 8 * a, ly = ly0 + 32 * b;
      if (lx < tw && ly < th) P.gK[(size_t)(bx0 + lx) * P.Y + by0 + ly] = gk[a][b];
    }
}

}  // namespace pde
