// Weakly compressible flow, one RK2 (midpoint) step per launch (new: the
// reference composes the step from ~40 module launches, examples/LDC/LDC_RK2.py).
//
// Fields: momentum m (X, Y, 1, 2) and density rho (X, Y, 1, 1).  With the
// reference's operators (every product and sum rounded on its own, in their order):
//
//   bc(m, rho):  u = m / rho;  u = BC_u(u);  rho = BC_rho(rho);  m = rho * u
//   f(m, rho):   u = m / rho
//                m_div  = Div(m, -1)                        (divergence.py, vec -> scalar)
//                u_diff = Lap(u, nu)
//                u_conv = Div(outer(m, u), 1)               (elementWiseOps.py, divergence of a matrix)
//                u_damp = Lap(u_diff, eps)                  (biharmonic damping)
//                dp     = Grad(c2 * (rho - rho0), -1)
//                k_m    = ((dp - u_conv) + u_diff) + u_damp;  k_rho = m_div
//   step (time_step/rungeKatta.py:123-174):
//                y0 = bc(y);  y1 = bc(y0 + (dt/2) f(y0));  y' = y0 + dt f(y1)
//
// The operators' outputs are 0 outside the array interior (their launch domain),
// so f is 0 on ghost cells and y' keeps y0's boundary-filled ghosts there.
// A block owns a tile and works on the tile grown by 4 cells (clipped to the
// array) in shared memory: each f consumes 2 cells of the region's cut edges
// (Lap of Lap), the boundary fills read inward only, so the tile's result is exact.
#pragma once
#include "common.cuh"
#include "fused.cuh"

namespace pde {

struct WCParams {
  int X, Y, g;
  int TBX, TBY, tiles_y, RC;  // tile, tiles along Y, region capacity (cells)
  float wl[3];                // Laplacian weights (1, -2, 1) / dx^2
  float wd[3];                // first-derivative weights (-1, 0, 1) / (2 dx)
  float nu, eps, c2, rho0;
  float dt_half, dt;          // fp32 of dt/2 and of dt, each rounded from the caller's double
};

constexpr int WC_HALO = 4;

template <class F>
__device__ __forceinline__ void wc_region(int RC, int RY, F fn) {
  RectWalk wk(RY, (int)blockDim.x);
  for (int i = threadIdx.x; i < RC; i += blockDim.x, wk.next()) fn(i, wk.row, wk.col);
}

__global__ void __launch_bounds__(512) wc_rk2_kernel(const float* __restrict__ m_in, const float* __restrict__ r_in,
                                                     float* __restrict__ m_out, float* __restrict__ r_out,
                                                     const WCParams P, const PdeBCRules Ru, const PdeBCRules Rr) {
  extern __shared__ __align__(16) float sm[];
  const int X = P.X, Y = P.Y, g = P.g;
  const int tx = blockIdx.x / P.tiles_y, ty = blockIdx.x % P.tiles_y;
  const int bx0 = tx * P.TBX, by0 = ty * P.TBY;
  const int rx0 = max(bx0 - WC_HALO, 0), rx1 = min(bx0 + P.TBX + WC_HALO, X);
  const int ry0 = max(by0 - WC_HALO, 0), ry1 = min(by0 + P.TBY + WC_HALO, Y);
  const int RX = rx1 - rx0, RY = ry1 - ry0, RC = RX * RY;
  float* M0 = sm;             // y0: momentum (2 per cell), density
  float* R0 = M0 + 2 * P.RC;
  float* U = R0 + P.RC;       // velocity (2 per cell)
  float* D = U + 2 * P.RC;    // Lap(u, nu) (2 per cell)
  float* M1 = D + 2 * P.RC;   // y1
  float* R1 = M1 + 2 * P.RC;
  H2Params hp;                // the boundary fill reads the array shape and ghost width only
  hp.X = X;
  hp.Y = Y;
  hp.g = g;
  BcPlan<2> bp;               // one region for both fields and all four fills
  bc_plan(bp, hp, rx0, RX, ry0, RY);
  wc_region(RC, RY, [&](int i, int lx, int ly) {
    const size_t c = (size_t)(rx0 + lx) * Y + ry0 + ly;
    cp_async4(M0 + 2 * i, m_in + 2 * c, true);
    cp_async4(M0 + 2 * i + 1, m_in + 2 * c + 1, true);
    cp_async4(R0 + i, r_in + c, true);
  });
  cp_async_wait_all();
  __syncthreads();

  auto interior = [&](int lx, int ly) {
    const int x = rx0 + lx, y = ry0 + ly;
    return x >= g && x < X - g && y >= g && y < Y - g;
  };
  auto nbrs_in = [&](int lx, int ly) { return lx >= 1 && lx < RX - 1 && ly >= 1 && ly < RY - 1; };
  const float* wl = P.wl;
  const float* wd = P.wd;

  // bc(M, Rh) in place: u = m / rho, fill u and rho, m = rho * u
  auto bc = [&](float* M, float* Rh) {
    wc_region(RC, RY, [&](int i, int, int) {
      U[2 * i] = __fdiv_rn(M[2 * i], Rh[i]);
      U[2 * i + 1] = __fdiv_rn(M[2 * i + 1], Rh[i]);
    });
    __syncthreads();
    bc_fill_planned<2, 2>(U, bp, hp, Ru, rx0, RX, ry0, RY, Ru.dx32);
    bc_fill_planned<1, 1>(Rh, bp, hp, Rr, rx0, RX, ry0, RY, Rr.dx32);
    __syncthreads();
    wc_region(RC, RY, [&](int i, int, int) {
      M[2 * i] = mul(Rh[i], U[2 * i]);
      M[2 * i + 1] = mul(Rh[i], U[2 * i + 1]);
    });
    __syncthreads();
  };
  // u = m / rho and D = Lap(u, nu) for the f of (M, Rh)
  auto prep_f = [&](const float* M, const float* Rh) {
    wc_region(RC, RY, [&](int i, int, int) {
      U[2 * i] = __fdiv_rn(M[2 * i], Rh[i]);
      U[2 * i + 1] = __fdiv_rn(M[2 * i + 1], Rh[i]);
    });
    __syncthreads();
    wc_region(RC, RY, [&](int i, int lx, int ly) {
      float d0 = 0.0f, d1 = 0.0f;
      if (interior(lx, ly) && nbrs_in(lx, ly)) {
#pragma unroll
        for (int v = 0; v < 2; ++v) {
          float acc = 0.0f;
          acc = add(acc, mul(wl[0], U[2 * (i - RY) + v]));
          acc = add(acc, mul(wl[1], U[2 * i + v]));
          acc = add(acc, mul(wl[2], U[2 * (i + RY) + v]));
          acc = add(acc, mul(wl[0], U[2 * (i - 1) + v]));
          acc = add(acc, mul(wl[1], U[2 * i + v]));
          acc = add(acc, mul(wl[2], U[2 * (i + 1) + v]));
          if (v == 0) d0 = mul(P.nu, acc);
          else d1 = mul(P.nu, acc);
        }
      }
      D[2 * i] = d0;
      D[2 * i + 1] = d1;
    });
    __syncthreads();
  };
  // f at region cell i of (M, Rh) (u, D prepared): k = (k_m0, k_m1, k_rho)
  auto f_at = [&](const float* M, const float* Rh, int i, float& k0, float& k1, float& kr) {
    const int off[2] = {RY, 1};  // neighbour offsets along x, y
    // m_div = Div(m, -1): one sum over axes and taps
    float acc = 0.0f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int t = 0; t < 3; ++t) acc = add(acc, mul(wd[t], M[2 * (i + (t - 1) * off[a]) + a]));
    kr = mul(-1.0f, acc);
    float kv[2];
#pragma unroll
    for (int v = 0; v < 2; ++v) {
      // u_conv[v] = Div(outer(m, u))[v]: sum over axes a, taps of w * (m_v u_a)
      float conv = 0.0f;
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int t = 0; t < 3; ++t) {
          const int j = i + (t - 1) * off[a];
          conv = add(conv, mul(wd[t], mul(M[2 * j + v], U[2 * j + a])));
        }
      conv = mul(1.0f, conv);
      // u_damp[v] = Lap(u_diff, eps)
      float lap = 0.0f;
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int t = 0; t < 3; ++t) lap = add(lap, mul(wl[t], D[2 * (i + (t - 1) * off[a]) + v]));
      const float damp = mul(P.eps, lap);
      // dp[v] = Grad(c2 * (rho - rho0), -1) along axis v
      float gp = 0.0f;
#pragma unroll
      for (int t = 0; t < 3; ++t)
        gp = add(gp, mul(wd[t], mul(P.c2, sub(Rh[i + (t - 1) * off[v]], P.rho0))));
      const float dp = mul(-1.0f, gp);
      kv[v] = add(add(sub(dp, conv), D[2 * i + v]), damp);
    }
    k0 = kv[0];
    k1 = kv[1];
  };

  // ---- stage 1: y0 = bc(y); y1 = y0 + dt/2 f(y0) ----
  bc(M0, R0);
  prep_f(M0, R0);
  wc_region(RC, RY, [&](int i, int lx, int ly) {
    float k0 = 0.0f, k1 = 0.0f, kr = 0.0f;
    if (interior(lx, ly) && nbrs_in(lx, ly)) f_at(M0, R0, i, k0, k1, kr);
    M1[2 * i] = add(M0[2 * i], mul(P.dt_half, k0));
    M1[2 * i + 1] = add(M0[2 * i + 1], mul(P.dt_half, k1));
    R1[i] = add(R0[i], mul(P.dt_half, kr));
  });
  __syncthreads();
  // ---- stage 2: y' = y0 + dt f(bc(y1)) on the tile ----
  bc(M1, R1);
  prep_f(M1, R1);
  const int ox1 = min(bx0 + P.TBX, X), oy1 = min(by0 + P.TBY, Y);
  const int OY = oy1 - by0, OC = (ox1 - bx0) * OY;
  RectWalk wo(OY, (int)blockDim.x);
  for (int o = threadIdx.x; o < OC; o += blockDim.x, wo.next()) {
    const int lx = bx0 - rx0 + wo.row, ly = by0 - ry0 + wo.col;
    const int i = lx * RY + ly;
    float k0 = 0.0f, k1 = 0.0f, kr = 0.0f;
    if (interior(lx, ly)) f_at(M1, R1, i, k0, k1, kr);  // tile cells are 4 cells from any cut
    const size_t c = (size_t)(bx0 + wo.row) * Y + by0 + wo.col;
    m_out[2 * c] = add(M0[2 * i], mul(P.dt, k0));
    m_out[2 * c + 1] = add(M0[2 * i + 1], mul(P.dt, k1));
    r_out[c] = add(R0[i], mul(P.dt, kr));
  }
}

}  // namespace pde
