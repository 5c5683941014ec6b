// Fractional-step (projection) solver for the 2D lid-driven cavity, composed
// from the operators of the reference's LDC examples (examples/LDC/*.py:
// GridBoundary, Laplacian, Grad, Divergence, ForwardEuler) with a Jacobi
// pressure-Poisson sweep, which the reference does not have (it uses
// artificial compressibility).  Each kernel evaluates exactly the float32
// operations of that module composition, one rounding per product and sum:
//
//   u2   = BC_u(u)
//   u*   = u2 + dt * (nu*Lap(u2) - Grad(u2) u2)        (predictor)
//   rhs  = (1/dt) * Div(BC_u(u*))                        (divergence)
//   p    <- 0.25 * (pW + pE + pS + pN - dx^2 * rhs)      (Jacobi, p_bc = BC_p(p)), 50 sweeps
//   u    = BC_u(u*) + dt * (-Grad(BC_p(p)))              (projection)
#pragma once
#include "common.cuh"
#include "fused.cuh"

namespace pde {

struct LdcConst {
  float wl[3];    // Laplacian weights
  float wd[3];    // first-derivative weights
  float nu, dt, inv_dt, h2;
};

// Predictor: thread per cell of the whole (X, Y, 1, 2) array.
__global__ void __launch_bounds__(256) ldc_predictor_kernel(const float* __restrict__ u, float* __restrict__ us,
                                                             Geo G, const PdeBCRules Ru, LdcConst K) {
  const int64_t total = G.n[0] * G.n[1];
  GlobalAcc U{u, G.cstride[0], G.cstride[1], 2};
  for (int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; cell < total;
       cell += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = cell / G.n[1], j = cell - i * G.n[1];
    const float a0 = bc_eval2d(G, Ru, U, i, j, 0), a1 = bc_eval2d(G, Ru, U, i, j, 1);
    const bool st = i >= G.g && i < G.n[0] - G.g && j >= G.g && j < G.n[1] - G.g;
    if (!st) {
      us[cell * 2 + 0] = a0;
      us[cell * 2 + 1] = a1;
      continue;
    }
    float nb[2][2][3];  // [axis][comp][tap]
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      nb[0][c][1] = c == 0 ? a0 : a1;
      nb[1][c][1] = nb[0][c][1];
      nb[0][c][0] = bc_eval2d(G, Ru, U, i - 1, j, c);
      nb[0][c][2] = bc_eval2d(G, Ru, U, i + 1, j, c);
      nb[1][c][0] = bc_eval2d(G, Ru, U, i, j - 1, c);
      nb[1][c][2] = bc_eval2d(G, Ru, U, i, j + 1, c);
    }
    const float uc[2] = {a0, a1};
    float res[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      float acc = 0.0f;  // Laplacian, FDM/kernel/laplacian.py:40-46 order
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int t = 0; t < 3; ++t) acc = add(acc, mul(K.wl[t], nb[a][c][t]));
      const float lap = mul(K.nu, acc);
      float gr[2];  // Grad(u2, 1.0): row c of the 2x2 matrix
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        float g = 0.0f;
#pragma unroll
        for (int t = 0; t < 3; ++t) g = add(g, mul(K.wd[t], nb[a][c][t]));
        gr[a] = mul(1.0f, g);
      }
      const float conv = add(mul(gr[0], uc[0]), mul(gr[1], uc[1]));
      res[c] = add(uc[c], mul(K.dt, sub(lap, conv)));
    }
    us[cell * 2 + 0] = res[0];
    us[cell * 2 + 1] = res[1];
  }
}

// rhs = (1/dt) * Div(BC_u(u*)) on stencil cells (ghosts of rhs are never read).
__global__ void __launch_bounds__(256) ldc_divergence_kernel(const float* __restrict__ us, float* __restrict__ rhs,
                                                              Geo G, const PdeBCRules Ru, LdcConst K) {
  const int64_t total = G.n[0] * G.n[1];
  GlobalAcc U{us, G.cstride[0], G.cstride[1], 2};
  for (int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; cell < total;
       cell += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = cell / G.n[1], j = cell - i * G.n[1];
    const bool st = i >= G.g && i < G.n[0] - G.g && j >= G.g && j < G.n[1] - G.g;
    if (!st) {
      rhs[cell] = 0.0f;
      continue;
    }
    float acc = 0.0f;  // FDM/kernel/divergence.py:85-106: axis 0 on component 0, axis 1 on component 1
#pragma unroll
    for (int t = 0; t < 3; ++t) acc = add(acc, mul(K.wd[t], bc_eval2d(G, Ru, U, i + t - 1, j, 0)));
#pragma unroll
    for (int t = 0; t < 3; ++t) acc = add(acc, mul(K.wd[t], bc_eval2d(G, Ru, U, i, j + t - 1, 1)));
    rhs[cell] = mul(K.inv_dt, acc);
  }
}

// u = BC_u(u*) + dt * Grad(BC_p(p), -1)
__global__ void __launch_bounds__(256) ldc_project_kernel(const float* __restrict__ us, const float* __restrict__ p,
                                                           float* __restrict__ u, Geo G, const PdeBCRules Ru,
                                                           const PdeBCRules Rp, LdcConst K) {
  const int64_t total = G.n[0] * G.n[1];
  GlobalAcc U{us, G.cstride[0], G.cstride[1], 2};
  GlobalAcc Pa{p, G.cstride[0], G.cstride[1], 1};
  for (int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; cell < total;
       cell += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = cell / G.n[1], j = cell - i * G.n[1];
    const float a0 = bc_eval2d(G, Ru, U, i, j, 0), a1 = bc_eval2d(G, Ru, U, i, j, 1);
    const bool st = i >= G.g && i < G.n[0] - G.g && j >= G.g && j < G.n[1] - G.g;
    if (!st) {
      u[cell * 2 + 0] = a0;
      u[cell * 2 + 1] = a1;
      continue;
    }
    float gx = 0.0f, gy = 0.0f;
#pragma unroll
    for (int t = 0; t < 3; ++t) gx = add(gx, mul(K.wd[t], bc_eval2d(G, Rp, Pa, i + t - 1, j, 0)));
#pragma unroll
    for (int t = 0; t < 3; ++t) gy = add(gy, mul(K.wd[t], bc_eval2d(G, Rp, Pa, i, j + t - 1, 0)));
    u[cell * 2 + 0] = add(a0, mul(K.dt, mul(-1.0f, gx)));
    u[cell * 2 + 1] = add(a1, mul(K.dt, mul(-1.0f, gy)));
  }
}

// k Jacobi sweeps per pass on shared-memory tiles (halo k + 1, as in
// heat2d_tb_kernel), Neumann ghosts refilled in shared memory every sweep.
// On the pass's last sweep the squared update of the tile's stencil cells is
// reduced (warp shuffles, then one atomic per block) into *resid.
struct J2Params {
  int X, Y, g;
  int k;
  int TBX, TBY, tiles_y;
  int RXM, RYM;
  float h2;
  int last;  // this pass ends the step's sweeps: accumulate the residual
};

__global__ void __launch_bounds__(256) jacobi2d_tb_kernel(const float* __restrict__ pin, float* __restrict__ pout,
                                                           const float* __restrict__ rhs, float* __restrict__ resid,
                                                           const J2Params P, const PdeBCRules Rp) {
  extern __shared__ __align__(16) float sm[];
  const int tx = blockIdx.x / P.tiles_y, ty = blockIdx.x % P.tiles_y;
  const int bx0 = tx * P.TBX, by0 = ty * P.TBY;
  const int H = P.k + 1;
  const int rx0 = max(bx0 - H, 0), rx1 = min(bx0 + P.TBX + H, P.X);
  const int ry0 = max(by0 - H, 0), ry1 = min(by0 + P.TBY + H, P.Y);
  const int RX = rx1 - rx0, RY = ry1 - ry0;
  float* A = sm;
  float* B = sm + P.RXM * P.RYM;
  float* Rh = sm + 2 * P.RXM * P.RYM;
  // 2D thread layout: 32 lanes along y (contiguous), blockDim.x / 32 rows along x
  const int ly0 = threadIdx.x & 31, lx0 = threadIdx.x >> 5, nrows = blockDim.x >> 5;
  for (int lx = lx0; lx < RX; lx += nrows)
    for (int ly = ly0; ly < RY; ly += 32) {
      const size_t gi = (size_t)(rx0 + lx) * P.Y + ry0 + ly;
      A[lx * RY + ly] = __ldg(pin + gi);
      Rh[lx * RY + ly] = __ldg(rhs + gi);
    }
  __syncthreads();
  H2Params HP;
  HP.X = P.X; HP.Y = P.Y; HP.g = P.g; HP.N = 1;
  const int g = P.g;
  // stencil cells of the region whose four neighbours are inside it
  const int sx0 = max(g, rx0 + 1) - rx0, sx1 = min(P.X - g, rx0 + RX - 1) - rx0;
  const int sy0 = max(g, ry0 + 1) - ry0, sy1 = min(P.Y - g, ry0 + RY - 1) - ry0;
  float sq = 0.0f;
  for (int s = 0; s < P.k; ++s) {
    bc_fill_region<1>(A, HP, Rp, rx0, RX, ry0, RY, Rp.dx32);
    const bool acc_res = P.last && s == P.k - 1;
    for (int lx = lx0; lx < RX; lx += nrows)
      for (int ly = ly0; ly < RY; ly += 32) {
        const int idx = lx * RY + ly;
        const float c = A[idx];
        float res = c;
        if (lx >= sx0 && lx < sx1 && ly >= sy0 && ly < sy1) {
          const float sum = add(add(add(A[idx - RY], A[idx + RY]), A[idx - 1]), A[idx + 1]);
          res = mul(0.25f, sub(sum, mul(P.h2, Rh[idx])));
          const int x = rx0 + lx, y = ry0 + ly;
          if (acc_res && x >= bx0 && x < bx0 + P.TBX && y >= by0 && y < by0 + P.TBY) {
            const float d = res - c;
            sq = fmaf(d, d, sq);
          }
        }
        B[idx] = res;
      }
    __syncthreads();
    float* t = A;
    A = B;
    B = t;
  }
  const int ox1 = min(bx0 + P.TBX, P.X), oy1 = min(by0 + P.TBY, P.Y);
  for (int lx = lx0; lx < ox1 - bx0; lx += nrows)
    for (int ly = ly0; ly < oy1 - by0; ly += 32)
      pout[(size_t)(bx0 + lx) * P.Y + by0 + ly] = A[(bx0 + lx - rx0) * RY + (by0 + ly - ry0)];
  if (P.last && resid) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    __shared__ float wsum[8];
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
      float b = 0.0f;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += wsum[w];
      atomicAdd(resid, b);
    }
  }
}

}  // namespace pde
