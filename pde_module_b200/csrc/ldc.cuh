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
#include <type_traits>

#include "common.cuh"
#include "fused.cuh"

namespace pde {

struct LdcConst {
  float wl[3];    // Laplacian weights
  float wd[3];    // first-derivative weights
  float nu, dt, inv_dt, h2;
};

// The three pointwise kernels run one thread per cell on a 2D grid (row =
// row0 + blockIdx.y; a slab of a larger domain passes its first owned row and
// pointers shifted so that global row indices address its local rows).  A cell whose neighbours are all at least one cell inside the
// node ring ("deep": x, y in [g+2, n-g-3]) reads raw values; the others go
// through bc_eval2d, which returns the boundary-filled value of any cell.
__device__ __forceinline__ bool ldc_deep(const Geo& G, int i, int j) {
  return i >= G.g + 2 && i < (int)G.n[0] - G.g - 2 && j >= G.g + 2 && j < (int)G.n[1] - G.g - 2;
}
__device__ __forceinline__ bool ldc_stencil(const Geo& G, int i, int j) {
  return i >= G.g && i < (int)G.n[0] - G.g && j >= G.g && j < (int)G.n[1] - G.g;
}

// Raw 2D access (ncomp N) with 32-bit cell indices.
template <int N>
struct Raw2 {
  const float* u;
  int n1;
  __device__ __forceinline__ float operator()(int i, int j, int v) const { return __ldg(u + (i * n1 + j) * N + v); }
};
// Boundary-filled access.
struct Bc2 {
  const Geo& G;
  const PdeBCRules& R;
  const GlobalAcc& U;
  __device__ __forceinline__ float operator()(int i, int j, int v) const { return bc_eval2d(G, R, U, i, j, v); }
};

// Predictor of one stencil cell: u* = u2 + dt * (nu*Lap(u2) - Grad(u2) u2), with u2 = BC_u(u).
template <class Get>
__device__ __forceinline__ void ldc_predict_cell(const Get& at, int i, int j, const LdcConst& K, float* res) {
  const float uc[2] = {at(i, j, 0), at(i, j, 1)};
  float nb[2][2][3];  // [axis][comp][tap]
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    nb[0][c][1] = uc[c];
    nb[1][c][1] = uc[c];
    nb[0][c][0] = at(i - 1, j, c);
    nb[0][c][2] = at(i + 1, j, c);
    nb[1][c][0] = at(i, j - 1, c);
    nb[1][c][2] = at(i, j + 1, c);
  }
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
}

__global__ void __launch_bounds__(256) ldc_predictor_kernel(const float* __restrict__ u, float* __restrict__ us,
                                                             Geo G, const PdeBCRules Ru, LdcConst K, int row0) {
  const int i = row0 + (int)blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (int)G.n[1]) return;
  const int n1 = (int)G.n[1];
  const int cell = i * n1 + j;
  GlobalAcc U{u, G.cstride[0], G.cstride[1], 2};
  if (!ldc_stencil(G, i, j)) {
    us[cell * 2 + 0] = bc_eval2d(G, Ru, U, i, j, 0);
    us[cell * 2 + 1] = bc_eval2d(G, Ru, U, i, j, 1);
    return;
  }
  float res[2];
  if (ldc_deep(G, i, j)) ldc_predict_cell(Raw2<2>{u, n1}, i, j, K, res);
  else ldc_predict_cell(Bc2{G, Ru, U}, i, j, K, res);
  us[cell * 2 + 0] = res[0];
  us[cell * 2 + 1] = res[1];
}

// rhs = (1/dt) * Div(BC_u(u*)) on stencil cells (ghosts of rhs are never read).
template <class Get>
__device__ __forceinline__ float ldc_div_cell(const Get& at, int i, int j, const LdcConst& K) {
  float acc = 0.0f;  // FDM/kernel/divergence.py:85-106: axis 0 on component 0, axis 1 on component 1
#pragma unroll
  for (int t = 0; t < 3; ++t) acc = add(acc, mul(K.wd[t], at(i + t - 1, j, 0)));
#pragma unroll
  for (int t = 0; t < 3; ++t) acc = add(acc, mul(K.wd[t], at(i, j + t - 1, 1)));
  return mul(K.inv_dt, acc);
}

__global__ void __launch_bounds__(256) ldc_divergence_kernel(const float* __restrict__ us, float* __restrict__ rhs,
                                                              Geo G, const PdeBCRules Ru, LdcConst K, int row0) {
  const int i = row0 + (int)blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (int)G.n[1]) return;
  const int n1 = (int)G.n[1];
  const int cell = i * n1 + j;
  if (!ldc_stencil(G, i, j)) {
    rhs[cell] = 0.0f;
    return;
  }
  GlobalAcc U{us, G.cstride[0], G.cstride[1], 2};
  rhs[cell] = ldc_deep(G, i, j) ? ldc_div_cell(Raw2<2>{us, n1}, i, j, K) : ldc_div_cell(Bc2{G, Ru, U}, i, j, K);
}

// u = BC_u(u*) + dt * Grad(BC_p(p), -1)
template <class GetU, class GetP>
__device__ __forceinline__ void ldc_project_cell(const GetU& au, const GetP& ap, int i, int j, const LdcConst& K,
                                                 float* res) {
  const float a0 = au(i, j, 0), a1 = au(i, j, 1);
  float gx = 0.0f, gy = 0.0f;
#pragma unroll
  for (int t = 0; t < 3; ++t) gx = add(gx, mul(K.wd[t], ap(i + t - 1, j, 0)));
#pragma unroll
  for (int t = 0; t < 3; ++t) gy = add(gy, mul(K.wd[t], ap(i, j + t - 1, 0)));
  res[0] = add(a0, mul(K.dt, mul(-1.0f, gx)));
  res[1] = add(a1, mul(K.dt, mul(-1.0f, gy)));
}

__global__ void __launch_bounds__(256) ldc_project_kernel(const float* __restrict__ us, const float* __restrict__ p,
                                                           float* __restrict__ u, Geo G, const PdeBCRules Ru,
                                                           const PdeBCRules Rp, LdcConst K, int row0) {
  const int i = row0 + (int)blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (int)G.n[1]) return;
  const int n1 = (int)G.n[1];
  const int cell = i * n1 + j;
  GlobalAcc U{us, G.cstride[0], G.cstride[1], 2};
  GlobalAcc Pa{p, G.cstride[0], G.cstride[1], 1};
  if (!ldc_stencil(G, i, j)) {
    u[cell * 2 + 0] = bc_eval2d(G, Ru, U, i, j, 0);
    u[cell * 2 + 1] = bc_eval2d(G, Ru, U, i, j, 1);
    return;
  }
  float res[2];
  if (ldc_deep(G, i, j)) ldc_project_cell(Raw2<2>{us, n1}, Raw2<1>{p, n1}, i, j, K, res);
  else ldc_project_cell(Bc2{G, Ru, U}, Bc2{G, Rp, Pa}, i, j, K, res);
  u[cell * 2 + 0] = res[0];
  u[cell * 2 + 1] = res[1];
}

// k Jacobi sweeps per pass on shared-memory tiles (halo k + 1, as in
// heat2d_tb_kernel), Neumann ghosts refilled in shared memory every sweep.
// On the pass's last sweep the squared update of the tile's stencil cells is
// reduced (warp shuffles, then one atomic per block) into *resid.
struct J2Params {
  int X, Y, g;            // X: rows of the whole domain (a slab's arrays are addressed by global row)
  int own_lo, own_hi;     // rows whose results this launch writes
  int held_lo, held_hi;   // rows the arrays hold (owned rows plus halo rows on a slab's cut sides)
  int k;
  int TBX, TBY, tiles_y;
  int RXM, RYM;
  float h2;
  int last;  // this pass ends the step's sweeps: accumulate the residual
};

__global__ void __launch_bounds__(1024) jacobi2d_tb_kernel(const float* __restrict__ pin, float* __restrict__ pout,
                                                           const float* __restrict__ rhs, float* __restrict__ resid,
                                                           const J2Params P, const PdeBCRules Rp) {
  extern __shared__ __align__(16) float sm[];
  const int tx = blockIdx.x / P.tiles_y, ty = blockIdx.x % P.tiles_y;
  const int bx0 = P.own_lo + tx * P.TBX, by0 = ty * P.TBY;
  const int H = P.k + 1;
  const int rx0 = max(bx0 - H, P.held_lo), rx1 = min(bx0 + P.TBX + H, P.held_hi);
  const int ry0 = max(by0 - H, 0), ry1 = min(by0 + P.TBY + H, P.Y);
  const int RX = rx1 - rx0, RY = ry1 - ry0, RC = RX * RY;
  const int cap = P.RXM * P.RYM;
  float* A = sm;
  float* B = sm + cap;
  float* Rh = sm + 2 * cap;
  const int nt = (int)blockDim.x;
  // Both level buffers start with the region (cp.async, every copy of a thread
  // in flight at once); a sweep writes only its stencil rectangle, so the other
  // cells keep their loaded or last boundary-filled value.
  {
    RectWalk wk(RY, nt);
    for (int i = threadIdx.x; i < RC; i += nt, wk.next()) {
      const size_t gi = (size_t)(rx0 + wk.row) * P.Y + ry0 + wk.col;
      cp_async4(A + i, pin + gi, true);
      cp_async4(B + i, pin + gi, true);
      cp_async4(Rh + i, rhs + gi, true);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  H2Params HP;
  HP.X = P.X; HP.Y = P.Y; HP.g = P.g; HP.N = 1;
  const int g = P.g;
  // stencil rectangle: cells of [g, n-g) whose four neighbours are inside the region
  const int sx0 = max(g, rx0 + 1) - rx0, sx1 = min(P.X - g, rx0 + RX - 1) - rx0;
  const int sy0 = max(g, ry0 + 1) - ry0, sy1 = min(P.Y - g, ry0 + RY - 1) - ry0;
  const int tw = min(bx0 + P.TBX, P.own_hi) - bx0, th = min(by0 + P.TBY, P.Y) - by0;
  float sq = 0.0f;
  for (int s = 0; s < P.k; ++s) {
    bc_fill_region<1>(A, HP, Rp, rx0, RX, ry0, RY, Rp.dx32);
    const bool acc_res = P.last && s == P.k - 1;
    // Sweep s only has to update the stencil cells within (k - 1 - s) + 1 of the
    // tile (the boundary fills read inward): the stencil rectangle cut to that box.
    const int reach = P.k - s;
    const int qx0 = max(sx0, bx0 - rx0 - reach), qx1 = min(sx1, bx0 - rx0 + tw + reach);
    const int qy0 = max(sy0, by0 - ry0 - reach), qy1 = min(sy1, by0 - ry0 + th + reach);
    const int SW = max(qy1 - qy0, 1), SC = max(qx1 - qx0, 0) * max(qy1 - qy0, 0);
    const int dq = nt / SW, dr = nt - dq * SW;
    // the tile in box coordinates (residual cells)
    const int tx0 = bx0 - rx0 - qx0, ty0 = by0 - ry0 - qy0;
    int lx = (int)threadIdx.x / SW, ly = (int)threadIdx.x - lx * SW;
    for (int c = threadIdx.x; c < SC; c += nt) {
      const int i = (qx0 + lx) * RY + qy0 + ly;
      const float old = A[i];
      const float sum = add(add(add(A[i - RY], A[i + RY]), A[i - 1]), A[i + 1]);
      const float res = mul(0.25f, sub(sum, mul(P.h2, Rh[i])));
      B[i] = res;
      if (acc_res) {
        const int ox = lx - tx0, oy = ly - ty0;
        if (ox >= 0 && ox < tw && oy >= 0 && oy < th) {
          const float d = res - old;
          sq = fmaf(d, d, sq);
        }
      }
      lx += dq;
      ly += dr;
      if (ly >= SW) { ly -= SW; ++lx; }
    }
    __syncthreads();
    float* t = A;
    A = B;
    B = t;
  }
  // output: stencil cells from the newest level, the others as last filled (B)
  RectWalk wo(th, nt);
  for (int i = threadIdx.x; i < tw * th; i += nt, wo.next()) {
    const int x = bx0 + wo.row, y = by0 + wo.col;
    const int ri = (x - rx0) * RY + (y - ry0);
    const bool st = x >= g && x < P.X - g && y >= g && y < P.Y - g;
    pout[(size_t)x * P.Y + y] = st ? A[ri] : B[ri];  // (equal when k = 0: both hold the loaded values)
  }
  if (P.last && resid) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    __shared__ float wsum[32];
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
      float b = 0.0f;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += wsum[w];
      atomicAdd(resid, b);
    }
  }
}

// The same passes with register cell lists (as the wave kernels): the region's
// cells interleave the two levels and the right-hand side (3 floats per cell, an
// odd stride: no bank conflicts), each thread's stencil cells are fixed for the
// pass (slots q = threadIdx.x + c * blockDim.x over the stencil rectangle's rows
// at full region width, the columns outside the rectangle idle), with their
// region index and distance from the tile (one packed word: index in the low 16
// bits, regions hold fewer than 2^16 cells) and h^2 rhs in registers (h^2 rhs is
// the same product every sweep).  Sweep s reads level s & 1 and writes the other;
// two sweeps per loop iteration make the levels compile-time offsets.  Same
// arithmetic and order per cell as jacobi2d_tb_kernel; needs the rectangle's
// rows x RY <= MAXC * blockDim.x.
template <int MAXC>
__global__ void __launch_bounds__(1024) jacobi2d_cells_kernel(const float* __restrict__ pin,
                                                              float* __restrict__ pout,
                                                              const float* __restrict__ rhs,
                                                              float* __restrict__ resid, const J2Params P,
                                                              const PdeBCRules Rp) {
  pdl_launch_dependents();  // the next pass may be scheduled; it waits for this one
  extern __shared__ __align__(16) float sm[];
  constexpr int NB = 3;  // per region cell: level 0, level 1, rhs
  const int tx = blockIdx.x / P.tiles_y, ty = blockIdx.x % P.tiles_y;
  const int bx0 = P.own_lo + tx * P.TBX, by0 = ty * P.TBY;
  const int H = P.k + 1;
  const int rx0 = max(bx0 - H, P.held_lo), rx1 = min(bx0 + P.TBX + H, P.held_hi);
  const int ry0 = max(by0 - H, 0), ry1 = min(by0 + P.TBY + H, P.Y);
  const int RX = rx1 - rx0, RY = ry1 - ry0, RC = RX * RY;
  const int nt = (int)blockDim.x;
  H2Params HP;
  HP.X = P.X; HP.Y = P.Y; HP.g = P.g; HP.N = 1;
  const int g = P.g;
  // stencil rectangle: cells of [g, n-g) whose four neighbours are inside the region
  const int sx0 = max(g, rx0 + 1) - rx0, sx1 = min(P.X - g, rx0 + RX - 1) - rx0;
  const int sy0 = max(g, ry0 + 1) - ry0, sy1 = min(P.Y - g, ry0 + RY - 1) - ry0;
  const int tw = min(bx0 + P.TBX, P.own_hi) - bx0, th = min(by0 + P.TBY, P.Y) - by0;
  const int tlx = bx0 - rx0, tly = by0 - ry0;  // the tile's origin in the region
  int key[MAXC];  // region index | distance from the tile << 16; idle slots: INT_MAX
  float hr[MAXC];
  unsigned tile = 0;  // bit c: slot c holds a tile cell (residual)
  {
    const int n = max(sx1 - sx0, 0) * RY;
    RectWalk wk(RY, nt);
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      key[c] = 0x7fffffff;
      if ((int)threadIdx.x + c * nt < n && wk.col >= sy0 && wk.col < sy1) {
        const int lx = sx0 + wk.row, ly = wk.col;
        const int ox = lx - tlx, oy = ly - tly;
        const int d = max(max(max(-ox, ox - (tw - 1)), max(-oy, oy - (th - 1))), 0);
        key[c] = (lx * RY + ly) | (d << 16);
        if (ox >= 0 && ox < tw && oy >= 0 && oy < th) tile |= 1u << c;
      }
      wk.next();
    }
  }
  const int rs = NB * RY;
  float sq = 0.0f;
  BcPlan<1> bp;
  bc_plan(bp, HP, rx0, RX, ry0, RY);
  pdl_wait();  // the previous pass's pressure (this pass's input) is complete
  {
    RectWalk wk(RY, nt);
    for (int i = threadIdx.x; i < RC; i += nt, wk.next()) {
      const size_t gi = (size_t)(rx0 + wk.row) * P.Y + ry0 + wk.col;
      cp_async4(sm + NB * i, pin + gi, true);
      cp_async4(sm + NB * i + 1, pin + gi, true);
      cp_async4(sm + NB * i + 2, rhs + gi, true);
    }
  }
  cp_async_wait_all();
  __syncthreads();
#pragma unroll
  for (int c = 0; c < MAXC; ++c)  // h^2 rhs of the thread's cells (the same product every sweep)
    hr[c] = key[c] != 0x7fffffff ? mul(P.h2, sm[NB * (key[c] & 0xffff) + 2]) : 0.0f;
  // Sweep s only has to update the stencil cells within (k - 1 - s) + 1 of the
  // tile (the boundary fills read inward): those with dist <= k - s.
  auto sweep = [&](auto PAR, int s) {
    constexpr int p = decltype(PAR)::value;  // reads level p, writes level 1 - p
    bc_fill_planned<1, NB>(sm + p, bp, HP, Rp, rx0, RX, ry0, RY, Rp.dx32);
    const bool acc_res = P.last && s == P.k - 1;
    const int lim = (P.k - s + 1) << 16;  // dist <= k - s  <=>  key < lim
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      if (key[c] >= lim) continue;
      float* pc = sm + NB * (key[c] & 0xffff);
      const float sum = add(add(add(pc[p - rs], pc[p + rs]), pc[p - NB]), pc[p + NB]);
      const float res = mul(0.25f, sub(sum, hr[c]));
      if (acc_res && ((tile >> c) & 1u)) {
        const float d = res - pc[p];
        sq = fmaf(d, d, sq);
      }
      pc[1 - p] = res;
    }
    __syncthreads();
  };
  for (int s = 0; s < P.k; s += 2) {
    sweep(std::integral_constant<int, 0>{}, s);
    if (s + 1 < P.k) sweep(std::integral_constant<int, 1>{}, s + 1);
  }
  // output: stencil cells from the newest level, the others as last filled
  const int nw = P.k & 1;  // the level the last sweep wrote
  RectWalk wo(th, nt);
  for (int i = threadIdx.x; i < tw * th; i += nt, wo.next()) {
    const int x = bx0 + wo.row, y = by0 + wo.col;
    const int r = (x - rx0) * RY + (y - ry0);
    const bool st = x >= g && x < P.X - g && y >= g && y < P.Y - g;
    pout[(size_t)x * P.Y + y] = sm[NB * r + (st ? nw : 1 - nw)];
  }
  if (P.last && resid) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    __shared__ float wsum[32];
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
