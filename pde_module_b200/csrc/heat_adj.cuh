// Differentiable 2D heat rollout: forward with a per-cell diffusivity field and
// its discrete adjoint.  New: the reference has the forward loop only
// (examples/2D_Heat_Equation.py:57-65, scalar alpha).
//
// Forward step (scalar field, one component), as heat2d_tb_kernel with alpha
// taken per cell:
//   v = B(u^n)                          boundary fill (GridBoundary semantics)
//   S^n = L(v)   on stencil cells       the reference's Laplacian sum, alpha 1
//   u^{n+1} = v + dt * (alpha o S^n)    stencil cells;  v elsewhere
// With a constant field the result is bit-identical to pde_heat_rollout.
//
// Adjoint of one step, lam = dJ/du^{n+1} -> dJ/du^n (every product and sum
// rounded on its own, in the order written):
//   dJ/dalpha_c += lam_c * (dt * S^n_c)           stencil cells, n = N-1 .. 0
//   z   = dt * (alpha o lam)                      stencil cells, 0 elsewhere
//   mu  = lam + L^T(z)                            L^T = L (symmetric weights),
//                                                 neighbours outside the array 0
//   lam = B^T(mu):  (cell overwritten by B ? 0 : mu_j)
//                   then -/+ mu_G for each filled ghost G whose partner is j
//                   (Dirichlet ghost = 2 val - u_j: -1; Neumann = c + u_j: +1),
//                   in the order x-low, x-high, y-low, y-high ghost.
// A ghost's partner is two cells inward (the cell across its node).
//
// Temporal blocking as in heat2d_tb_kernel: k steps per pass on shared-memory
// regions (tile + halo).  Adjoint halo: k*R; cut edges move R cells per step;
// a region edge that would fall within g+2 cells of the array edge is moved to
// the array edge, so no ghost/partner pair straddles a cut.
#pragma once
#include "common.cuh"
#include "fused.cuh"

namespace pde {

struct HAParams {
  int X, Y, g;
  int k;               // steps in this pass
  int TBX, TBY, tiles_y;
  int RC;              // region capacity (cells)
  float w[5];
  float dt;
  long long cells;     // X*Y
  const float* alpha;  // per-cell diffusivity (X, Y)
  float* lst;          // forward: if set, S^{n0+s} stored at lst + s*cells
  const float* lsts;   // adjoint: S^n at lsts + n*cells
  int ntop;            // adjoint: this pass runs n = ntop, ntop-1, ..., ntop-k+1
  float* galpha;       // adjoint: dJ/dalpha, accumulated in place
  int ramp;            // forward: time-dependent groups
  int n0;              // forward: rollout step of the pass's first step
  double t0, tstep;    // forward ramps: step n fills the boundary at fp32(t0 + n * tstep)
};

__device__ __forceinline__ bool heat_stencil_cell(int x, int y, int X, int Y, int g) {
  return x >= g && x < X - g && y >= g && y < Y - g;
}

// k forward steps on the stencil rectangle; STORE: S^{n0+s} of the tile's cells.
template <int R, bool STORE>
__device__ __forceinline__ float* heat_field_steps(const HAParams& P, const PdeBCRules& Rl, float* A, float* B,
                                                   const float* AL, int rx0, int RX, int ry0, int RY, int bx0,
                                                   int by0, int OX, int OY, PdeBCRules* SR) {
  H2Params HP;
  HP.X = P.X; HP.Y = P.Y; HP.g = P.g; HP.N = 1;
  const int g = P.g, X = P.X, Y = P.Y;
  const int sx0 = max(g, rx0 + R) - rx0, sx1 = min(X - g, rx0 + RX - R) - rx0;
  const int sy0 = max(g, ry0 + R) - ry0, sy1 = min(Y - g, ry0 + RY - R) - ry0;
  const int SW = max(sy1 - sy0, 1), SC = max(sx1 - sx0, 0) * max(sy1 - sy0, 0);
  const int nt = (int)blockDim.x;
  const int dq = nt / SW, dr = nt - dq * SW;
  const int tx0 = bx0 - rx0 - sx0, ty0 = by0 - ry0 - sy0;  // the tile in rectangle coordinates
  BcPlan<2> bp;  // the region is the same for every step of the pass
  bc_plan(bp, HP, rx0, RX, ry0, RY);
  for (int s = 0; s < P.k; ++s) {
    if (SR) {  // ramps: this step's group values (the previous step's fill is behind the barrier)
      const int gi = (int)threadIdx.x;
      if (gi < Rl.ngroups && Rl.group[gi].func == PDE_BC_FUNC_RAMP) {
        const float t = step_time(P.t0, P.tstep, P.n0 + s);
        SR->group[gi].value = bc_value(PDE_BC_FUNC_RAMP, Rl.group[gi].value, Rl.group[gi].t_max, &t);
      }
      __syncthreads();
    }
    bc_fill_planned<1, 1>(A, bp, HP, SR ? *SR : Rl, rx0, RX, ry0, RY, Rl.dx32);
    float* Ls = STORE ? P.lst + (size_t)s * P.cells : nullptr;
    int lx = (int)threadIdx.x / SW, ly = (int)threadIdx.x - lx * SW;
    for (int c = threadIdx.x; c < SC; c += nt) {
      const int i = (sx0 + lx) * RY + sy0 + ly;
      const float u2 = A[i];
      float acc = 0.0f;
#pragma unroll
      for (int t = 0; t < 2 * R + 1; ++t) acc = add(acc, mul(P.w[t], A[i + (t - R) * RY]));
#pragma unroll
      for (int t = 0; t < 2 * R + 1; ++t) acc = add(acc, mul(P.w[t], A[i + (t - R)]));
      B[i] = add(u2, mul(P.dt, mul(AL[i], acc)));
      if (STORE) {
        const int ox = lx - tx0, oy = ly - ty0;
        if (ox >= 0 && ox < OX && oy >= 0 && oy < OY) Ls[(size_t)(bx0 + ox) * Y + by0 + oy] = acc;
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
  return A;
}

template <int R>
__global__ void __launch_bounds__(1024) heat2d_field_fwd_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                                const HAParams P, const PdeBCRules Rl) {
  extern __shared__ __align__(16) float sm[];
  __shared__ PdeBCRules SR;  // ramps: the rules with the current step's group values
  if (P.ramp && threadIdx.x == 0) SR = Rl;
  const int tx = blockIdx.x / P.tiles_y, ty = blockIdx.x % P.tiles_y;
  const int bx0 = tx * P.TBX, by0 = ty * P.TBY;
  const int H = P.k * R + 1;
  const int X = P.X, Y = P.Y, g = P.g;
  const int rx0 = max(bx0 - H, 0), rx1 = min(bx0 + P.TBX + H, X);
  const int ry0 = max(by0 - H, 0), ry1 = min(by0 + P.TBY + H, Y);
  const int RX = rx1 - rx0, RY = ry1 - ry0, RC = RX * RY;
  const int OX = min(bx0 + P.TBX, X) - bx0, OY = min(by0 + P.TBY, Y) - by0;
  // Both level buffers start with the region; a step writes only its stencil
  // rectangle, so the other cells keep their loaded or last filled value.
  float* A0 = sm;
  float* B0 = sm + P.RC;
  float* AL = sm + 2 * P.RC;
  {
    RectWalk wk(RY, (int)blockDim.x);
    for (int i = threadIdx.x; i < RC; i += blockDim.x, wk.next()) {
      const size_t gi = (size_t)(rx0 + wk.row) * Y + ry0 + wk.col;
      cp_async4(A0 + i, in + gi, true);
      cp_async4(B0 + i, in + gi, true);
      cp_async4(AL + i, P.alpha + gi, true);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  PdeBCRules* srp = P.ramp ? &SR : nullptr;
  float* A = P.lst ? heat_field_steps<R, true>(P, Rl, A0, B0, AL, rx0, RX, ry0, RY, bx0, by0, OX, OY, srp)
                   : heat_field_steps<R, false>(P, Rl, A0, B0, AL, rx0, RX, ry0, RY, bx0, by0, OX, OY, srp);
  const float* Bf = (A == A0) ? B0 : A0;  // the last boundary-filled level
  // output: stencil cells from the newest level, the others as last filled
  RectWalk wo(OY, (int)blockDim.x);
  for (int i = threadIdx.x; i < OX * OY; i += blockDim.x, wo.next()) {
    const int x = bx0 + wo.row, y = by0 + wo.col;
    const int ri = (x - rx0) * RY + (y - ry0);
    out[(size_t)x * Y + y] = heat_stencil_cell(x, y, X, Y, g) ? A[ri] : Bf[ri];
  }
}

// Is cell (x, y) overwritten by the boundary fill (a filled ghost or a
// Dirichlet node)?  2D, one component.
__device__ __forceinline__ bool bc_overwritten(const PdeBCRules& Rl, int x, int y, int X, int Y, int g) {
  const bool yin = y >= g && y < Y - g, xin = x >= g && x < X - g;
  if (yin && (x == g - 1 || x == X - g)) {
    const int px = x == g - 1 ? g : X - g - 1;
    const int K = node_class_axis(px, X, g, true) * 9 + node_class_axis(y, Y, g, true) * 3 + 1;
    return Rl.ghost_group[K][0][0] >= 0;
  }
  if (xin && (y == g - 1 || y == Y - g)) {
    const int py = y == g - 1 ? g : Y - g - 1;
    const int K = node_class_axis(x, X, g, true) * 9 + node_class_axis(py, Y, g, true) * 3 + 1;
    return Rl.ghost_group[K][1][0] >= 0;
  }
  if (xin && yin && (x == g || x == X - g - 1 || y == g || y == Y - g - 1)) {
    const int K = node_class_axis(x, X, g, true) * 9 + node_class_axis(y, Y, g, true) * 3 + 1;
    const int gi = Rl.node_group[K];
    return gi >= 0 && (Rl.group[gi].comp_mask & 1u);
  }
  return false;
}

// How the mu of the ghost across node (px, py) on `axis` folds into its partner:
// 0 not at all (no ghost group), 1 subtracted (Dirichlet), 2 added.
__device__ __forceinline__ int bt_code(const PdeBCRules& Rl, int px, int py, int axis, int X, int Y, int g) {
  const int K = node_class_axis(px, X, g, true) * 9 + node_class_axis(py, Y, g, true) * 3 + 1;
  const int gi = Rl.ghost_group[K][axis][0];
  if (gi < 0) return 0;
  return Rl.group[gi].type == PDE_BC_DIRICHLET ? 1 : 2;
}

__device__ __forceinline__ float bt_fold(float v, float mG, int code) {
  return code == 1 ? sub(v, mG) : add(v, mG);
}

// The boundary role of region cell (x, y), fixed for a launch: bit 0 overwritten
// by the fill (bc_overwritten), bits 1-2 / 3-4 / 5-6 / 7-8 the fold codes of the
// x-low, x-high, y-low and y-high ghost whose partner it is, bit 9 stencil cell.
__device__ __forceinline__ int bt_flags(const PdeBCRules& Rl, int x, int y, int X, int Y, int g) {
  int f = bc_overwritten(Rl, x, y, X, Y, g) ? 1 : 0;
  const bool yin = y >= g && y < Y - g, xin = x >= g && x < X - g;
  if (yin && x == g + 1) f |= bt_code(Rl, g, y, 0, X, Y, g) << 1;
  if (yin && x == X - g - 2) f |= bt_code(Rl, X - g - 1, y, 0, X, Y, g) << 3;
  if (xin && y == g + 1) f |= bt_code(Rl, x, g, 1, X, Y, g) << 5;
  if (xin && y == Y - g - 2) f |= bt_code(Rl, x, Y - g - 1, 1, X, Y, g) << 7;
  if (heat_stencil_cell(x, y, X, Y, g)) f |= 1 << 9;
  return f;
}

template <int R>
__global__ void __launch_bounds__(1024) heat2d_adj_kernel(const float* __restrict__ lam_in,
                                                          float* __restrict__ lam_out, const HAParams P,
                                                          const PdeBCRules Rl) {
  extern __shared__ __align__(16) float sm[];
  const int tx = blockIdx.x / P.tiles_y, ty = blockIdx.x % P.tiles_y;
  const int bx0 = tx * P.TBX, by0 = ty * P.TBY;
  const int H = P.k * R;
  const int X = P.X, Y = P.Y, g = P.g;
  int rx0 = max(bx0 - H, 0), rx1 = min(bx0 + P.TBX + H, X);
  int ry0 = max(by0 - H, 0), ry1 = min(by0 + P.TBY + H, Y);
  if (rx0 <= g + 1) rx0 = 0;
  if (rx1 >= X - g - 1) rx1 = X;
  if (ry0 <= g + 1) ry0 = 0;
  if (ry1 >= Y - g - 1) ry1 = Y;
  const int RX = rx1 - rx0, RY = ry1 - ry0, RC = RX * RY;
  const int ox1 = min(bx0 + P.TBX, X), oy1 = min(by0 + P.TBY, Y);
  const int OX = ox1 - bx0, OY = oy1 - by0;
  float* Lm = sm;
  float* Z = sm + P.RC;
  float* M = sm + 2 * P.RC;
  float* AL = sm + 3 * P.RC;
  float* GA = sm + 4 * P.RC;  // dJ/dalpha of the tile (OX x OY)
  // S^n of the tile for the current and the next step (two slots): the next
  // step's values are copied in (cp.async) while the current step computes
  float* GL = GA + P.TBX * P.TBY;
  // bt_flags of the region's cells (regions that touch the boundary)
  int* FL = reinterpret_cast<int*>(GL + 2 * P.TBX * P.TBY);
  const int OT = OX * OY;
  auto fetch_S = [&](int s, int slot) {
    const float* Sn = P.lsts + (size_t)(P.ntop - s) * P.cells;
    RectWalk wk(OY, (int)blockDim.x);
    for (int i = threadIdx.x; i < OT; i += blockDim.x, wk.next())
      cp_async4(GL + slot * OT + i, Sn + (size_t)(bx0 + wk.row) * Y + by0 + wk.col, true);
  };
  const float dt = P.dt;
  {
    RectWalk wk(RY, (int)blockDim.x);
    for (int i = threadIdx.x; i < RC; i += blockDim.x, wk.next()) {
      const size_t gi = (size_t)(rx0 + wk.row) * Y + ry0 + wk.col;
      cp_async4(Lm + i, lam_in + gi, true);
      cp_async4(AL + i, P.alpha + gi, true);
    }
    RectWalk wt(OY, (int)blockDim.x);
    for (int i = threadIdx.x; i < OX * OY; i += blockDim.x, wt.next())
      cp_async4(GA + i, P.galpha + (size_t)(bx0 + wt.row) * Y + by0 + wt.col, true);
  }
  fetch_S(0, 0);
  cp_async_wait_all();
  {
    RectWalk wk(RY, (int)blockDim.x);  // the cells this thread copied
    for (int i = threadIdx.x; i < RC; i += blockDim.x, wk.next())
      Z[i] = heat_stencil_cell(rx0 + wk.row, ry0 + wk.col, X, Y, g) ? mul(dt, mul(AL[i], Lm[i])) : 0.0f;
  }
  __syncthreads();
  const int dq = (int)blockDim.x / RY, dr = (int)blockDim.x - dq * RY;
  const int lxs = (int)threadIdx.x / RY, lys = (int)threadIdx.x - lxs * RY;
  // A region without ghost, node or partner cells (x, y in [g+2, n-g-3] throughout)
  // has B^T = identity and only stencil cells: a step is one pass, mu written as the
  // new lam in place (a cell reads only its own lam) and the next z into a second
  // buffer (M, not otherwise needed here).  The same values as the two-pass step.
  const bool interior = rx0 > g + 1 && rx0 + RX < X - g - 2 && ry0 > g + 1 && ry0 + RY < Y - g - 2;
  float* Zc = Z;
  float* Zn = M;
  for (int s = 0; s < P.k && interior; ++s) {
    if (s + 1 < P.k) fetch_S(s + 1, (s + 1) & 1);  // its slot was last read in step s-1
    const float* Sg = GL + (s & 1) * OT;
    int lx = lxs, ly = lys;
    for (int i = threadIdx.x; i < RC; i += blockDim.x) {
      float acc = 0.0f;
#pragma unroll
      for (int t = 0; t < 2 * R + 1; ++t) {
        const int nx = lx + t - R;
        const float zv = (nx >= 0 && nx < RX) ? Zc[i + (t - R) * RY] : 0.0f;
        acc = add(acc, mul(P.w[t], zv));
      }
#pragma unroll
      for (int t = 0; t < 2 * R + 1; ++t) {
        const int ny = ly + t - R;
        const float zv = (ny >= 0 && ny < RY) ? Zc[i + (t - R)] : 0.0f;
        acc = add(acc, mul(P.w[t], zv));
      }
      const float l = Lm[i];
      const float m = add(l, acc);
      const int x = rx0 + lx, y = ry0 + ly;
      if (x >= bx0 && x < ox1 && y >= by0 && y < oy1) {
        const int gi = (x - bx0) * OY + (y - by0);
        GA[gi] = add(GA[gi], mul(l, mul(dt, Sg[gi])));
      }
      Lm[i] = m;
      Zn[i] = mul(dt, mul(AL[i], m));
      lx += dq;
      ly += dr;
      if (ly >= RY) { ly -= RY; ++lx; }
    }
    cp_async_wait_all();  // this thread's copies of the next step's S; the barrier publishes them
    __syncthreads();
    float* t = Zc;
    Zc = Zn;
    Zn = t;
  }
  if (!interior) {
    RectWalk wk(RY, (int)blockDim.x);
    for (int i = threadIdx.x; i < RC; i += blockDim.x, wk.next())
      FL[i] = bt_flags(Rl, rx0 + wk.row, ry0 + wk.col, X, Y, g);
    __syncthreads();
  }
  for (int s = 0; s < P.k && !interior; ++s) {
    if (s + 1 < P.k) fetch_S(s + 1, (s + 1) & 1);  // its slot was last read in step s-1
    const float* Sg = GL + (s & 1) * OT;
    // mu = lam + L^T(z); the gradient term of step n on the tile
    int lx = lxs, ly = lys;
    for (int i = threadIdx.x; i < RC; i += blockDim.x) {
      float acc = 0.0f;
#pragma unroll
      for (int t = 0; t < 2 * R + 1; ++t) {
        const int nx = lx + t - R;
        const float zv = (nx >= 0 && nx < RX) ? Z[i + (t - R) * RY] : 0.0f;
        acc = add(acc, mul(P.w[t], zv));
      }
#pragma unroll
      for (int t = 0; t < 2 * R + 1; ++t) {
        const int ny = ly + t - R;
        const float zv = (ny >= 0 && ny < RY) ? Z[i + (t - R)] : 0.0f;
        acc = add(acc, mul(P.w[t], zv));
      }
      const float l = Lm[i];
      M[i] = add(l, acc);
      const int x = rx0 + lx, y = ry0 + ly;
      if (x >= bx0 && x < ox1 && y >= by0 && y < oy1 && ((FL[i] >> 9) & 1)) {
        const int gi = (x - bx0) * OY + (y - by0);
        GA[gi] = add(GA[gi], mul(l, mul(dt, Sg[gi])));
      }
      lx += dq;
      ly += dr;
      if (ly >= RY) { ly -= RY; ++lx; }
    }
    __syncthreads();
    // lam = B^T(mu); z for the next step
    for (int i = threadIdx.x; i < RC; i += blockDim.x) {
      const int f = FL[i];
      float v = (f & 1) ? 0.0f : M[i];
      // the ghost of each pair lies in the region whenever its partner does (edge snapping)
      if (f & (3 << 1)) v = bt_fold(v, M[i - 2 * RY], (f >> 1) & 3);
      if (f & (3 << 3)) v = bt_fold(v, M[i + 2 * RY], (f >> 3) & 3);
      if (f & (3 << 5)) v = bt_fold(v, M[i - 2], (f >> 5) & 3);
      if (f & (3 << 7)) v = bt_fold(v, M[i + 2], (f >> 7) & 3);
      Lm[i] = v;
      Z[i] = ((f >> 9) & 1) ? mul(dt, mul(AL[i], v)) : 0.0f;
    }
    cp_async_wait_all();  // this thread's copies of the next step's S; the barrier publishes them
    __syncthreads();
  }
  RectWalk wo(OY, (int)blockDim.x);
  for (int i = threadIdx.x; i < OX * OY; i += blockDim.x, wo.next()) {
    const size_t gi = (size_t)(bx0 + wo.row) * Y + by0 + wo.col;
    lam_out[gi] = Lm[(bx0 + wo.row - rx0) * RY + (by0 + wo.col - ry0)];
    P.galpha[gi] = GA[i];
  }
}

}  // namespace pde
