// Batched rollouts: many independent 2D grids of uneven sizes advance nsteps
// in ONE persistent launch driven by a tile work queue.  The reference advances
// each grid with its own module chain (examples/2D_Heat_Equation.py:57-65:
// GridBoundary -> Laplacian -> ForwardEuler, three launches per step).
//
// Work items are (time block, grid, tile) triples in time-block-major order,
// taken from a global counter by persistent blocks.  An item runs the block's
// steps on its tile grown by a halo H (heat: k*R + 1 as heat2d_tb_kernel; wave:
// k as wave_fwd_tb_kernel), reading the grid's buffers of the block's parity
// and writing the others.  Before it starts it waits until the 3x3
// neighbouring tiles of its grid have finished the previous time block: their
// output is its input, and they no longer read the buffers it overwrites (the
// halo is at most one tile wide, so no other tile is involved).  An item only
// waits on items taken before it, which running blocks hold, so the queue
// cannot deadlock; every wait is still bounded (~2 s, then PDE_ERR_TIMEOUT is
// recorded and the block goes on).  A tile publishes its progress with a
// release store after a __threadfence; waiters read it with acquire loads.
//
// Heat step (per grid alpha, dt, dx):  u2 = BC(u);  u = u2 + dt*(alpha*Lap(u2)),
//   the arithmetic of heat2d_tb_kernel, bit-identical to pde_heat_rollout.
// Wave step (per grid K = dt^2 c^2):   u^{n+1} = 2u^n - u^{n-1} + K*Lap(u^n) on
//   the cells inside the node ring, zero elsewhere, as wave_fwd_tb_kernel with
//   a constant K field and no source.
#pragma once
#include "common.cuh"
#include "fused.cuh"
#include "tma.cuh"

namespace pde {

enum { BATCH_HEAT = 0, BATCH_WAVE = 1 };

struct BatchGridDev {
  float* a0;          // parity-0 input: heat u; wave u^n
  float* a1;          // wave u^{n-1} (parity 0)
  float* b0;          // parity-1 buffers (scratch)
  float* b1;
  int X, Y;           // array extents incl. ghosts (Z = 1, one component)
  int tiles_y;        // tiles along Y
  int tile_base;      // first queue index of this grid's tiles
  int ntiles;
  float coef, dt, dx32;  // heat: alpha, dt, dx; wave: K
  float w[5];         // Laplacian weights of this grid's dx
};

struct BatchParams {
  const BatchGridDev* grids;
  int ngrids;
  int total_tiles;
  int ntb;            // time blocks (even: the result lands in the parity-0 buffers)
  int nsteps;         // steps of time block tb: nsteps / ntb + (tb < nsteps % ntb)
  int H;              // halo of the longest block
  int TBX, TBY;
  int RC;             // region capacity (cells)
  int g;
  unsigned int* counter;   // work queue head (zeroed before the launch)
  unsigned int* progress;  // per tile: completed time blocks (zeroed before the launch)
  uint64_t wait_ns;        // bound of every progress wait
  int ramp;                // heat: some groups are time-dependent (ramps)
  double t0;               // heat ramps: step n of a grid fills its boundary at fp32(t0 + n * (double)dt)
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded wait until *p >= target.  Returns false after limit_ns, or at once
// when the library's device error word is set (another wait gave up: the
// launch's results are void, so no block spends its own limit on it).
__device__ __forceinline__ bool wait_at_least(const unsigned* p, unsigned target, uint64_t limit_ns) {
  if (ld_acquire_gpu(p) >= target) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t it = 0;; ++it) {
    __nanosleep(100);
    if (ld_acquire_gpu(p) >= target) return true;
    if ((it & 15u) == 15u &&
        (globaltimer_ns() - t0 > limit_ns || *reinterpret_cast<const volatile int*>(&g_err) != 0))
      return false;
  }
}

// Test hook of the bounded wait (pde_wait_probe): thread 0 waits until
// *word >= target under the library's limit and records PDE_ERR_TIMEOUT if it
// gives up.
__global__ void wait_probe_kernel(const unsigned* word, unsigned target, uint64_t limit_ns) {
  if (threadIdx.x == 0 && !wait_at_least(word, target, limit_ns)) flag_error(PDE_ERR_TIMEOUT);
}

template <int OP, int R>
__global__ void __launch_bounds__(256) batched_kernel(const BatchParams P, const PdeBCRules Rl) {
  extern __shared__ __align__(16) float sm[];
  __shared__ int s_item;
  __shared__ PdeBCRules SR;  // ramps: the rules with the current step's group values
  if (OP == BATCH_HEAT && P.ramp && threadIdx.x == 0) SR = Rl;
  const unsigned total_items = (unsigned)P.total_tiles * (unsigned)P.ntb;
  const int q = P.nsteps / P.ntb, rmd = P.nsteps % P.ntb;
  const int H = P.H, g = P.g;
  bool timed_out = false;
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(P.counter, 1u);
    __syncthreads();
    const unsigned item = (unsigned)s_item;
    __syncthreads();  // s_item is rewritten at the top of the next item
    if (item >= total_items) break;
    const int tb = (int)(item / (unsigned)P.total_tiles);
    const int gt = (int)(item - (unsigned)tb * (unsigned)P.total_tiles);
    int lo = 0, hi = P.ngrids - 1;  // the last grid whose tile_base <= gt
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (P.grids[mid].tile_base <= gt) lo = mid; else hi = mid - 1;
    }
    const BatchGridDev& Gd = P.grids[lo];
    const int X = Gd.X, Y = Gd.Y, tiles_y = Gd.tiles_y;
    const int lt = gt - Gd.tile_base;
    const int tx = lt / tiles_y, ty = lt - tx * tiles_y;
    const int tiles_x = Gd.ntiles / tiles_y;
    if (tb > 0 && threadIdx.x < 9) {
      const int nx = tx + (int)threadIdx.x / 3 - 1, ny = ty + (int)threadIdx.x % 3 - 1;
      if (nx >= 0 && nx < tiles_x && ny >= 0 && ny < tiles_y && !timed_out) {
        if (!wait_at_least(P.progress + Gd.tile_base + nx * tiles_y + ny, (unsigned)tb, P.wait_ns)) {
          timed_out = true;
          flag_error(PDE_ERR_TIMEOUT);
        }
      }
      __threadfence();
    }
    __syncthreads();
    const int ks = q + (tb < rmd ? 1 : 0);
    const bool odd = (tb & 1) != 0;
    const float* in0 = odd ? Gd.b0 : Gd.a0;
    const float* in1 = odd ? Gd.b1 : Gd.a1;
    float* out0 = odd ? Gd.a0 : Gd.b0;
    float* out1 = odd ? Gd.a1 : Gd.b1;
    const float coef = Gd.coef, dt = Gd.dt, dx32 = Gd.dx32;
    float w[2 * R + 1];
#pragma unroll
    for (int t = 0; t < 2 * R + 1; ++t) w[t] = Gd.w[t];
    const int bx0 = tx * P.TBX, by0 = ty * P.TBY;
    const int rx0 = max(bx0 - H, 0), rx1 = min(bx0 + P.TBX + H, X);
    const int ry0 = max(by0 - H, 0), ry1 = min(by0 + P.TBY + H, Y);
    const int RX = rx1 - rx0, RY = ry1 - ry0, RC = RX * RY;
    const int OX = min(bx0 + P.TBX, X) - bx0, OY = min(by0 + P.TBY, Y) - by0;
    const int nt = (int)blockDim.x;
    // Each step walks its rectangle flattened (start at cell tid, advance by
    // blockDim.x = dq rows + dr cells), so every lane has a cell.
    if (OP == BATCH_HEAT) {
      // Both buffers start with the region; a step writes only its stencil
      // rectangle, so cells outside it keep their loaded or last filled value.
      float* A = sm;  // newest level
      float* B = sm + P.RC;
      {
        RectWalk wk(RY, nt);
        for (int i = threadIdx.x; i < RC; i += nt, wk.next()) {
          const float* src = in0 + (size_t)(rx0 + wk.row) * Y + ry0 + wk.col;
          cp_async4(A + i, src, true);
          cp_async4(B + i, src, true);
        }
      }
      cp_async_wait_all();
      __syncthreads();
      H2Params HP;
      HP.X = X; HP.Y = Y; HP.g = g; HP.N = 1;
      const int sx0 = max(g, rx0 + R) - rx0, sx1 = min(X - g, rx0 + RX - R) - rx0;
      const int sy0 = max(g, ry0 + R) - ry0, sy1 = min(Y - g, ry0 + RY - R) - ry0;
      const int tlx0 = bx0 - rx0, tly0 = by0 - ry0;  // the tile in region coordinates
      BcPlan<2> bp;
      bc_plan(bp, HP, rx0, RX, ry0, RY);
      const int n_first = tb * q + min(tb, rmd);  // rollout step of the block's first step
      for (int s = 0; s < ks; ++s) {
        if (P.ramp) {  // this step's ramp values (the previous step's fill is behind the barrier)
          const int gi = (int)threadIdx.x;
          if (gi < Rl.ngroups && Rl.group[gi].func == PDE_BC_FUNC_RAMP) {
            const float t = step_time(P.t0, (double)dt, n_first + s);
            SR.group[gi].value = bc_value(PDE_BC_FUNC_RAMP, Rl.group[gi].value, Rl.group[gi].t_max, &t);
          }
          __syncthreads();
        }
        bc_fill_planned<1, 1>(A, bp, HP, P.ramp ? SR : Rl, rx0, RX, ry0, RY, dx32);
        // Step s only has to update the stencil cells within R (ks - 1 - s) + 1 of
        // the tile (the boundary fills read inward): the stencil rectangle cut to
        // that box; the cells outside it keep stale values nobody reads.
        const int reach = R * (ks - 1 - s) + 1;
        const int qx0 = max(sx0, tlx0 - reach), qx1 = min(sx1, tlx0 + OX + reach);
        const int qy0 = max(sy0, tly0 - reach), qy1 = min(sy1, tly0 + OY + reach);
        const int SW = max(qy1 - qy0, 1), SC = max(qx1 - qx0, 0) * max(qy1 - qy0, 0);
        const int dq = nt / SW, dr = nt - dq * SW;
        int lx = (int)threadIdx.x / SW, ly = (int)threadIdx.x - lx * SW;
        for (int c = threadIdx.x; c < SC; c += nt) {
          const int i = (qx0 + lx) * RY + qy0 + ly;
          const float u2 = A[i];
          float acc = 0.0f;
#pragma unroll
          for (int t = 0; t < 2 * R + 1; ++t) acc = add(acc, mul(w[t], A[i + (t - R) * RY]));
#pragma unroll
          for (int t = 0; t < 2 * R + 1; ++t) acc = add(acc, mul(w[t], A[i + (t - R)]));
          B[i] = add(u2, mul(dt, mul(coef, acc)));
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
      {
        RectWalk wk(OY, nt);
        for (int i = threadIdx.x; i < OX * OY; i += nt, wk.next()) {
          const int x = bx0 + wk.row, y = by0 + wk.col;
          const int ri = (x - rx0) * RY + (y - ry0);
          const bool st = x >= g && x < X - g && y >= g && y < Y - g;
          out0[(size_t)x * Y + y] = st ? A[ri] : B[ri];
        }
      }
    } else {
      float* Bm = sm;
      float* B0 = sm + P.RC;
      float* Bp = sm + 2 * P.RC;
      // the state is zero outside the node ring (x, y in [g+1, n-g-2]) in every buffer
      RectWalk wl(RY, nt);
      for (int i = threadIdx.x; i < RC; i += nt, wl.next()) {
        const int x = rx0 + wl.row, y = ry0 + wl.col;
        const bool inside = x > g && x < X - 1 - g && y > g && y < Y - 1 - g;
        const size_t gi = (size_t)x * Y + y;
        cp_async4(Bm + i, in1 + gi, inside);
        cp_async4(B0 + i, in0 + gi, inside);
        Bp[i] = 0.0f;
      }
      cp_async_wait_all();
      __syncthreads();
      // computed rectangle: inside the ring, one cell away from the region's edges
      const int cx0 = max(g + 1, rx0 + 1) - rx0, cx1 = min(X - 1 - g, rx0 + RX - 1) - rx0;
      const int cy0 = max(g + 1, ry0 + 1) - ry0, cy1 = min(Y - 1 - g, ry0 + RY - 1) - ry0;
      const int tlx0 = bx0 - rx0, tly0 = by0 - ry0;  // the tile in region coordinates
      for (int s = 0; s < ks; ++s) {
        // step s only has to update the cells within ks - 1 - s of the tile
        const int reach = ks - 1 - s;
        const int qx0 = max(cx0, tlx0 - reach), qx1 = min(cx1, tlx0 + OX + reach);
        const int qy0 = max(cy0, tly0 - reach), qy1 = min(cy1, tly0 + OY + reach);
        const int CW = max(qy1 - qy0, 1), CC = max(qx1 - qx0, 0) * max(qy1 - qy0, 0);
        const int dq = nt / CW, dr = nt - dq * CW;
        int lx = (int)threadIdx.x / CW, ly = (int)threadIdx.x - lx * CW;
        for (int c = threadIdx.x; c < CC; c += nt) {
          const int i = (qx0 + lx) * RY + qy0 + ly;
          float acc = 0.0f;  // Laplacian, alpha 1 (FDM/kernel/laplacian.py:40-46 order)
          acc = add(acc, mul(w[0], B0[i - RY]));
          acc = add(acc, mul(w[1], B0[i]));
          acc = add(acc, mul(w[2], B0[i + RY]));
          acc = add(acc, mul(w[0], B0[i - 1]));
          acc = add(acc, mul(w[1], B0[i]));
          acc = add(acc, mul(w[2], B0[i + 1]));
          Bp[i] = add(sub(mul(2.0f, B0[i]), Bm[i]), mul(coef, acc));
          lx += dq;
          ly += dr;
          if (ly >= CW) { ly -= CW; ++lx; }
        }
        __syncthreads();
        float* t = Bm;
        Bm = B0;
        B0 = Bp;
        Bp = t;
      }
      RectWalk wo(OY, nt);
      for (int i = threadIdx.x; i < OX * OY; i += nt, wo.next()) {
        const int ri = (bx0 + wo.row - rx0) * RY + (by0 + wo.col - ry0);
        const size_t gi = (size_t)(bx0 + wo.row) * Y + by0 + wo.col;
        out1[gi] = Bm[ri];
        out0[gi] = B0[ri];
      }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) st_release_gpu(P.progress + gt, (unsigned)(tb + 1));
  }
}

}  // namespace pde
