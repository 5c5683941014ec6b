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
// region's cut edges lose one valid cell per step).  Regions are loaded with
// cp.async (every copy of a thread in flight at once; cells outside the ring
// zero-filled), and each step computes only the rectangle of cells that change.  Every product and sum is
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
};

// Rectangle of region cells a step computes: inside the node ring and one cell
// away from the region's edges (region indices [cx0, cx1) x [cy0, cy1)).  Cells
// outside the ring hold 0 in every buffer; region-edge cells are never
// rewritten, so their values go stale and, as cut edges do, invalidate one more
// cell inward per step.  Tile cells inside the ring are at least k cells from
// any cut edge, so they always lie in the rectangle.
struct WaveRect {
  int cx0, cy0, W, count;
  __device__ WaveRect(const WaveParams& P, const WaveRegion& Rg) {
    cx0 = max(P.g + 1, Rg.rx0 + 1) - Rg.rx0;
    const int cx1 = min(P.X - 1 - P.g, Rg.rx0 + Rg.RX - 1) - Rg.rx0;
    cy0 = max(P.g + 1, Rg.ry0 + 1) - Rg.ry0;
    const int cy1 = min(P.Y - 1 - P.g, Rg.ry0 + Rg.RY - 1) - Rg.ry0;
    W = max(cy1 - cy0, 0);
    count = max(cx1 - cx0, 0) * W;
  }
};

// The rectangle cells of this thread, q = threadIdx.x + c * blockDim.x for
// c < MAXC: the same cells in every step (the rectangle is fixed for the pass),
// so their indices, the gradient sums of the tile cells among them and the next
// step's L(u^n) values stay in registers.  Needs count <= MAXC * blockDim.x.
// dist: the cell's distance from the tile (the larger of its x and y distances).
// Step s of a k-step pass only has to update cells with dist <= k - 1 - s: the
// tile's values after the pass depend on no other cell, so the rest is skipped.
template <int MAXC>
struct WaveCells {
  int ri[MAXC];    // region index; -1 past the rectangle
  int gi[MAXC];    // array index of a tile cell; -1 for the other cells
  int dist[MAXC];  // distance from the tile
  __device__ WaveCells(const WaveRect& Rt, const WaveRegion& Rg, int Y) {
    const int nt = (int)blockDim.x;
    const int tx0 = Rg.bx0 - Rg.rx0 - Rt.cx0, ty0 = Rg.by0 - Rg.ry0 - Rt.cy0;
    RectWalk wk(Rt.W, nt);
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      ri[c] = -1;
      gi[c] = -1;
      dist[c] = 1 << 20;
      if ((int)threadIdx.x + c * nt < Rt.count) {
        ri[c] = (Rt.cx0 + wk.row) * Rg.RY + Rt.cy0 + wk.col;
        const int ox = wk.row - tx0, oy = wk.col - ty0;
        if (ox >= 0 && ox < Rg.OX && oy >= 0 && oy < Rg.OY) gi[c] = (Rg.bx0 + ox) * Y + Rg.by0 + oy;
        dist[c] = max(max(max(-ox, ox - (Rg.OX - 1)), max(-oy, oy - (Rg.OY - 1))), 0);
      }
      wk.next();
    }
  }
};

// Load a region row-major (RX x RY) with fn(region index, array x, array y).
template <class F>
__device__ __forceinline__ void for_region(const WaveRegion& Rg, F fn) {
  RectWalk wk(Rg.RY, (int)blockDim.x);
  for (int i = threadIdx.x; i < Rg.RX * Rg.RY; i += blockDim.x, wk.next()) fn(i, Rg.rx0 + wk.row, Rg.ry0 + wk.col);
}

// Tile cells (OX x OY) with fn(tile index, region index, global index).
template <class F>
__device__ __forceinline__ void for_tile(const WaveRegion& Rg, int Y, F fn) {
  RectWalk wk(Rg.OY, (int)blockDim.x);
  for (int t = threadIdx.x; t < Rg.OX * Rg.OY; t += blockDim.x, wk.next())
    fn(t, (Rg.bx0 - Rg.rx0 + wk.row) * Rg.RY + (Rg.by0 - Rg.ry0 + wk.col),
       (size_t)(Rg.bx0 + wk.row) * Y + Rg.by0 + wk.col);
}

// Laplacian at shared-memory index i (alpha 1), rows of RY cells.
__device__ __forceinline__ float lap5s(const float* sm, int i, int RY, const float* w) {
  float acc = 0.0f;
  acc = add(acc, mul(w[0], sm[i - RY]));
  acc = add(acc, mul(w[1], sm[i]));
  acc = add(acc, mul(w[2], sm[i + RY]));
  acc = add(acc, mul(w[0], sm[i - 1]));
  acc = add(acc, mul(w[1], sm[i]));
  acc = add(acc, mul(w[2], sm[i + 1]));
  return acc;
}

// k forward steps; the three levels are rotated as offsets into the one
// shared-memory array (om: u^{n-1}, o0: u^n, op: u^{n+1}).
template <bool STORE, int MAXC>
__device__ __forceinline__ void wave_fwd_steps(const WaveParams& P, const WaveRegion& Rg, float* sm, int& om,
                                               int& o0, int& op, int ok) {
  const int RY = Rg.RY, rx0 = Rg.rx0, ry0 = Rg.ry0;
  const WaveRect Rt(P, Rg);
  const int nt = (int)blockDim.x;
  const int srci = (P.srcx >= 0 && P.srcx >= rx0 && P.srcx < rx0 + Rg.RX && P.srcy >= ry0 && P.srcy < ry0 + RY)
                       ? (P.srcx - rx0) * RY + (P.srcy - ry0) : -1;
  if constexpr (MAXC > 0) {
    const WaveCells<MAXC> C(Rt, Rg, P.Y);
    float kc[MAXC];  // K of the thread's cells (constant over the pass)
#pragma unroll
    for (int c = 0; c < MAXC; ++c) kc[c] = C.ri[c] >= 0 ? sm[ok + C.ri[c]] : 0.0f;
    for (int s = 0; s < P.k; ++s) {
      const float sn = (srci >= 0) ? P.src[P.n0 + s] : 0.0f;
      float* Ls = STORE ? P.lst + (size_t)s * P.cells : nullptr;
      const int reach = P.k - 1 - s;
#pragma unroll
      for (int c = 0; c < MAXC; ++c) {
        const int i = C.ri[c];
        if (i < 0 || C.dist[c] > reach) continue;
        const float lap = lap5s(sm, o0 + i, RY, P.w);
        float v = sub(mul(2.0f, sm[o0 + i]), sm[om + i]);
        v = add(v, mul(kc[c], lap));
        if (i == srci) v = add(v, sn);
        sm[op + i] = v;
        if (STORE && C.gi[c] >= 0) Ls[C.gi[c]] = lap;
      }
      __syncthreads();
      const int t = om;
      om = o0;
      o0 = op;
      op = t;
    }
    return;
  }
  // the tile in rectangle coordinates (for the stored Laplacians)
  const int tx0 = Rg.bx0 - rx0 - Rt.cx0, ty0 = Rg.by0 - ry0 - Rt.cy0;
  for (int s = 0; s < P.k; ++s) {
    const float sn = (srci >= 0) ? P.src[P.n0 + s] : 0.0f;
    float* Ls = STORE ? P.lst + (size_t)s * P.cells : nullptr;
    RectWalk wk(Rt.W, nt);
    for (int q = threadIdx.x; q < Rt.count; q += nt, wk.next()) {
      const int i = (Rt.cx0 + wk.row) * RY + Rt.cy0 + wk.col;
      const float lap = lap5s(sm, o0 + i, RY, P.w);
      float v = sub(mul(2.0f, sm[o0 + i]), sm[om + i]);
      v = add(v, mul(sm[ok + i], lap));
      if (i == srci) v = add(v, sn);
      sm[op + i] = v;
      if (STORE) {
        const int ox = wk.row - tx0, oy = wk.col - ty0;
        if (ox >= 0 && ox < Rg.OX && oy >= 0 && oy < Rg.OY)
          Ls[(size_t)(Rg.bx0 + ox) * P.Y + Rg.by0 + oy] = lap;
      }
    }
    __syncthreads();
    const int t = om;
    om = o0;
    o0 = op;
    op = t;
  }
}

template <int MAXC>
__global__ void __launch_bounds__(1024) wave_fwd_tb_kernel(const float* __restrict__ um_in,
                                                            const float* __restrict__ u0_in,
                                                            const float* __restrict__ Kf, float* __restrict__ um_out,
                                                            float* __restrict__ u0_out, const WaveParams P) {
  extern __shared__ __align__(16) float sm[];
  const WaveRegion Rg(P, P.k);
  int om = 0, o0 = P.RC, op = 2 * P.RC;
  const int ok = 3 * P.RC;
  for_region(Rg, [&](int i, int x, int y) {
    const size_t gi = (size_t)x * P.Y + y;
    const bool in = wave_inside(P, x, y);  // the state is zero outside the node ring
    cp_async4(sm + om + i, um_in + gi, in);
    cp_async4(sm + o0 + i, u0_in + gi, in);
    cp_async4(sm + ok + i, Kf + gi, true);
    sm[op + i] = 0.0f;
  });
  cp_async_wait_all();
  __syncthreads();
  if (P.lst) wave_fwd_steps<true, MAXC>(P, Rg, sm, om, o0, op, ok);
  else wave_fwd_steps<false, MAXC>(P, Rg, sm, om, o0, op, ok);
  for_tile(Rg, P.Y, [&](int t, int ri, size_t gi) {
    um_out[gi] = sm[om + ri];
    u0_out[gi] = sm[o0 + ri];
  });
}

// MAXC > 0: the cells of a thread in registers (WaveCells), the gradient sums
// of its tile cells in registers and L(u^n) of the next step loaded while this
// one computes; MAXC = 0: any rectangle size, gradient tile in shared memory.
template <int MAXC>
__global__ void __launch_bounds__(1024) wave_adj_tb_kernel(const float* __restrict__ m1_in,
                                                            const float* __restrict__ m2_in,
                                                            const float* __restrict__ Kf, float* __restrict__ m1_out,
                                                            float* __restrict__ m2_out, const WaveParams P) {
  extern __shared__ __align__(16) float sm[];
  const WaveRegion Rg(P, P.k);
  const int RY = Rg.RY, rx0 = Rg.rx0, ry0 = Rg.ry0;
  // offsets into sm: mu^{n+2}, mu^{n+1}, mu^n; K o mu^{n+1}, K o mu^n; K; dJ/dK of the tile
  int o2 = 0, o1 = P.RC, o0 = 2 * P.RC, k1 = 3 * P.RC, k0 = 4 * P.RC;
  const int okk = 5 * P.RC, oga = 6 * P.RC;
  for_region(Rg, [&](int i, int x, int y) {
    const size_t gi = (size_t)x * P.Y + y;
    const bool in = wave_inside(P, x, y);
    cp_async4(sm + o2 + i, m2_in + gi, in);
    cp_async4(sm + o1 + i, m1_in + gi, in);
    cp_async4(sm + okk + i, Kf + gi, true);
    sm[o0 + i] = 0.0f;
    sm[k0 + i] = 0.0f;
  });
  if (MAXC == 0) for_tile(Rg, P.Y, [&](int t, int ri, size_t gi) { cp_async4(sm + oga + t, P.gK + gi, true); });
  cp_async_wait_all();
  // K o mu^{n+1} of the cells this thread copied (its own copies are complete)
  for_region(Rg, [&](int i, int x, int y) { sm[k1 + i] = mul(sm[okk + i], sm[o1 + i]); });
  __syncthreads();
  const WaveRect Rt(P, Rg);
  if constexpr (MAXC > 0) {
    const WaveCells<MAXC> C(Rt, Rg, P.Y);
    float ga[MAXC], lnext[MAXC], kc[MAXC];
    const float* L0 = P.lsts + (size_t)P.ntop * P.cells;
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      ga[c] = C.gi[c] >= 0 ? P.gK[C.gi[c]] : 0.0f;
      lnext[c] = C.gi[c] >= 0 ? __ldg(L0 + C.gi[c]) : 0.0f;
      kc[c] = C.ri[c] >= 0 ? sm[okk + C.ri[c]] : 0.0f;  // K of the thread's cells
    }
    for (int s = 0; s < P.k; ++s) {
      float ln[MAXC];
#pragma unroll
      for (int c = 0; c < MAXC; ++c) ln[c] = lnext[c];
      if (s + 1 < P.k) {
        const float* L1 = P.lsts + (size_t)(P.ntop - s - 1) * P.cells;
#pragma unroll
        for (int c = 0; c < MAXC; ++c)
          if (C.gi[c] >= 0) lnext[c] = __ldg(L1 + C.gi[c]);
      }
      const int reach = P.k - 1 - s;
#pragma unroll
      for (int c = 0; c < MAXC; ++c) {
        const int i = C.ri[c];
        if (i < 0 || C.dist[c] > reach) continue;
        const float m1 = sm[o1 + i];
        if (C.gi[c] >= 0) ga[c] = add(ga[c], mul(m1, ln[c]));  // dJ/dK += mu^{n+1} o L(u^n)
        const float acc = lap5s(sm, k1 + i, RY, P.w);
        const float v = add(sub(mul(2.0f, m1), sm[o2 + i]), acc);
        sm[o0 + i] = v;
        sm[k0 + i] = mul(kc[c], v);
      }
      __syncthreads();
      const int t = o2;
      o2 = o1;
      o1 = o0;
      o0 = t;
      const int u = k1;
      k1 = k0;
      k0 = u;
    }
#pragma unroll
    for (int c = 0; c < MAXC; ++c)
      if (C.gi[c] >= 0) P.gK[C.gi[c]] = ga[c];
    for_tile(Rg, P.Y, [&](int t, int ri, size_t gi) {
      m1_out[gi] = sm[o1 + ri];
      m2_out[gi] = sm[o2 + ri];
    });
    return;
  }
  const int nt = (int)blockDim.x;
  const int tx0 = Rg.bx0 - rx0 - Rt.cx0, ty0 = Rg.by0 - ry0 - Rt.cy0;
  for (int s = 0; s < P.k; ++s) {
    const float* Ln = P.lsts + (size_t)(P.ntop - s) * P.cells;
    RectWalk wk(Rt.W, nt);
    for (int q = threadIdx.x; q < Rt.count; q += nt, wk.next()) {
      const int i = (Rt.cx0 + wk.row) * RY + Rt.cy0 + wk.col;
      const float m1 = sm[o1 + i];
      {  // gradient term of step n on the tile: dJ/dK += mu^{n+1} o L(u^n)
        const int ox = wk.row - tx0, oy = wk.col - ty0;
        if (ox >= 0 && ox < Rg.OX && oy >= 0 && oy < Rg.OY) {
          const int t = oga + ox * Rg.OY + oy;
          sm[t] = add(sm[t], mul(m1, __ldg(Ln + (size_t)(Rg.bx0 + ox) * P.Y + Rg.by0 + oy)));
        }
      }
      // mu^n = 2 mu^{n+1} - mu^{n+2} + L(K o mu^{n+1})
      const float acc = lap5s(sm, k1 + i, RY, P.w);
      const float v = add(sub(mul(2.0f, m1), sm[o2 + i]), acc);
      sm[o0 + i] = v;
      sm[k0 + i] = mul(sm[okk + i], v);
    }
    __syncthreads();
    const int t = o2;
    o2 = o1;
    o1 = o0;
    o0 = t;
    const int u = k1;
    k1 = k0;
    k0 = u;
  }
  for_tile(Rg, P.Y, [&](int t, int ri, size_t gi) {
    m1_out[gi] = sm[o1 + ri];
    m2_out[gi] = sm[o2 + ri];
    P.gK[gi] = sm[oga + t];
  });
}

// ---- paired launch: forward recomputation beside the adjoint --------------
// One launch advances the same tile through up to k forward steps of one
// segment (storing L(u^n) of the tile, as wave_fwd_tb_kernel with lst set) and
// up to k adjoint steps of another segment (as wave_adj_tb_kernel).  The two
// are independent, so each warp interleaves two dependency chains and a step
// of both costs one barrier.  Arithmetic and per-cell operation order are
// those of the two kernels above.  Shared memory (offsets of RC cells): forward
// levels 0-2, adjoint levels 3-5, K o mu 6-7, K 8, then the gradient tile.
// MAXC as in wave_adj_tb_kernel (the forward's stored Laplacians use the same
// tile indices).
template <int MAXC>
__global__ void __launch_bounds__(1024) wave_pair_tb_kernel(const float* __restrict__ um_in,
                                                             const float* __restrict__ u0_in,
                                                             float* __restrict__ um_out, float* __restrict__ u0_out,
                                                             const float* __restrict__ m1_in,
                                                             const float* __restrict__ m2_in,
                                                             float* __restrict__ m1_out, float* __restrict__ m2_out,
                                                             const float* __restrict__ Kf, const WaveParams Pf,
                                                             const WaveParams Pa) {
  extern __shared__ __align__(16) float sm[];
  const int H = max(Pf.k, Pa.k);
  const WaveRegion Rg(Pa, H);  // Pf and Pa share the grid, tile and region capacity
  const int RY = Rg.RY, rx0 = Rg.rx0, ry0 = Rg.ry0;
  const int RC = Pa.RC;
  int fm = 0, f0 = RC, fp = 2 * RC;
  int a2 = 3 * RC, a1 = 4 * RC, a0 = 5 * RC, k1 = 6 * RC, k0 = 7 * RC;
  const int okk = 8 * RC, oga = 9 * RC;
  const bool fwd = Pf.k > 0, adj = Pa.k > 0;
  for_region(Rg, [&](int i, int x, int y) {
    const size_t gi = (size_t)x * Pa.Y + y;
    const bool in = wave_inside(Pa, x, y);  // the states are zero outside the node ring
    cp_async4(sm + okk + i, Kf + gi, true);
    if (fwd) {
      cp_async4(sm + fm + i, um_in + gi, in);
      cp_async4(sm + f0 + i, u0_in + gi, in);
      sm[fp + i] = 0.0f;
    }
    if (adj) {
      cp_async4(sm + a2 + i, m2_in + gi, in);
      cp_async4(sm + a1 + i, m1_in + gi, in);
      sm[a0 + i] = 0.0f;
      sm[k0 + i] = 0.0f;
    }
  });
  if (adj && MAXC == 0)
    for_tile(Rg, Pa.Y, [&](int t, int ri, size_t gi) { cp_async4(sm + oga + t, Pa.gK + gi, true); });
  cp_async_wait_all();
  if (adj) for_region(Rg, [&](int i, int x, int y) { sm[k1 + i] = mul(sm[okk + i], sm[a1 + i]); });
  __syncthreads();
  const WaveRect Rt(Pa, Rg);
  const int srci = (Pf.srcx >= 0 && Pf.srcx >= rx0 && Pf.srcx < rx0 + Rg.RX && Pf.srcy >= ry0 && Pf.srcy < ry0 + RY)
                       ? (Pf.srcx - rx0) * RY + (Pf.srcy - ry0) : -1;
  if constexpr (MAXC > 0) {
    const WaveCells<MAXC> C(Rt, Rg, Pa.Y);
    float ga[MAXC], lnext[MAXC], kc[MAXC];
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      ga[c] = 0.0f;
      lnext[c] = 0.0f;
      kc[c] = C.ri[c] >= 0 ? sm[okk + C.ri[c]] : 0.0f;  // K of the thread's cells, for both chains
      if (adj && C.gi[c] >= 0) {
        ga[c] = Pa.gK[C.gi[c]];
        lnext[c] = __ldg(Pa.lsts + (size_t)Pa.ntop * Pa.cells + C.gi[c]);
      }
    }
    for (int s = 0; s < H; ++s) {
      const bool fs = s < Pf.k, as = s < Pa.k;
      const float sn = (fs && srci >= 0) ? Pf.src[Pf.n0 + s] : 0.0f;
      float* Ls = fs ? Pf.lst + (size_t)s * Pf.cells : nullptr;
      float ln[MAXC];
#pragma unroll
      for (int c = 0; c < MAXC; ++c) ln[c] = lnext[c];
      if (s + 1 < Pa.k) {
        const float* L1 = Pa.lsts + (size_t)(Pa.ntop - s - 1) * Pa.cells;
#pragma unroll
        for (int c = 0; c < MAXC; ++c)
          if (C.gi[c] >= 0) lnext[c] = __ldg(L1 + C.gi[c]);
      }
      const int freach = Pf.k - 1 - s, areach = Pa.k - 1 - s;
#pragma unroll
      for (int c = 0; c < MAXC; ++c) {
        const int i = C.ri[c];
        if (i < 0) continue;
        if (fs && C.dist[c] <= freach) {  // u^{n+1} = 2 u^n - u^{n-1} + K o L(u^n) (+ source)
          const float lap = lap5s(sm, f0 + i, RY, Pf.w);
          float v = sub(mul(2.0f, sm[f0 + i]), sm[fm + i]);
          v = add(v, mul(kc[c], lap));
          if (i == srci) v = add(v, sn);
          sm[fp + i] = v;
          if (C.gi[c] >= 0) Ls[C.gi[c]] = lap;
        }
        if (as && C.dist[c] <= areach) {
          const float m1 = sm[a1 + i];
          if (C.gi[c] >= 0) ga[c] = add(ga[c], mul(m1, ln[c]));  // dJ/dK += mu^{n+1} o L(u^n)
          // mu^n = 2 mu^{n+1} - mu^{n+2} + L(K o mu^{n+1})
          const float acc = lap5s(sm, k1 + i, RY, Pa.w);
          const float v = add(sub(mul(2.0f, m1), sm[a2 + i]), acc);
          sm[a0 + i] = v;
          sm[k0 + i] = mul(kc[c], v);
        }
      }
      __syncthreads();
      if (fs) {
        const int t = fm;
        fm = f0;
        f0 = fp;
        fp = t;
      }
      if (as) {
        int t = a2;
        a2 = a1;
        a1 = a0;
        a0 = t;
        t = k1;
        k1 = k0;
        k0 = t;
      }
    }
    if (adj) {
#pragma unroll
      for (int c = 0; c < MAXC; ++c)
        if (C.gi[c] >= 0) Pa.gK[C.gi[c]] = ga[c];
    }
    for_tile(Rg, Pa.Y, [&](int t, int ri, size_t gi) {
      if (fwd) {
        um_out[gi] = sm[fm + ri];
        u0_out[gi] = sm[f0 + ri];
      }
      if (adj) {
        m1_out[gi] = sm[a1 + ri];
        m2_out[gi] = sm[a2 + ri];
      }
    });
    return;
  }
  const int nt = (int)blockDim.x;
  const int tx0 = Rg.bx0 - rx0 - Rt.cx0, ty0 = Rg.by0 - ry0 - Rt.cy0;
  for (int s = 0; s < H; ++s) {
    const bool fs = s < Pf.k, as = s < Pa.k;
    const float sn = (fs && srci >= 0) ? Pf.src[Pf.n0 + s] : 0.0f;
    float* Ls = fs ? Pf.lst + (size_t)s * Pf.cells : nullptr;
    const float* Ln = as ? Pa.lsts + (size_t)(Pa.ntop - s) * Pa.cells : nullptr;
    RectWalk wk(Rt.W, nt);
    for (int q = threadIdx.x; q < Rt.count; q += nt, wk.next()) {
      const int i = (Rt.cx0 + wk.row) * RY + Rt.cy0 + wk.col;
      const int ox = wk.row - tx0, oy = wk.col - ty0;
      const bool tile = ox >= 0 && ox < Rg.OX && oy >= 0 && oy < Rg.OY;
      if (fs) {  // u^{n+1} = 2 u^n - u^{n-1} + K o L(u^n) (+ source)
        const float lap = lap5s(sm, f0 + i, RY, Pf.w);
        float v = sub(mul(2.0f, sm[f0 + i]), sm[fm + i]);
        v = add(v, mul(sm[okk + i], lap));
        if (i == srci) v = add(v, sn);
        sm[fp + i] = v;
        if (tile) Ls[(size_t)(Rg.bx0 + ox) * Pf.Y + Rg.by0 + oy] = lap;
      }
      if (as) {
        const float m1 = sm[a1 + i];
        if (tile) {  // dJ/dK += mu^{n+1} o L(u^n)
          const int t = oga + ox * Rg.OY + oy;
          sm[t] = add(sm[t], mul(m1, __ldg(Ln + (size_t)(Rg.bx0 + ox) * Pa.Y + Rg.by0 + oy)));
        }
        // mu^n = 2 mu^{n+1} - mu^{n+2} + L(K o mu^{n+1})
        const float acc = lap5s(sm, k1 + i, RY, Pa.w);
        const float v = add(sub(mul(2.0f, m1), sm[a2 + i]), acc);
        sm[a0 + i] = v;
        sm[k0 + i] = mul(sm[okk + i], v);
      }
    }
    __syncthreads();
    if (fs) {
      const int t = fm;
      fm = f0;
      f0 = fp;
      fp = t;
    }
    if (as) {
      int t = a2;
      a2 = a1;
      a1 = a0;
      a0 = t;
      t = k1;
      k1 = k0;
      k0 = t;
    }
  }
  for_tile(Rg, Pa.Y, [&](int t, int ri, size_t gi) {
    if (fwd) {
      um_out[gi] = sm[fm + ri];
      u0_out[gi] = sm[f0 + ri];
    }
    if (adj) {
      m1_out[gi] = sm[a1 + ri];
      m2_out[gi] = sm[a2 + ri];
      Pa.gK[gi] = sm[oga + t];
    }
  });
}

}  // namespace pde
