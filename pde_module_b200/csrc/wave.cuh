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
#include <type_traits>

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
  int cx0, cy0, W, NR, count;  // NR rows of W cells
  __device__ WaveRect(const WaveParams& P, const WaveRegion& Rg) {
    cx0 = max(P.g + 1, Rg.rx0 + 1) - Rg.rx0;
    const int cx1 = min(P.X - 1 - P.g, Rg.rx0 + Rg.RX - 1) - Rg.rx0;
    cy0 = max(P.g + 1, Rg.ry0 + 1) - Rg.ry0;
    const int cy1 = min(P.Y - 1 - P.g, Rg.ry0 + Rg.RY - 1) - Rg.ry0;
    W = max(cy1 - cy0, 0);
    NR = max(cx1 - cx0, 0);
    count = NR * W;
  }
};

// The rectangle cells of this thread: its slots q = threadIdx.x + c * blockDim.x
// (c < MAXC) walk the rectangle's rows at their full region width RY, the
// columns outside the rectangle left idle, so a warp's 32 slots are 32
// consecutive region cells (NB-float stride in shared memory: no bank
// conflicts) and no warp straddles the gap between two rectangle rows.  The
// same cells in every step (the rectangle is fixed for the pass), so their
// indices, the gradient sums of the tile cells among them and the next step's
// L(u^n) values stay in registers.  Needs NR * RY <= MAXC * blockDim.x.
// dist: the cell's distance from the tile (the larger of its x and y distances).
// Step s of a k-step pass only has to update cells with dist <= k - 1 - s: the
// tile's values after the pass depend on no other cell, so the rest is skipped.
template <int MAXC>
struct WaveCells {
  int ri[MAXC];    // region index; -1 for an idle slot
  int gi[MAXC];    // array index of a tile cell; 0 (a valid address) for the other cells
  int dist[MAXC];  // distance from the tile; 1 << 20 for an idle slot
  unsigned tile;   // bit c: slot c holds a tile cell
  __device__ bool is_tile(int c) const { return (tile >> c) & 1u; }
  __device__ WaveCells(const WaveRect& Rt, const WaveRegion& Rg, int Y) {
    const int nt = (int)blockDim.x;
    // tile origin: rows relative to the rectangle, columns relative to the region
    const int tx0 = Rg.bx0 - Rg.rx0 - Rt.cx0, ty0 = Rg.by0 - Rg.ry0;
    const int n = Rt.NR * Rg.RY;
    RectWalk wk(Rg.RY, nt);
    tile = 0;
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      ri[c] = -1;
      gi[c] = 0;
      dist[c] = 1 << 20;
      if ((int)threadIdx.x + c * nt < n && wk.col >= Rt.cy0 && wk.col < Rt.cy0 + Rt.W) {
        ri[c] = (Rt.cx0 + wk.row) * Rg.RY + wk.col;
        const int ox = wk.row - tx0, oy = wk.col - ty0;
        if (ox >= 0 && ox < Rg.OX && oy >= 0 && oy < Rg.OY) {
          gi[c] = (Rg.bx0 + ox) * Y + Rg.by0 + oy;
          tile |= 1u << c;
        }
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

// ---- shared-memory layout ---------------------------------------------------
// A region's cells are interleaved, NB floats per cell, so a cell's time levels
// and K sit at fixed offsets from one base: every access of a step is the cell's
// base plus a constant (neighbours: +-NB along y, +-NB*RY along x).  Leapfrog
// keeps two levels per field: step n overwrites u^{n-1}, which only its own cell
// reads, with u^{n+1}, so the two levels swap roles every step (parity
// p = s & 1) and the step loop runs two steps per iteration with p a
// compile-time constant.  The adjoint does the same with mu^{n+2} and keeps two
// levels of K o mu (its neighbours are read while the next level is written).
//   forward  (NB 3): 0, 1 levels of u (u^n in 1 - p, u^{n-1} in p), 2 K
//   adjoint  (NB 5): 0, 1 levels of mu (mu^{n+1} in 1 - p), 2, 3 levels of K o mu
//                    (K o mu^{n+1} in 3 - p), 4 K
//   paired   (NB 7): 0, 1 u; 2, 3 mu; 4, 5 K o mu; 6 K
template <int V>
using IC = std::integral_constant<int, V>;

// st.global under a predicate, without a branch around it
__device__ __forceinline__ void st_global_if(float* p, float v, bool on) {
  asm volatile(
      "{\n .reg .pred q;\n setp.ne.b32 q, %2, 0;\n @q st.global.f32 [%0], %1;\n}\n" ::"l"(p), "f"(v),
      "r"((int)on)
      : "memory");
}

// Laplacian (alpha 1) around the interleaved element c: rows rs floats apart,
// neighbours along y NB floats apart; the reference's term order.
template <int NB>
__device__ __forceinline__ float lap5n(const float* c, int rs, const float* w) {
  float acc = 0.0f;
  acc = add(acc, mul(w[0], c[-rs]));
  acc = add(acc, mul(w[1], c[0]));
  acc = add(acc, mul(w[2], c[rs]));
  acc = add(acc, mul(w[0], c[-NB]));
  acc = add(acc, mul(w[1], c[0]));
  acc = add(acc, mul(w[2], c[NB]));
  return acc;
}

__device__ __forceinline__ int wave_src_index(const WaveParams& P, const WaveRegion& Rg) {
  return (P.srcx >= 0 && P.srcx >= Rg.rx0 && P.srcx < Rg.rx0 + Rg.RX && P.srcy >= Rg.ry0 &&
          P.srcy < Rg.ry0 + Rg.RY)
             ? (P.srcx - Rg.rx0) * Rg.RY + (P.srcy - Rg.ry0)
             : -1;
}

// k forward steps: u^{n+1} = 2 u^n - u^{n-1} + K o L(u^n) (+ source), written over u^{n-1}.
template <bool STORE, int MAXC>
__device__ __forceinline__ void wave_fwd_steps(const WaveParams& P, const WaveRegion& Rg, float* sm) {
  constexpr int NB = 3;
  const int RY = Rg.RY, rs = NB * RY;
  const WaveRect Rt(P, Rg);
  const int srci = wave_src_index(P, Rg);
  if constexpr (MAXC > 0) {
    const WaveCells<MAXC> C(Rt, Rg, P.Y);
    float kc[MAXC];  // K of the thread's cells (constant over the pass)
#pragma unroll
    for (int c = 0; c < MAXC; ++c) kc[c] = C.ri[c] >= 0 ? sm[NB * C.ri[c] + 2] : 0.0f;
    auto step = [&](auto PAR, int s) {
      constexpr int p = decltype(PAR)::value;
      const float sn = (srci >= 0) ? P.src[P.n0 + s] : 0.0f;
      float* Ls = STORE ? P.lst + (size_t)s * P.cells : nullptr;
      const int reach = P.k - 1 - s;
#pragma unroll
      for (int c = 0; c < MAXC; ++c) {
        if (C.dist[c] > reach) continue;  // past the rectangle: dist is out of reach
        float* pc = sm + NB * C.ri[c];
        const float lap = lap5n<NB>(pc + (1 - p), rs, P.w);
        float v = sub(mul(2.0f, pc[1 - p]), pc[p]);
        v = add(v, mul(kc[c], lap));
        if (C.ri[c] == srci) v = add(v, sn);
        pc[p] = v;
        if (STORE) st_global_if(Ls + C.gi[c], lap, C.is_tile(c));
      }
      __syncthreads();
    };
    for (int s = 0; s < P.k; s += 2) {
      step(IC<0>{}, s);
      if (s + 1 < P.k) step(IC<1>{}, s + 1);
    }
    return;
  }
  // the tile in rectangle coordinates (for the stored Laplacians)
  const int nt = (int)blockDim.x;
  const int tx0 = Rg.bx0 - Rg.rx0 - Rt.cx0, ty0 = Rg.by0 - Rg.ry0 - Rt.cy0;
  for (int s = 0; s < P.k; ++s) {
    const int p = s & 1;
    const float sn = (srci >= 0) ? P.src[P.n0 + s] : 0.0f;
    float* Ls = STORE ? P.lst + (size_t)s * P.cells : nullptr;
    RectWalk wk(Rt.W, nt);
    for (int q = threadIdx.x; q < Rt.count; q += nt, wk.next()) {
      const int i = (Rt.cx0 + wk.row) * RY + Rt.cy0 + wk.col;
      float* pc = sm + NB * i;
      const float lap = lap5n<NB>(pc + (1 - p), rs, P.w);
      float v = sub(mul(2.0f, pc[1 - p]), pc[p]);
      v = add(v, mul(pc[2], lap));
      if (i == srci) v = add(v, sn);
      pc[p] = v;
      if (STORE) {
        const int ox = wk.row - tx0, oy = wk.col - ty0;
        if (ox >= 0 && ox < Rg.OX && oy >= 0 && oy < Rg.OY)
          Ls[(size_t)(Rg.bx0 + ox) * P.Y + Rg.by0 + oy] = lap;
      }
    }
    __syncthreads();
  }
}

template <int MAXC>
__global__ void __launch_bounds__(1024) wave_fwd_tb_kernel(const float* __restrict__ um_in,
                                                            const float* __restrict__ u0_in,
                                                            const float* __restrict__ Kf, float* __restrict__ um_out,
                                                            float* __restrict__ u0_out, const WaveParams P) {
  extern __shared__ __align__(16) float sm[];
  constexpr int NB = 3;
  const WaveRegion Rg(P, P.k);
  for_region(Rg, [&](int i, int x, int y) {
    const size_t gi = (size_t)x * P.Y + y;
    const bool in = wave_inside(P, x, y);  // the state is zero outside the node ring
    cp_async4(sm + NB * i, um_in + gi, in);
    cp_async4(sm + NB * i + 1, u0_in + gi, in);
    cp_async4(sm + NB * i + 2, Kf + gi, true);
  });
  cp_async_wait_all();
  __syncthreads();
  if (P.lst) wave_fwd_steps<true, MAXC>(P, Rg, sm);
  else wave_fwd_steps<false, MAXC>(P, Rg, sm);
  const int nw = (P.k & 1) ? 0 : 1;  // level the last step wrote
  for_tile(Rg, P.Y, [&](int t, int ri, size_t gi) {
    um_out[gi] = sm[NB * ri + (1 - nw)];
    u0_out[gi] = sm[NB * ri + nw];
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
  constexpr int NB = 5;
  const WaveRegion Rg(P, P.k);
  const int RY = Rg.RY, rs = NB * RY;
  const int oga = NB * P.RC;  // dJ/dK of the tile (MAXC = 0)
  for_region(Rg, [&](int i, int x, int y) {
    const size_t gi = (size_t)x * P.Y + y;
    const bool in = wave_inside(P, x, y);
    cp_async4(sm + NB * i, m2_in + gi, in);      // mu^{n+2}
    cp_async4(sm + NB * i + 1, m1_in + gi, in);  // mu^{n+1}
    cp_async4(sm + NB * i + 4, Kf + gi, true);
    sm[NB * i + 2] = 0.0f;
  });
  if (MAXC == 0) for_tile(Rg, P.Y, [&](int t, int ri, size_t gi) { cp_async4(sm + oga + t, P.gK + gi, true); });
  cp_async_wait_all();
  // K o mu^{n+1} of the cells this thread copied (its own copies are complete)
  for_region(Rg, [&](int i, int x, int y) { sm[NB * i + 3] = mul(sm[NB * i + 4], sm[NB * i + 1]); });
  __syncthreads();
  const WaveRect Rt(P, Rg);
  if constexpr (MAXC > 0) {
    const WaveCells<MAXC> C(Rt, Rg, P.Y);
    // lv: L(u^n) of the step at the thread's cells, the next step's issued before
    // each barrier; the other cells load from index 0 and their gradient sums go
    // unused (no per-cell branches)
    float ga[MAXC], lv[MAXC], kc[MAXC];
    const float* L0 = P.lsts + (size_t)P.ntop * P.cells;
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      ga[c] = C.is_tile(c) ? P.gK[C.gi[c]] : 0.0f;
      lv[c] = __ldg(L0 + C.gi[c]);
      kc[c] = C.ri[c] >= 0 ? sm[NB * C.ri[c] + 4] : 0.0f;  // K of the thread's cells
    }
    auto step = [&](auto PAR, int s) {
      constexpr int p = decltype(PAR)::value;
      const int reach = P.k - 1 - s;
#pragma unroll
      for (int c = 0; c < MAXC; ++c) {
        if (C.dist[c] > reach) continue;
        float* pc = sm + NB * C.ri[c];
        const float m1 = pc[1 - p];
        ga[c] = add(ga[c], mul(m1, lv[c]));  // dJ/dK += mu^{n+1} o L(u^n) (kept for tile cells)
        // mu^n = 2 mu^{n+1} - mu^{n+2} + L(K o mu^{n+1})
        const float acc = lap5n<NB>(pc + (3 - p), rs, P.w);
        const float v = add(sub(mul(2.0f, m1), pc[p]), acc);
        pc[p] = v;
        pc[2 + p] = mul(kc[c], v);
      }
      if (s + 1 < P.k) {
        const float* L1 = P.lsts + (size_t)(P.ntop - s - 1) * P.cells;
#pragma unroll
        for (int c = 0; c < MAXC; ++c) lv[c] = __ldg(L1 + C.gi[c]);
      }
      __syncthreads();
    };
    for (int s = 0; s < P.k; s += 2) {
      step(IC<0>{}, s);
      if (s + 1 < P.k) step(IC<1>{}, s + 1);
    }
#pragma unroll
    for (int c = 0; c < MAXC; ++c)
      if (C.is_tile(c)) P.gK[C.gi[c]] = ga[c];
  } else {
    const int nt = (int)blockDim.x;
    const int tx0 = Rg.bx0 - Rg.rx0 - Rt.cx0, ty0 = Rg.by0 - Rg.ry0 - Rt.cy0;
    for (int s = 0; s < P.k; ++s) {
      const int p = s & 1;
      const float* Ln = P.lsts + (size_t)(P.ntop - s) * P.cells;
      RectWalk wk(Rt.W, nt);
      for (int q = threadIdx.x; q < Rt.count; q += nt, wk.next()) {
        const int i = (Rt.cx0 + wk.row) * RY + Rt.cy0 + wk.col;
        float* pc = sm + NB * i;
        const float m1 = pc[1 - p];
        {  // gradient term of step n on the tile: dJ/dK += mu^{n+1} o L(u^n)
          const int ox = wk.row - tx0, oy = wk.col - ty0;
          if (ox >= 0 && ox < Rg.OX && oy >= 0 && oy < Rg.OY) {
            const int t = oga + ox * Rg.OY + oy;
            sm[t] = add(sm[t], mul(m1, __ldg(Ln + (size_t)(Rg.bx0 + ox) * P.Y + Rg.by0 + oy)));
          }
        }
        // mu^n = 2 mu^{n+1} - mu^{n+2} + L(K o mu^{n+1})
        const float acc = lap5n<NB>(pc + (3 - p), rs, P.w);
        const float v = add(sub(mul(2.0f, m1), pc[p]), acc);
        pc[p] = v;
        pc[2 + p] = mul(pc[4], v);
      }
      __syncthreads();
    }
    for_tile(Rg, P.Y, [&](int t, int ri, size_t gi) { P.gK[gi] = sm[oga + t]; });
  }
  const int nw = (P.k & 1) ? 0 : 1;  // level the last step wrote
  for_tile(Rg, P.Y, [&](int t, int ri, size_t gi) {
    m1_out[gi] = sm[NB * ri + nw];
    m2_out[gi] = sm[NB * ri + (1 - nw)];
  });
}

// ---- paired launch: forward recomputation beside the adjoint --------------
// One launch advances the same tile through up to k forward steps of one
// segment (storing L(u^n) of the tile, as wave_fwd_tb_kernel with lst set) and
// up to k adjoint steps of another segment (as wave_adj_tb_kernel).  The two
// are independent, so each warp interleaves two dependency chains and a step
// of both costs one barrier.  Arithmetic and per-cell operation order are
// those of the two kernels above.  Shared memory: the NB = 7 interleaved
// region, then the gradient tile.  This is the general loop over the
// rectangle (any region size); rectangles of up to 8 cells per thread run
// the packed register-list kernel below.
__global__ void __launch_bounds__(1024) wave_pair_tb_kernel(const float* __restrict__ um_in,
                                                             const float* __restrict__ u0_in,
                                                             float* __restrict__ um_out, float* __restrict__ u0_out,
                                                             const float* __restrict__ m1_in,
                                                             const float* __restrict__ m2_in,
                                                             float* __restrict__ m1_out, float* __restrict__ m2_out,
                                                             const float* __restrict__ Kf, const WaveParams Pf,
                                                             const WaveParams Pa) {
  extern __shared__ __align__(16) float sm[];
  constexpr int NB = 7;
  const int H = max(Pf.k, Pa.k);
  const WaveRegion Rg(Pa, H);  // Pf and Pa share the grid, tile and region capacity
  const int RY = Rg.RY, rs = NB * RY;
  const int oga = NB * Pa.RC;
  const bool fwd = Pf.k > 0, adj = Pa.k > 0;
  for_region(Rg, [&](int i, int x, int y) {
    const size_t gi = (size_t)x * Pa.Y + y;
    const bool in = wave_inside(Pa, x, y);  // the states are zero outside the node ring
    float* pc = sm + NB * i;
    cp_async4(pc + 6, Kf + gi, true);
    if (fwd) {
      cp_async4(pc, um_in + gi, in);
      cp_async4(pc + 1, u0_in + gi, in);
    }
    if (adj) {
      cp_async4(pc + 2, m2_in + gi, in);
      cp_async4(pc + 3, m1_in + gi, in);
      pc[4] = 0.0f;
    }
  });
  if (adj) for_tile(Rg, Pa.Y, [&](int t, int ri, size_t gi) { cp_async4(sm + oga + t, Pa.gK + gi, true); });
  cp_async_wait_all();
  if (adj) for_region(Rg, [&](int i, int x, int y) { sm[NB * i + 5] = mul(sm[NB * i + 6], sm[NB * i + 3]); });
  __syncthreads();
  const WaveRect Rt(Pa, Rg);
  const int srci = wave_src_index(Pf, Rg);
  const int nt = (int)blockDim.x;
  const int tx0 = Rg.bx0 - Rg.rx0 - Rt.cx0, ty0 = Rg.by0 - Rg.ry0 - Rt.cy0;
  for (int s = 0; s < H; ++s) {
    const int p = s & 1;
    const bool fs = s < Pf.k, as = s < Pa.k;
    const float sn = (fs && srci >= 0) ? Pf.src[Pf.n0 + s] : 0.0f;
    float* Ls = fs ? Pf.lst + (size_t)s * Pf.cells : nullptr;
    const float* Ln = as ? Pa.lsts + (size_t)(Pa.ntop - s) * Pa.cells : nullptr;
    RectWalk wk(Rt.W, nt);
    for (int q = threadIdx.x; q < Rt.count; q += nt, wk.next()) {
      const int i = (Rt.cx0 + wk.row) * RY + Rt.cy0 + wk.col;
      float* pc = sm + NB * i;
      const int ox = wk.row - tx0, oy = wk.col - ty0;
      const bool tile = ox >= 0 && ox < Rg.OX && oy >= 0 && oy < Rg.OY;
      if (fs) {  // u^{n+1} = 2 u^n - u^{n-1} + K o L(u^n) (+ source)
        const float lap = lap5n<NB>(pc + (1 - p), rs, Pf.w);
        float v = sub(mul(2.0f, pc[1 - p]), pc[p]);
        v = add(v, mul(pc[6], lap));
        if (i == srci) v = add(v, sn);
        pc[p] = v;
        if (tile) Ls[(size_t)(Rg.bx0 + ox) * Pf.Y + Rg.by0 + oy] = lap;
      }
      if (as) {
        const float m1 = pc[3 - p];
        if (tile) {  // dJ/dK += mu^{n+1} o L(u^n)
          const int t = oga + ox * Rg.OY + oy;
          sm[t] = add(sm[t], mul(m1, __ldg(Ln + (size_t)(Rg.bx0 + ox) * Pa.Y + Rg.by0 + oy)));
        }
        // mu^n = 2 mu^{n+1} - mu^{n+2} + L(K o mu^{n+1})
        const float acc = lap5n<NB>(pc + (5 - p), rs, Pa.w);
        const float v = add(sub(mul(2.0f, m1), pc[2 + p]), acc);
        pc[2 + p] = v;
        pc[4 + p] = mul(pc[6], v);
      }
    }
    __syncthreads();
  }
  if (adj) for_tile(Rg, Pa.Y, [&](int t, int ri, size_t gi) { Pa.gK[gi] = sm[oga + t]; });
  const int fw = (Pf.k & 1) ? 0 : 1, aw = (Pa.k & 1) ? 0 : 1;  // levels the last steps wrote
  for_tile(Rg, Pa.Y, [&](int t, int ri, size_t gi) {
    const float* pc = sm + NB * ri;
    if (fwd) {
      um_out[gi] = pc[1 - fw];
      u0_out[gi] = pc[fw];
    }
    if (adj) {
      m1_out[gi] = pc[2 + aw];
      m2_out[gi] = pc[3 - aw];
    }
  });
}

// ---- paired launch, packed: two cells per register slot --------------------
// The paired launch's register-list form, each slot holding two cells of
// the rectangle walked at full region width: warp w's slot c covers the 64
// consecutive cells from 64 (w + c W) (W warps), lane l taking cells l and
// l + 32 of them, so each half of a slot reads 32 consecutive cells (odd
// NB-float stride: no bank conflicts).  Both chains' arithmetic runs as packed
// pairs -- each product __ffma2_rn with a run-time -0 addend (the exactly
// rounded product), each sum __fadd2_rn, a - b as a + (-b) -- so each half is
// the scalar kernel's operation sequence and the results are bit-identical to
// it.  A half outside the rectangle computes on an in-region cell (its own, or
// the first rectangle cell past the last row) and stores nothing.
template <int MAXP>
struct WavePairs {
  int ri[MAXP][2];    // region index (always inside the region)
  int gi[MAXP][2];    // array index of a tile cell; 0 (a valid address) for the other cells
  int dist[MAXP][2];  // distance from the tile; 1 << 20 for a half outside the rectangle
  unsigned tile;      // bit 2c + h: half h of slot c holds a tile cell
  __device__ bool is_tile(int c, int h) const { return (tile >> (2 * c + h)) & 1u; }
  __device__ WavePairs(const WaveRect& Rt, const WaveRegion& Rg, int Y) {
    const int nw = (int)blockDim.x >> 5, w = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
    const int tx0 = Rg.bx0 - Rg.rx0 - Rt.cx0, ty0 = Rg.by0 - Rg.ry0;
    const int n = Rt.NR * Rg.RY;
    const int ri_safe = Rt.cx0 * Rg.RY + Rt.cy0;  // a rectangle cell: every neighbour inside the region
    tile = 0;
#pragma unroll
    for (int c = 0; c < MAXP; ++c) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int q = 64 * (w + c * nw) + lane + 32 * h;  // cell of the walk: row q / RY, region column q % RY
        ri[c][h] = ri_safe;
        gi[c][h] = 0;
        dist[c][h] = 1 << 20;
        if (q < n) {
          const int row = q / Rg.RY, col = q - row * Rg.RY;
          ri[c][h] = (Rt.cx0 + row) * Rg.RY + col;  // rows cx0 .. cx0+NR-1: neighbours inside the region
          if (col >= Rt.cy0 && col < Rt.cy0 + Rt.W) {
            const int ox = row - tx0, oy = col - ty0;
            if (ox >= 0 && ox < Rg.OX && oy >= 0 && oy < Rg.OY) {
              gi[c][h] = (Rg.bx0 + ox) * Y + Rg.by0 + oy;
              tile |= 1u << (2 * c + h);
            }
            dist[c][h] = max(max(max(-ox, ox - (Rg.OX - 1)), max(-oy, oy - (Rg.OY - 1))), 0);
          }
        }
      }
    }
  }
};

__device__ __forceinline__ float2 wv_neg(float2 a) { return make_float2(-a.x, -a.y); }

template <int MAXP>
__global__ void __launch_bounds__(1024) wave_pair2_tb_kernel(const float* __restrict__ um_in,
                                                              const float* __restrict__ u0_in,
                                                              float* __restrict__ um_out, float* __restrict__ u0_out,
                                                              const float* __restrict__ m1_in,
                                                              const float* __restrict__ m2_in,
                                                              float* __restrict__ m1_out, float* __restrict__ m2_out,
                                                              const float* __restrict__ Kf, const WaveParams Pf,
                                                              const WaveParams Pa, const float negzero) {
  extern __shared__ __align__(16) float sm[];
  constexpr int NB = 7;
  const int H = max(Pf.k, Pa.k);
  const WaveRegion Rg(Pa, H);
  const int RY = Rg.RY, rs = NB * RY;
  const bool fwd = Pf.k > 0, adj = Pa.k > 0;
  for_region(Rg, [&](int i, int x, int y) {
    const size_t gi = (size_t)x * Pa.Y + y;
    const bool in = wave_inside(Pa, x, y);
    float* pc = sm + NB * i;
    cp_async4(pc + 6, Kf + gi, true);
    if (fwd) {
      cp_async4(pc, um_in + gi, in);
      cp_async4(pc + 1, u0_in + gi, in);
    }
    if (adj) {
      cp_async4(pc + 2, m2_in + gi, in);
      cp_async4(pc + 3, m1_in + gi, in);
      pc[4] = 0.0f;
    }
  });
  cp_async_wait_all();
  if (adj) for_region(Rg, [&](int i, int x, int y) { sm[NB * i + 5] = mul(sm[NB * i + 6], sm[NB * i + 3]); });
  __syncthreads();
  const WaveRect Rt(Pa, Rg);
  const int srci = wave_src_index(Pf, Rg);
  const WavePairs<MAXP> C(Rt, Rg, Pa.Y);
  const float2 nz2 = make_float2(negzero, negzero), two2 = make_float2(2.0f, 2.0f), zero2 = make_float2(0.0f, 0.0f);
  auto M2 = [&](float2 a, float2 b) { return __ffma2_rn(a, b, nz2); };
  float2 wf[3], wa[3];
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    wf[t] = make_float2(Pf.w[t], Pf.w[t]);
    wa[t] = make_float2(Pa.w[t], Pa.w[t]);
  }
  // the reference's 5-point sum (lap5n): x taps low to high, then y taps, from 0
  auto lap2 = [&](const float* p0, const float* p1, const float2 (&w)[3]) {
    auto ld = [&](int o) { return make_float2(p0[o], p1[o]); };
    float2 acc = __fadd2_rn(zero2, M2(w[0], ld(-rs)));
    acc = __fadd2_rn(acc, M2(w[1], ld(0)));
    acc = __fadd2_rn(acc, M2(w[2], ld(rs)));
    acc = __fadd2_rn(acc, M2(w[0], ld(-NB)));
    acc = __fadd2_rn(acc, M2(w[1], ld(0)));
    return __fadd2_rn(acc, M2(w[2], ld(NB)));
  };
  float2 ga[MAXP], lv[MAXP], kc[MAXP];
#pragma unroll
  for (int c = 0; c < MAXP; ++c) {
    ga[c] = zero2;
    lv[c] = zero2;
    kc[c] = make_float2(sm[NB * C.ri[c][0] + 6], sm[NB * C.ri[c][1] + 6]);
    if (adj) {
      const float* L0 = Pa.lsts + (size_t)Pa.ntop * Pa.cells;
      ga[c] = make_float2(C.is_tile(c, 0) ? Pa.gK[C.gi[c][0]] : 0.0f, C.is_tile(c, 1) ? Pa.gK[C.gi[c][1]] : 0.0f);
      lv[c] = make_float2(__ldg(L0 + C.gi[c][0]), __ldg(L0 + C.gi[c][1]));
    }
  }
  auto step = [&](auto PAR, int s) {
    constexpr int p = decltype(PAR)::value;
    const bool fs = s < Pf.k;
    const float sn = (fs && srci >= 0) ? Pf.src[Pf.n0 + s] : 0.0f;
    float* Ls = fs ? Pf.lst + (size_t)s * Pf.cells : nullptr;
    const int freach = Pf.k - 1 - s, areach = Pa.k - 1 - s;  // negative past a chain's last step
#pragma unroll
    for (int c = 0; c < MAXP; ++c) {
      float* p0 = sm + NB * C.ri[c][0];
      float* p1 = sm + NB * C.ri[c][1];
      const bool f0 = C.dist[c][0] <= freach, f1 = C.dist[c][1] <= freach;
      if (f0 || f1) {  // u^{n+1} = 2 u^n - u^{n-1} + K o L(u^n) (+ source)
        const float2 lap = lap2(p0 + (1 - p), p1 + (1 - p), wf);
        float2 v = __fadd2_rn(M2(two2, make_float2(p0[1 - p], p1[1 - p])), wv_neg(make_float2(p0[p], p1[p])));
        v = __fadd2_rn(v, M2(kc[c], lap));
        if (C.ri[c][0] == srci) v.x = add(v.x, sn);
        if (C.ri[c][1] == srci) v.y = add(v.y, sn);
        if (f0) p0[p] = v.x;
        if (f1) p1[p] = v.y;
        st_global_if(Ls + C.gi[c][0], lap.x, f0 && C.is_tile(c, 0));
        st_global_if(Ls + C.gi[c][1], lap.y, f1 && C.is_tile(c, 1));
      }
      const bool a0 = C.dist[c][0] <= areach, a1 = C.dist[c][1] <= areach;
      if (a0 || a1) {  // mu^n = 2 mu^{n+1} - mu^{n+2} + L(K o mu^{n+1}); dJ/dK += mu^{n+1} o L(u^n)
        const float2 m1 = make_float2(p0[3 - p], p1[3 - p]);
        ga[c] = __fadd2_rn(ga[c], M2(m1, lv[c]));  // a tile half is always in reach: no other half's sum is kept
        const float2 acc = lap2(p0 + (5 - p), p1 + (5 - p), wa);
        const float2 v =
            __fadd2_rn(__fadd2_rn(M2(two2, m1), wv_neg(make_float2(p0[2 + p], p1[2 + p]))), acc);
        const float2 km = M2(kc[c], v);
        if (a0) {
          p0[2 + p] = v.x;
          p0[4 + p] = km.x;
        }
        if (a1) {
          p1[2 + p] = v.y;
          p1[4 + p] = km.y;
        }
      }
    }
    if (s + 1 < Pa.k) {  // the next step's L(u^n), in flight across the barrier
      const float* L1 = Pa.lsts + (size_t)(Pa.ntop - s - 1) * Pa.cells;
#pragma unroll
      for (int c = 0; c < MAXP; ++c) lv[c] = make_float2(__ldg(L1 + C.gi[c][0]), __ldg(L1 + C.gi[c][1]));
    }
    __syncthreads();
  };
  for (int s = 0; s < H; s += 2) {
    step(IC<0>{}, s);
    if (s + 1 < H) step(IC<1>{}, s + 1);
  }
  if (adj) {
#pragma unroll
    for (int c = 0; c < MAXP; ++c) {
      if (C.is_tile(c, 0)) Pa.gK[C.gi[c][0]] = ga[c].x;
      if (C.is_tile(c, 1)) Pa.gK[C.gi[c][1]] = ga[c].y;
    }
  }
  const int fw = (Pf.k & 1) ? 0 : 1, aw = (Pa.k & 1) ? 0 : 1;  // levels the last steps wrote
  for_tile(Rg, Pa.Y, [&](int t, int ri, size_t gi) {
    const float* pc = sm + NB * ri;
    if (fwd) {
      um_out[gi] = pc[1 - fw];
      u0_out[gi] = pc[fw];
    }
    if (adj) {
      m1_out[gi] = pc[2 + aw];
      m2_out[gi] = pc[3 - aw];
    }
  });
}

}  // namespace pde
