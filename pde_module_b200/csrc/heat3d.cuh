// Fused 3D heat rollout: boundary fill + Laplacian + forward Euler, K time
// steps per pass over HBM (temporal blocking), 2.5D streaming along X.
//
// Step (examples/2D_Heat_Equation.py:57-65 on a 3D grid, exact arithmetic):
//   u2 = BC(u);  u' = u2 + dt*(alpha*Lap(u2)) on stencil cells, u2 elsewhere.
//
// Tiling.  Tiles of (y, z) columns cover the whole array, ghost layers
// included (balanced sizes, at most TYM x TZM); a block holds its tile plus a
// halo of H = K*R + 1 cells ("region", clipped to the array) and marches along
// X over a chunk of planes.  Level s (s = 0..K) is the field after s steps of
// the pass; at loop iteration i level 0 receives plane i and level s computes
// plane i - s*R, so every plane a level reads was written at least one
// iteration earlier and ONE block barrier per plane orders all levels.
// Level s is valid on the region cells at least s*R from a cut edge of the
// region (the tile, at level K): what they read was valid at level s-1.
//
// Storage.  A region row is stored from an even float (the row's first cell
// rounded down), so a plane is a sequence of float pairs.  Pairs are dealt to
// warps in "warp tiles" of 8 rows x 4 pairs (lane = 4 * row + pair), warp w
// taking tiles w + c*W: cells at the array's boundary then fall into a few
// warps, and the rest run a path with no boundary test.  Per level each thread keeps its pairs' boundary-filled values for
// the last 2R+1 planes in registers (X taps, a queue rotated each plane).  Y and
// Z taps come from the plane of the level below in shared memory: level 0's
// plane is the cp.async staging slot (4-byte copies: any row pitch), levels
// 1..K-1 have rings of R+1 planes.  Every plane slot has R guard rows on both
// sides, so a pair computed outside its level's window (its result unused)
// reads inside its own slot.
//
// Arithmetic.  A pair advances with packed f32x2 operations, each lane rounded
// exactly as one scalar operation of the reference order (axes ascending, taps
// low to high, alpha last, then Euler): products are __ffma2_rn with a run-time
// -0 addend (the correctly rounded product, and an FMA the compiler cannot fuse
// with the add that follows), sums __fadd2_rn.  Results equal the step-by-step
// operator chain bit for bit (up to the sign of an exact zero: the leading
// 0 + w*u of the sum is skipped).
//
// Boundary fill (functional_boundary.py:343-400 through the compiled rules,
// fused.cuh bc_eval semantics), done when a level produces a plane:
//  * a node takes the value of the last Dirichlet group containing it;
//  * a first-layer ghost along Y or Z is written by the owner of its adjacent
//    cell (two cells inward), from that cell's pre-boundary value; the ghost's
//    owner leaves it alone;
//  * the ghost plane x = g-1 reads plane g+1 of the same level: its value is
//    set in the owner's register queue when plane g+1 is computed (with R = 1
//    the final level writes plane g-1 one plane late, beside plane g); the
//    ghost plane x = X-g reads plane X-g-2, whose ghost values are kept in a
//    per-level shared "stash" plane until plane X-g is produced.
// What a cell does is packed per work item into one descriptor per X plane
// class (x = g, the planes between, x = X-1-g), so boundary cells cost a few
// shared-memory reads and stores; a thread whose pairs need none of it runs a
// path without any boundary test.
#pragma once
#include "common.cuh"

namespace pde {

// Packed helpers on float2 (register pairs the compiler allocates itself).
__device__ __forceinline__ float2 h3_mul(float2 a, float2 b, float2 nz) { return __ffma2_rn(a, b, nz); }
__device__ __forceinline__ float2 h3_add(float2 a, float2 b) { return __fadd2_rn(a, b); }

struct H3Params {
  int X, Y, Z, g;
  int ny_t, nz_t, ntiles;  // tiles per axis: tile t covers [t*n/nt, (t+1)*n/nt)
  int nch, nitems;         // X chunks (chunk c covers [c*X/nch, (c+1)*X/nch)); items = ntiles x nch, chunk-major
  float w[5];
  float alpha, dt;
  float negzero;           // -0.0f: the addend of the packed products (must not be a compile-time constant)
  double t0, tstep;        // ramp groups: level s fills the boundary at fp32(t0 + (n0 + s)*tstep)
  int n0;
};

template <int R, int K, int N, int TYM, int TZM, int T>
struct H3Cfg {
  static constexpr int H = K * R + 1;                     // region halo
  static constexpr int RYM = TYM + 2 * H;                 // region rows (max)
  static constexpr int PW = ((TZM + 2 * H) * N + 2 + 7) & ~7;  // row width (floats): row + even-start lead
  // Row pitch: 8 mod 16 floats, so the four rows of a half warp's pair loads
  // (lanes 4r..4r+3 read floats 8w..8w+7 of row r) fall in four distinct bank octets.
  static constexpr int P = (PW % 16 == 0) ? PW + 8 : PW;
  static constexpr int W = T / 32;                        // warps
  static constexpr int NWC = PW / 8, NWR = (RYM + 7) / 8;  // warp tiles (8 rows x 8 floats) per row / column
  static constexpr int NWT = NWR * NWC;
  static constexpr int C = (NWT + W - 1) / W;             // pairs per thread (warp tiles per warp)
  static constexpr int PLANE = NWR * 8 * P;               // floats of a plane (rows rounded up to 8)
  static constexpr int G0 = R * P;                        // guard floats before a plane's first row
  static constexpr int PS = (PLANE + 2 * R * P + 3) & ~3;  // plane slot stride (floats)
  static constexpr int PF = 3;                            // planes in flight ahead of level 0
  static constexpr int S = PF + R + 1;                    // staging slots
  static constexpr int NB = (K - 1) * (R + 1);            // ring planes of levels 1..K-1
  static constexpr int Q = 2 * R + 1;                     // register queue length
  static constexpr int NPL = S + NB + K;                  // + one stash plane per level 0..K-1
  static constexpr int MINB = T <= 256 ? 2 : 1;           // resident blocks per SM the registers are capped for
  static constexpr size_t SMEM = (size_t)NPL * PS * 4 + (size_t)3 * PLANE * 4 + sizeof(PdeBCRules) +
                                 (size_t)K * PDE_MAX_GROUPS * 4;
  static_assert(2 * C <= 32, "lane masks");
  static_assert(T % 32 == 0, "whole warps");
  static_assert(SMEM <= 227 * 1024, "shared memory per block");
  static_assert(K >= 1 && K <= 4, "steps per pass");
};

__device__ __forceinline__ int h3_cls(int i, int n, int g) { return i == g ? 0 : (i == n - 1 - g ? 2 : 1); }

// Ghost value of group gi with the value of the current level (fused.cuh ghost_value).
__device__ __forceinline__ float h3_ghost(const PdeBCRules& Rl, const float* gv, int gi, int inc, float a) {
  const float v = gv[gi];
  if (Rl.group[gi].type == PDE_BC_DIRICHLET) return sub(mul(2.0f, v), a);
  return add(mul(mul((float)(-2 * inc), Rl.dx32), v), a);
}

// Boundary work of a cell on node-range planes of class cx (0: x = g,
// 1: g < x < X-1-g, 2: x = X-1-g), 32 bits (group ids stored + 1, 0 = none):
//   [4:0]   Dirichlet node value the cell takes
//   [5]     first-layer Y/Z ghost written by its adjacent cell's owner
//   [10:6], [15:11], [20:16], [25:21]: ghost this cell writes two cells away at
//           -Y (inc +1), +Y (inc -1), -Z (inc +1), +Z (inc -1)
//   [30:26] cx = 0: the cell's ghost on plane g-1 (written when plane g+1 is
//           produced); cx = 2: its ghost on plane X-g (from plane X-g-2)
__device__ __forceinline__ uint32_t h3_desc(const PdeBCRules& Rl, int cx, int Y, int Z, int g, int N, int y, int zv,
                                            int ya, int yb, int zlo, int zhi) {
  const int z = zv / N, v = zv - z * N;
  const bool yin = y >= g && y <= Y - 1 - g, zin = z >= g && z <= Z - 1 - g;
  const int cy = h3_cls(y, Y, g), cz = h3_cls(z, Z, g);
  const int kx = cx * 9;
  uint32_t d = 0;
  if (yin && zin) {
    const int Kc = kx + cy * 3 + cz;
    if (Kc != 13) {
      const int gi = Rl.node_group[Kc];
      if (gi >= 0 && ((Rl.group[gi].comp_mask >> v) & 1u)) d |= (uint32_t)(gi + 1);
    }
    if (cx != 1) d |= (uint32_t)(Rl.ghost_group[kx + cy * 3 + cz][0][v] + 1) << 26;
  }
  if ((y == g - 1 || y == Y - g) && zin && Rl.ghost_group[kx + (y == g - 1 ? 0 : 2) * 3 + cz][1][v] >= 0) d |= 32u;
  if ((z == g - 1 || z == Z - g) && yin && Rl.ghost_group[kx + cy * 3 + (z == g - 1 ? 0 : 2)][2][v] >= 0) d |= 32u;
  if (zin) {
    if (y == g + 1 && y - 2 >= ya) d |= (uint32_t)(Rl.ghost_group[kx + 0 * 3 + cz][1][v] + 1) << 6;
    if (y == Y - g - 2 && y + 2 < yb) d |= (uint32_t)(Rl.ghost_group[kx + 2 * 3 + cz][1][v] + 1) << 11;
  }
  if (yin) {
    if (z == g + 1 && zv - 2 * N >= zlo) d |= (uint32_t)(Rl.ghost_group[kx + cy * 3 + 0][2][v] + 1) << 16;
    if (z == Z - g - 2 && zv + 2 * N < zhi) d |= (uint32_t)(Rl.ghost_group[kx + cy * 3 + 2][2][v] + 1) << 21;
  }
  return d;
}

// In-plane boundary fill of one cell on a node-range plane from its descriptor
// d: writes the ghosts the cell fills, then (unless another thread writes the
// cell) its boundary-filled value to Bs[r]; returns whether it did (*u2).
template <int PP, int N>
__device__ __forceinline__ bool h3_apply(uint32_t d, const PdeBCRules& Rl, const float* gv, float u, float* Bs, int r,
                                         float* u2) {
  if (const uint32_t gi = (d >> 6) & 31u) Bs[r - 2 * PP] = h3_ghost(Rl, gv, (int)gi - 1, 1, u);
  if (const uint32_t gi = (d >> 11) & 31u) Bs[r + 2 * PP] = h3_ghost(Rl, gv, (int)gi - 1, -1, u);
  if (const uint32_t gi = (d >> 16) & 31u) Bs[r - 2 * N] = h3_ghost(Rl, gv, (int)gi - 1, 1, u);
  if (const uint32_t gi = (d >> 21) & 31u) Bs[r + 2 * N] = h3_ghost(Rl, gv, (int)gi - 1, -1, u);
  if (d & 32u) return false;
  const uint32_t gn = d & 31u;
  *u2 = gn ? gv[gn - 1] : u;
  Bs[r] = *u2;
  return true;
}

// Z taps (cells r + d*N, r + 1 + d*N for d = t - R) of the pair at float r of
// plane B; zt[R] is the pair itself (cen).  Even offsets are aligned pairs.
template <int R, int N>
__device__ __forceinline__ void h3_ztaps(const float* B, int r, float2 cen, float2 (&zt)[2 * R + 1]) {
  zt[R] = cen;
  if constexpr (N == 1 && R == 2) {
    const float2 m = *reinterpret_cast<const float2*>(B + r - 2), p = *reinterpret_cast<const float2*>(B + r + 2);
    zt[0] = m;
    zt[1] = make_float2(m.y, cen.x);
    zt[3] = make_float2(cen.y, p.x);
    zt[4] = p;
  } else {
#pragma unroll
    for (int t = 0; t < 2 * R + 1; ++t) {
      if (t == R) continue;
      const int o = (t - R) * N;
      if ((o & 1) == 0) zt[t] = *reinterpret_cast<const float2*>(B + r + o);
      else if (o == -1) zt[t] = make_float2(B[r - 1], cen.x);
      else if (o == 1) zt[t] = make_float2(cen.y, B[r + 2]);
      else zt[t] = make_float2(B[r + o], B[r + o + 1]);
    }
  }
}

template <int R, int K, int N, int TYM, int TZM, int T>
__global__ void __launch_bounds__(T, (H3Cfg<R, K, N, TYM, TZM, T>::MINB))
    heat3d_kernel(const float* __restrict__ in, float* __restrict__ out, const H3Params P,
                  const __grid_constant__ PdeBCRules rules) {
  using Cf = H3Cfg<R, K, N, TYM, TZM, T>;
  constexpr int PP = Cf::P, PS = Cf::PS, PL = Cf::PLANE, C = Cf::C, S = Cf::S, Q = Cf::Q, H = Cf::H, PF = Cf::PF;
  constexpr int T2 = 2 * R + 1;
  extern __shared__ __align__(16) float sm[];
  float* const stage = sm + Cf::G0;                        // level 0 slot j: stage + j*PS
  float* const ring = sm + S * PS + Cf::G0;                // level s in 1..K-1, slot j: ring + ((s-1)*(R+1) + j)*PS
  float* const stash = sm + (S + Cf::NB) * PS + Cf::G0;    // level s: stash + s*PS
  uint32_t* const desc = reinterpret_cast<uint32_t*>(sm + Cf::NPL * PS);  // [cx][PLANE], this item
  PdeBCRules* const Rl = reinterpret_cast<PdeBCRules*>(desc + 3 * PL);
  float* const gval = reinterpret_cast<float*>(Rl + 1);    // [K][PDE_MAX_GROUPS]: group values per level

  pdl_launch_dependents();
  {
    const int* src = reinterpret_cast<const int*>(&rules);
    int* dst = reinterpret_cast<int*>(Rl);
    for (int i = threadIdx.x; i < (int)(sizeof(PdeBCRules) / 4); i += T) dst[i] = src[i];
    for (int i = threadIdx.x; i < K * PDE_MAX_GROUPS; i += T) {
      const int s = i / PDE_MAX_GROUPS, gi = i - s * PDE_MAX_GROUPS;
      float v = 0.0f;
      if (gi < rules.ngroups) {
        const PdeBCGroupParam& G = rules.group[gi];
        v = G.value;
        if (G.func == PDE_BC_FUNC_RAMP) {
          const float t = step_time(P.t0, P.tstep, P.n0 + s);
          v = mul(fminf(__fdiv_rn(t, G.t_max), 1.0f), G.value);
        }
      }
      gval[i] = v;
    }
  }
  __syncthreads();

  const int X = P.X, Y = P.Y, Z = P.Z, g = P.g;
  const int ZN = Z * N;
  const long long YZN = (long long)Y * ZN;
  const int tid = threadIdx.x;
  float2 w2[T2];
#pragma unroll
  for (int t = 0; t < T2; ++t) w2[t] = make_float2(P.w[t], P.w[t]);
  const float2 al2 = make_float2(P.alpha, P.alpha), dt2 = make_float2(P.dt, P.dt),
               nz2 = make_float2(P.negzero, P.negzero);

  // float offset in a plane of each of this thread's pairs (PLANE: past the
  // plane, for the slots of warp tiles beyond the last)
  int rc[C];
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int wt = (tid >> 5) + c * Cf::W, lane = tid & 31;
    const int wr = wt / Cf::NWC, wc = wt - wr * Cf::NWC;
    rc[c] = wt < Cf::NWT ? (wr * 8 + (lane >> 2)) * PP + 2 * (wc * 4 + (lane & 3)) : PL;
  }

  pdl_wait();

  // Work items in order of cost: tiles at the Y/Z edges of the array (boundary
  // work) first, then the others, chunk-major within each class; round k of
  // the persistent grid deals items k*G .. k*G+G-1 to the blocks forward on
  // even rounds and backward on odd ones, so every block gets a like share.
  const int G = gridDim.x, nyt = P.ny_t, nzt = P.nz_t;
  const bool all_edge = nyt <= 2 || nzt <= 2;
  const int ne = all_edge ? P.ntiles : 2 * nzt + 2 * (nyt - 2), ni = P.ntiles - ne;
  for (int kr = 0;; ++kr) {
    const int item = kr * G + ((kr & 1) ? G - 1 - (int)blockIdx.x : (int)blockIdx.x);
    if (item >= P.nitems) break;
    int ch, ty, tz;
    if (item < ne * P.nch) {
      ch = item / ne;
      const int e = item - ch * ne;
      if (all_edge) { ty = e / nzt; tz = e - ty * nzt; }
      else if (e < nzt) { ty = 0; tz = e; }
      else if (e < 2 * nzt) { ty = nyt - 1; tz = e - nzt; }
      else { const int m = e - 2 * nzt; ty = 1 + (m >> 1); tz = (m & 1) ? nzt - 1 : 0; }
    } else {
      const int j = item - ne * P.nch;
      ch = j / ni;
      const int t2 = j - ch * ni;
      ty = 1 + t2 / (nzt - 2);
      tz = 1 + t2 % (nzt - 2);
    }
    const int y0 = (int)((long long)ty * Y / P.ny_t), y1 = (int)((long long)(ty + 1) * Y / P.ny_t);
    const int z0 = (int)((long long)tz * Z / P.nz_t), z1 = (int)((long long)(tz + 1) * Z / P.nz_t);
    const int ya = max(0, y0 - H), yb = min(Y, y1 + H);
    const int za = max(0, z0 - H), zb = min(Z, z1 + H);
    const int zlo = za * N, zhi = zb * N, zr0 = zlo & ~1;  // region row floats [zlo, zhi), stored from zr0
    const int x0 = (int)((long long)ch * X / P.nch), x1 = (int)((long long)(ch + 1) * X / P.nch);
    const int xa = max(0, x0 - H);              // first plane loaded
    const int xl = min(X - 1, x1 - 1 + K * R);  // last plane loaded
    const int ilast = x1 - 1 + K * R;           // last iteration
    const bool lowx = xa <= g + 1, highx = xl >= X - g - 2;  // the item reaches the X boundary planes

    // lane masks (bit 2c+l: lane l of pair c): active per level, fast (no boundary
    // work on planes g+2..X-g-3), first-layer Y/Z ghost column, stencil column
    uint32_t am[K + 1], fm = 0, gm = 0, scm = 0;
    uint32_t wtm = 0;  // bit c: pair c's warp tile holds region cells (the same in every lane of a warp)
#pragma unroll
    for (int s = 0; s <= K; ++s) am[s] = 0;
    int goff[C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const int r = rc[c];
      const int ry = r / PP, rz = r - ry * PP;
      {
        const int wt = (tid >> 5) + c * Cf::W;
        const int wr = wt / Cf::NWC, wc = wt - wr * Cf::NWC;
        if (wt < Cf::NWT && ya + wr * 8 < yb && zr0 + wc * 8 < zhi) wtm |= 1u << c;
      }
      const int y = ya + ry;
      goff[c] = y * ZN + zr0 + rz;
#pragma unroll
      for (int l = 0; l < 2; ++l) {
        const int zv = zr0 + rz + l;
        if (r >= PL || y >= yb || zv < zlo || zv >= zhi) continue;
        const int z = zv / N;
        int d = 1 << 20;
        if (ya > 0) d = min(d, y - ya);
        if (yb < Y) d = min(d, yb - 1 - y);
        if (za > 0) d = min(d, z - za);
        if (zb < Z) d = min(d, zb - 1 - z);
        const bool tl = y >= y0 && y < y1 && z >= z0 && z < z1;
        const int act = tl ? K : min(K - 1, d / R);
        const uint32_t b = 1u << (2 * c + l);
#pragma unroll
        for (int s = 0; s <= K; ++s)
          if (s <= act) am[s] |= b;
        const bool fast = y >= g + 2 && y <= Y - g - 3 && z >= g + 2 && z <= Z - g - 3;
        if (fast) fm |= b;
        if (((y == g - 1 || y == Y - g) && z >= g && z <= Z - 1 - g) ||
            ((z == g - 1 || z == Z - g) && y >= g && y <= Y - 1 - g))
          gm |= b;
        if (y >= g && y < Y - g && z >= g && z < Z - g) scm |= b;
        desc[PL + r + l] = fast ? 0u : h3_desc(*Rl, 1, Y, Z, g, N, y, zv, ya, yb, zlo, zhi);
        if (lowx) desc[r + l] = h3_desc(*Rl, 0, Y, Z, g, N, y, zv, ya, yb, zlo, zhi);
        if (highx) desc[2 * PL + r + l] = h3_desc(*Rl, 2, Y, Z, g, N, y, zv, ya, yb, zlo, zhi);
      }
    }

    const bool allw = wtm == (1u << C) - 1u;  // every warp tile of this warp live: loops without per-pair tests

    // level-0 staging: plane p lives in slot (p - xa) % S; lanes outside the
    // region are zero filled without a read
    auto issue = [&](int p, int slot) {
      if (p <= xl) {
        float* dst = stage + slot * PS;
        const float* src = in + (long long)p * YZN;
#pragma unroll
        for (int c = 0; c < C; ++c) {  // dead warp tiles: zero fill past the plane, no read
          const int r = rc[c];
          const bool v0 = (am[0] >> (2 * c)) & 1u, v1 = (am[0] >> (2 * c + 1)) & 1u;
          const float* s0 = src + goff[c];
          if (v0 && v1 && (reinterpret_cast<uintptr_t>(s0) & 7u) == 0) {
            cp_async8(dst + r, s0);  // a whole aligned pair
          } else {
            cp_async4(dst + r, v0 ? s0 : in, v0);
            cp_async4(dst + r + 1, v1 ? s0 + 1 : in, v1);
          }
        }
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
#pragma unroll
    for (int j = 0; j < PF; ++j) issue(xa + j, j);

    float2 q[K][C][Q];
#pragma unroll
    for (int s = 0; s < K; ++s)
#pragma unroll
      for (int c = 0; c < C; ++c)
#pragma unroll
        for (int t = 0; t < Q; ++t) q[s][c][t] = make_float2(0.0f, 0.0f);

    auto setlane = [](float2& p, int l, float v) {
      if (l) p.y = v;
      else p.x = v;
    };
    // one step of a pair at plane x from level-(s-1) values: X taps from the
    // queue qp, Y/Z taps from plane Bp, centre cen
    auto core = [&](const float2 (&qp)[Q], const float* Bp, int r, float2 cen) -> float2 {
      float2 zt[T2];
      h3_ztaps<R, N>(Bp, r, cen, zt);
      float2 acc = h3_mul(w2[0], qp[2 * R], nz2);
#pragma unroll
      for (int t = 1; t < T2; ++t) acc = h3_add(acc, h3_mul(w2[t], qp[2 * R - t], nz2));
#pragma unroll
      for (int t = 0; t < T2; ++t)
        acc = h3_add(acc, h3_mul(w2[t], t == R ? cen : *reinterpret_cast<const float2*>(Bp + r + (t - R) * PP), nz2));
#pragma unroll
      for (int t = 0; t < T2; ++t) acc = h3_add(acc, h3_mul(w2[t], zt[t], nz2));
      return h3_add(cen, h3_mul(dt2, h3_mul(al2, acc, nz2), nz2));
    };
    // the same with ghost-column centres from Bp, non-stencil lanes keeping their centre
    auto step = [&](const float2 (&qp)[Q], const float* Bp, int r, int c, bool xst) -> float2 {
      float2 cen = qp[R];
      const uint32_t g2 = (gm >> (2 * c)) & 3u;
      if (g2) cen = make_float2((g2 & 1u) ? Bp[r] : cen.x, (g2 & 2u) ? Bp[r + 1] : cen.y);
      const float2 u = core(qp, Bp, r, cen);
      const uint32_t s2 = xst ? ((scm >> (2 * c)) & 3u) : 0u;
      return make_float2((s2 & 1u) ? u.x : cen.x, (s2 & 2u) ? u.y : cen.y);
    };
    // boundary fill of lane l of pair c at level s, plane x, pre-boundary value u
    // (level 0: read here from Bs unless another thread writes the cell)
    auto fill = [&](int s, int x, int c, int l, float u, bool level0, float* Bs, float2 (&qs)[Q]) {
      const int rr = rc[c] + l;
      const float* gv = gval + s * PDE_MAX_GROUPS;
      if (x >= g && x <= X - 1 - g) {
        const int cx = x == g ? 0 : (x == X - 1 - g ? 2 : 1);
        const uint32_t d = desc[cx * PL + rr];
        if (level0) u = (d & 32u) ? 0.0f : Bs[rr];
        if (x == g + 1)
          if (const uint32_t gi = (desc[rr] >> 26) & 31u) setlane(qs[2], l, h3_ghost(*Rl, gv, (int)gi - 1, 1, u));
        if (x == X - g - 2)
          if (const uint32_t gi = (desc[2 * PL + rr] >> 26) & 31u)
            stash[s * PS + rr] = h3_ghost(*Rl, gv, (int)gi - 1, -1, u);
        float u2;
        if (h3_apply<PP, N>(d, *Rl, gv, u, Bs, rr, &u2)) setlane(qs[0], l, u2);
      } else {
        if (level0) u = Bs[rr];
        if (x == X - g)
          if ((desc[2 * PL + rr] >> 26) & 31u) u = stash[s * PS + rr];
        if (!level0 || x == X - g) Bs[rr] = u;
        setlane(qs[0], l, u);
      }
    };

    int sl0 = 0;  // staging slot of plane i
    int rsl = 0;  // (i - xa) mod (R+1)
    for (int i = xa; i <= ilast; ++i) {
      asm volatile("cp.async.wait_group %0;\n" ::"n"(PF - 1) : "memory");
      __syncthreads();
      issue(i + PF, sl0 + PF < S ? sl0 + PF : sl0 + PF - S);
      auto rslot = [&](int m) { return (rsl + (R + 1) * (K + 1) - m) % (R + 1); };
      auto sslot = [&](int m) { return (sl0 + S * (K + 1) - m) % S; };

      // ---- level 0: plane i ----
#pragma unroll
      for (int c = 0; c < C; ++c)
#pragma unroll
        for (int t = Q - 1; t > 0; --t) q[0][c][t] = q[0][c][t - 1];
      if (i <= xl) {
        float* St = stage + sl0 * PS;
        const bool inx = i >= g + 2 && i <= X - g - 3;
        const uint32_t gen = inx ? ((am[0] & ~fm) | gm) : am[0];  // lanes with boundary work
        if (allw && !gm) {
#pragma unroll
          for (int c = 0; c < C; ++c) q[0][c][0] = *reinterpret_cast<const float2*>(St + rc[c]);
        } else {
#pragma unroll
          for (int c = 0; c < C; ++c)
            if (((wtm >> c) & 1u) && !((gm >> (2 * c)) & 3u)) q[0][c][0] = *reinterpret_cast<const float2*>(St + rc[c]);
        }
        if (gen) {
#pragma unroll
          for (int c = 0; c < C; ++c)
#pragma unroll
            for (int l = 0; l < 2; ++l)
              if ((gen >> (2 * c + l)) & 1u) fill(0, i, c, l, 0.0f, true, St, q[0][c]);
        }
      }

      // ---- levels 1..K-1: plane i - s*R ----
      static_for<1, K>([&](auto SS) {
        constexpr int s = decltype(SS)::value;
#pragma unroll
        for (int c = 0; c < C; ++c)
#pragma unroll
          for (int t = Q - 1; t > 0; --t) q[s][c][t] = q[s][c][t - 1];
        const int x = i - s * R;
        if (x < 0 || x >= X) return;
        const float* Bp = (s == 1) ? stage + sslot(R) * PS : ring + ((s - 2) * (R + 1) + rslot(s * R)) * PS;
        float* Bs = ring + ((s - 1) * (R + 1) + rslot(s * R)) * PS;
        const bool inx = x >= g + 2 && x <= X - g - 3;
        const bool xst = x >= g && x < X - g;
        const uint32_t gen = inx ? ((am[s] & ~fm) | gm) : am[s];
        if (!gen) {  // no boundary work in this thread's pairs
          if (allw) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
              const float2 u = core(q[s - 1][c], Bp, rc[c], q[s - 1][c][R]);
              q[s][c][0] = u;
              *reinterpret_cast<float2*>(Bs + rc[c]) = u;
            }
          } else {
#pragma unroll
            for (int c = 0; c < C; ++c) {
              if (!((wtm >> c) & 1u)) continue;
              const float2 u = core(q[s - 1][c], Bp, rc[c], q[s - 1][c][R]);
              q[s][c][0] = u;
              *reinterpret_cast<float2*>(Bs + rc[c]) = u;
            }
          }
          return;
        }
#pragma unroll
        for (int c = 0; c < C; ++c) {
          if (!((wtm >> c) & 1u)) continue;
          const int r = rc[c];
          if (!((gen >> (2 * c)) & 3u)) {
            const float2 u = core(q[s - 1][c], Bp, r, q[s - 1][c][R]);
            q[s][c][0] = u;
            *reinterpret_cast<float2*>(Bs + r) = u;
            continue;
          }
          const float2 u = step(q[s - 1][c], Bp, r, c, xst);
          q[s][c][0] = u;
#pragma unroll
          for (int l = 0; l < 2; ++l) {
            const float ul = l ? u.y : u.x;
            if ((gen >> (2 * c + l)) & 1u) fill(s, x, c, l, ul, false, Bs, q[s][c]);
            else if (!((gm >> (2 * c + l)) & 1u)) Bs[r + l] = ul;
          }
        }
      });

      // ---- level K: plane i - K*R, written to the output ----
      {
        const int x = i - K * R;
        if (x >= x0 && x < x1 && !(R == 1 && x == g - 1)) {  // R = 1: plane g-1 is written beside plane g
          const float* Bp = (K == 1) ? stage + sslot(R) * PS : ring + ((K - 2) * (R + 1) + rslot(K * R)) * PS;
          const bool inx = x >= g + 2 && x <= X - g - 3;
          const bool xst = x >= g && x < X - g;
          float* orow = out + (long long)x * YZN;
          if (inx && !gm && !(am[K] & ~fm)) {  // every output lane a stencil cell
            float2 u[C];
            if (allw) {
#pragma unroll
              for (int c = 0; c < C; ++c) u[c] = core(q[K - 1][c], Bp, rc[c], q[K - 1][c][R]);
            } else {
#pragma unroll
              for (int c = 0; c < C; ++c)
                if ((wtm >> c) & 1u) u[c] = core(q[K - 1][c], Bp, rc[c], q[K - 1][c][R]);
            }
#pragma unroll
            for (int c = 0; c < C; ++c) {
              if ((am[K] >> (2 * c)) & 1u) orow[goff[c]] = u[c].x;
              if ((am[K] >> (2 * c + 1)) & 1u) orow[goff[c] + 1] = u[c].y;
            }
          } else {
#pragma unroll
            for (int c = 0; c < C; ++c) {
              if (!((wtm >> c) & 1u)) continue;
              const float2 u = step(q[K - 1][c], Bp, rc[c], c, xst);
              if ((am[K] >> (2 * c)) & 1u) orow[goff[c]] = u.x;
              if ((am[K] >> (2 * c + 1)) & 1u) orow[goff[c] + 1] = u.y;
            }
          }
          if (R == 1 && x == g && x0 <= g - 1) {
            float* o2 = out + (long long)(g - 1) * YZN;
#pragma unroll
            for (int c = 0; c < C; ++c) {
              if ((am[K] >> (2 * c)) & 1u) o2[goff[c]] = q[K - 1][c][R + 1].x;
              if ((am[K] >> (2 * c + 1)) & 1u) o2[goff[c] + 1] = q[K - 1][c][R + 1].y;
            }
          }
        }
      }
      if (++sl0 == S) sl0 = 0;
      if (++rsl == R + 1) rsl = 0;
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();  // the next item reuses the staging, ring and descriptor planes
  }
}

}  // namespace pde
