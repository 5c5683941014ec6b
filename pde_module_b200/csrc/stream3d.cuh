// 2.5D streaming stencils for 3D grids with TMA-staged halo tiles.
//
// A block owns a (TY x TZ) tile of interior (y, z) columns and marches along
// X (the slowest axis) over a chunk of planes.  One producer warp brings each
// input plane of the tile (TY + 2R rows of TZ + 2R cells plus an alignment
// lead) into a ring of S shared-memory stages with 1D TMA bulk-tensor copies,
// one per row: the array's row pitch is arbitrary (e.g. 514 floats), so a 3D
// tensor map's 16-byte stride rule cannot be met.  Each stage has a "full"
// mbarrier (TMA bytes landed) and an "empty" mbarrier (every consumer warp is
// done with the plane); there is no block-wide barrier in the plane loop.
//
// Consumer threads own a z column and YPT consecutive rows.  X-direction taps
// come from a register queue of the thread's own column (a plane's centre
// values are read once, when the plane arrives); Y and Z taps come from the
// centre plane's stage, which is released right after use, so a stage is
// held only while its plane is the centre or newest plane.  Every product and
// sum is rounded separately, in the reference's order (axes ascending, taps
// low to high, alpha last): results equal the general kernels' bit for bit,
// up to the sign of an exactly-zero result (the leading 0 + w*u is skipped).
#pragma once
#include "common.cuh"
#include "tma.cuh"
#include <type_traits>

namespace pde {

// OP_HEAT: the heat step of a boundary-filled scalar field, u2 + dt*(alpha*L(u2)),
// on the Laplacian's tiles (exact arithmetic only)
enum { OP_LAP = 0, OP_GRAD = 1, OP_DIV = 2, OP_HEAT = 3 };

struct S3Params {
  int X, Y, Z, g;
  int ny_tiles, nz_tiles, ntiles;
  int chunk;            // planes per work item
  int nitems;           // ntiles x chunks, chunk-major
  int pp, pr;           // (Y*Z*CIN) mod 4, (Z*CIN) mod 4: row alignment lead
  float w[5];
  float alpha;
  float dt;             // OP_HEAT: the Euler step
  float* out;
  uint64_t wait_ns;     // bound of every mbarrier wait
  float negzero;        // -0.0f: the addend of the packed products (not a compile-time constant)
};

__host__ __device__ constexpr int round4(int v) { return (v + 3) & ~3; }

// Plane addressing: MAP_ROWS_GEN / MAP_ROWS_PP0 bring each tile row with its
// own 1D TMA copy (the lead of a row inside its 16-byte aligned copy varies
// with the plane in the GEN case, is fixed in the PP0 case); MAP_PAIRS views
// the array as (2*Z*CIN, Y/2, X) "double rows" (pitch 8*Z*CIN bytes, a
// multiple of 16 when Z is even), so a plane tile arrives as two 2D boxes:
// the even rows and the odd rows.
enum { MAP_ROWS_GEN = 0, MAP_ROWS_PP0 = 1, MAP_PAIRS = 2 };

// Arithmetic of one output row: MODE_EXACT follows the reference sum term by
// term (every product and sum rounded separately); MODE_FAST sums the taps
// that share a weight first and uses FMA with alpha folded into the weights.
enum { MODE_EXACT = 0, MODE_FAST = 1 };

template <int R, int OP, int CIN, int TZ, int TY, int YPT, int PREF, int MAPK = MAP_ROWS_PP0, int MODE = MODE_EXACT>
struct S3Cfg {
  // z pairs (scalar Laplacian or Grad, radius 2, double-row map, exact): a
  // consumer lane owns two adjacent z cells, an 8-byte aligned pair in every
  // stage row (the radius and every row lead are even), see s3_zpairs
  static constexpr bool LAPL = OP == OP_LAP || OP == OP_HEAT;  // Laplacian-shaped: one output per input float
  static constexpr bool ZP =
      (LAPL || OP == OP_GRAD) && CIN == 1 && R == 2 && MAPK == MAP_PAIRS && MODE == MODE_EXACT;
  static constexpr int LANES = ZP ? TZ / 2 : LAPL ? TZ * CIN : TZ;  // consumer threads per row group
  static constexpr int TYG = TY / YPT;                           // row groups
  static constexpr int NCONS = LANES * TYG;                      // consumer threads
  static constexpr int NCW = NCONS / 32;                         // consumer warps
  static constexpr int THREADS = NCONS + 32;                     // + one producer warp
  static constexpr int ROWS = TY + 2 * R;
  static constexpr int W = round4(3 + (TZ + 2 * R) * CIN);  // TMA box (floats)
  static constexpr int WP = (W + 31) & ~31;                 // smem row pitch: 128-byte aligned rows
  static constexpr int S = R + 1 + PREF;                    // stages: centre .. newest + prefetch
  // MAP_PAIRS: each half (even / odd rows) is a dense [ROWS/2][W] box, 128-byte aligned
  static constexpr int HALF = ((ROWS / 2) * W + 31) & ~31;
  static constexpr int STAGE_FLOATS = (MAPK == MAP_PAIRS) ? 2 * HALF : ROWS * WP;
  // Grad: the tile's TY output rows of a plane (3 TZ floats each, placed at the
  // row's offset within a 128-byte line: pitch 3 TZ + 32); two planes' buffers
  // where two blocks per SM still fit, else one (and a second barrier per plane)
  static constexpr int OROW = 3 * TZ + 32;
  // + 128: the base is rounded up to a 128-byte boundary at run time
  static constexpr size_t SMEM_BASE = (size_t)S * STAGE_FLOATS * 4 + (size_t)2 * S * 8 + 128;
  static constexpr int OBUFS = (SMEM_BASE + (size_t)2 * TY * OROW * 4 <= 113 * 1024) ? 2 : 1;
  static constexpr int OBUF_FLOATS = (OP == OP_GRAD) ? OBUFS * TY * OROW : 0;
  static constexpr size_t SMEM = SMEM_BASE + (size_t)OBUF_FLOATS * 4;
  static_assert(NCONS % 32 == 0, "whole consumer warps");
  static_assert(OP != OP_GRAD || TZ % 4 == 0, "grad staging rows: 16-byte multiple pitch");
  static_assert(W <= 256, "TMA box extent");
  static_assert(TY % YPT == 0, "rows per thread");
  static_assert(!ZP || TZ % 2 == 0, "z pairs");
  static_assert(OP != OP_HEAT || (CIN == 1 && MODE == MODE_EXACT), "heat step: scalar, exact");
};

struct FastW {
  float a[3];  // LAP: alpha*w[t] for the off-centre taps t < R (mirror t' = T-1-t); [R]: alpha*D*w[R]
};              // D1: alpha*w[t] for t > R (antisymmetric: w[T-1-t] = -w[t])

// Grad output of one plane: tile row t owns 3 TZ consecutive output floats.
// Every consumer thread calls this once per plane after staging its results in
// ob, row t at float (r0 + t dzr) mod 32 (the row's offset within a 128-byte
// line of the array, whose offset of row t is rf0 + 3 Z t); the consumers meet
// at a named barrier and store the rows.  Order 4 (BULK): one lane per row hands
// the row's 16-byte aligned body to the bulk-copy unit (smem and global
// offsets agree mod 16 bytes) and lanes store the head and tail floats.  Order
// 2: every warp stores whole rows as line-aligned 128-byte pieces, one line per
// store.  (Measured at 512^3 on B200: bulk rows 0.79 vs 0.72 of HBM at order
// 4, 0.78 vs 0.83 at order 2.)  Two buffers: a buffer is rewritten two planes
// later, after the next plane's barrier, before which every issuing lane has
// waited for its bulk copies to finish reading; one buffer: a second barrier
// (after that wait) follows the stores.
template <class C, int R, int TZ, int TY>
__device__ __forceinline__ void s3_grad_rows(const S3Params& P, const float* ob, size_t rf0, int r0, int dzr,
                                             int y0, int z0) {
  const int tid = threadIdx.x;
  constexpr bool BULK = (R >= 2);
  if constexpr (BULK) {
    fence_proxy_async_smem();  // the staged rows are read by the async proxy
    bulk_wait_read();          // this lane's bulk stores of two planes ago have read their buffer
  }
  asm volatile("bar.sync 1, %0;" ::"r"(C::NCONS) : "memory");
  const int wl = tid & 31;
  const int nf = 3 * min(TZ, P.Z - P.g - z0);  // floats of the row's interior cells
  for (int t = tid >> 5; t < TY && y0 + t < P.Y - P.g; t += C::NCW) {
    const int r = (r0 + t * dzr) & 31;  // the row's float offset in its 128-byte line
    if constexpr (BULK) {
      float* gr = P.out + rf0 + (size_t)t * 3 * P.Z;
      const float* sr = ob + t * C::OROW + r;
      const int h = min((4 - (r & 3)) & 3, nf);  // floats before the first 16-byte boundary
      const int body = (nf - h) & ~3;            // whole 16-byte units after them
      const int e = h + body;                    // the tail: floats e .. nf-1 (< 4)
      if (wl < h) gr[wl] = sr[wl];
      else if (wl >= 4 && wl - 4 < nf - e) gr[e + wl - 4] = sr[e + wl - 4];
      if (wl == 0 && body > 0) {
        bulk_store(gr + h, sr + h, (uint32_t)body * 4u);
        bulk_commit();
      }
    } else {
      constexpr int NL = 3 * TZ / 32 + 1;  // lines a row can touch
      const int a = wl - r;  // float of the row this lane stores in the row's first line
      float* gr = P.out + rf0 + (size_t)t * 3 * P.Z + a;
      const float* sr = ob + t * C::OROW + r + a;
      if (nf == 3 * TZ) {  // a whole row: only the first and last lines are partial
        if (a >= 0) gr[0] = sr[0];
#pragma unroll
        for (int i = 1; i < NL - 1; ++i) gr[32 * i] = sr[32 * i];
        if (a + 32 * (NL - 1) < nf) gr[32 * (NL - 1)] = sr[32 * (NL - 1)];
      } else {
#pragma unroll
        for (int i = 0; i < NL; ++i)
          if (a + 32 * i >= 0 && a + 32 * i < nf) gr[32 * i] = sr[32 * i];
      }
    }
  }
  if (C::OBUFS == 1) {
    if constexpr (BULK) bulk_wait_read();
    asm volatile("bar.sync 1, %0;" ::"r"(C::NCONS) : "memory");
  }
}

// Consumers with z pairs (S3Cfg::ZP: scalar Laplacian or Grad at radius 2):
// lane l owns the z cells z0 + 2l and z0 + 2l + 1 of YPT consecutive rows, an
// aligned float2 in every stage row, so its x-queue entries, centre-plane rows
// and z taps are 8-byte loads (the z taps of the pair, cells z-2 .. z+3, are
// the row's pairs at -2, 0, +2 and two pairs recombined in registers) and its
// two cells are summed as one packed pair: products __ffma2_rn with a -0
// addend (exactly rounded), sums __fadd2_rn, in the reference order (x, y, z
// taps low to high, alpha last), each lane the scalar kernels' operations.
// Grad stages the pair's six output floats as three 8-byte stores.
template <int R, int OP, int TZ, int TY, int YPT, int PREF>
__device__ __forceinline__ void s3_zpairs(const S3Params& P, float* smem, uint64_t* full, uint64_t* empty,
                                          float* obuf) {
  using C = S3Cfg<R, OP, 1, TZ, TY, YPT, PREF, MAP_PAIRS, MODE_EXACT>;
  static_assert(R == 2 && YPT % 2 == 0, "z pairs: radius 2, even rows per thread");
  constexpr int S = C::S, T = 2 * R + 1, M = YPT + 2 * R;
  const int tid = threadIdx.x;
  const int lane = tid % C::LANES, yg = tid / C::LANES;
  const bool warp_leader = (tid & 31) == 0;
  const int row0 = yg * YPT;  // even: window row m has the parity of m
  auto rowoff = [&](int m) { return (m & 1) * C::HALF + (m >> 1) * C::W; };
  auto ld2 = [](const float* p) { return *reinterpret_cast<const float2*>(p); };
  const float* smem_c = smem + (row0 >> 1) * C::W + R + 2 * lane;
  float2 w2[T];
#pragma unroll
  for (int t = 0; t < T; ++t) w2[t] = make_float2(P.w[t], P.w[t]);
  const float2 al2 = make_float2(P.alpha, P.alpha), nz2 = make_float2(P.negzero, P.negzero);
  const float2 dt2 = make_float2(P.dt, P.dt);
  auto M2 = [&](float2 a, float2 b) { return __ffma2_rn(a, b, nz2); };
  // pair stores (Laplacian) and pair staging (Grad: even line offsets) need an 8-byte aligned output
  const bool st2 = (reinterpret_cast<uintptr_t>(P.out) & 7u) == 0;

  bool dead = false;
  int ns = 0, nph = 0, cs = 0;  // newest plane's stage and parity, centre plane's stage
  auto adv = [&](int& st) { if (++st == S) st = 0; };
  auto wait_new = [&]() {
    if (!dead && !mbar_wait_bounded(&full[ns], (uint32_t)nph, P.wait_ns, &g_err)) {
      dead = true;
      flag_error(PDE_ERR_TIMEOUT);
    }
  };
  auto release = [&](int st) {
    __syncwarp();
    if (warp_leader) mbar_arrive(&empty[st]);
  };
  const int nx = P.X - 2 * P.g;
  const int oplane = P.Y * P.Z;
  int opc = 0;  // grad: planes stored so far (selects the staging buffer)
  const int obase = (int)((reinterpret_cast<uintptr_t>(P.out) >> 2) & 31u);  // grad: out's float offset in its line
  const int dzr = (3 * P.Z) & 31;  // grad: line offset step from one output row to the next

  for (int item = blockIdx.x; item < P.nitems; item += gridDim.x) {
    const int c = item / P.ntiles, tile = item - c * P.ntiles;
    const int xoff = c * P.chunk, len = min(P.chunk, nx - xoff);
    const int tz = tile % P.nz_tiles, ty = tile / P.nz_tiles;
    const int z0 = P.g + tz * TZ, y0 = P.g + ty * TY, xs = P.g + xoff;
    const int zc = z0 - R;
    const int off[2] = {zc & 3, (P.Z + zc) & 3};  // row lead by row parity (even)
    const int zcell = z0 + 2 * lane;
    unsigned vm0 = 0, vm1 = 0;  // rows whose first / second cell of the pair is interior
#pragma unroll
    for (int k = 0; k < YPT; ++k) {
      if (y0 + row0 + k >= P.Y - P.g) continue;
      if (zcell < P.Z - P.g) vm0 |= 1u << k;
      if (zcell + 1 < P.Z - P.g) vm1 |= 1u << k;
    }
    const bool all_rows = st2 && vm1 == (1u << YPT) - 1u;  // vm1 full implies vm0 full
    float* optr = P.out + ((size_t)xs * P.Y + y0 + row0) * P.Z + zcell;

    float2 q[T][YPT];  // x-queue: plane p (item-relative) in slot p % T
#pragma unroll
    for (int i = 0; i < 2 * R; ++i) {
      wait_new();
      const float* sp = smem_c + ns * C::STAGE_FLOATS;
#pragma unroll
      for (int k = 0; k < YPT; ++k) q[i][k] = ld2(sp + rowoff(R + k) + off[(R + k) & 1]);
      if (i < R) {  // planes below R are never a centre plane
        release(cs);
        adv(cs);
      }
      adv(ns);
      if (ns == 0) nph ^= 1;
    }

    for (int j0 = 0; j0 < len; j0 += T) {
      static_for<0, T>([&](auto JJ) {
        constexpr int jj = decltype(JJ)::value;
        const int j = j0 + jj;
        if (j >= len) return;
        wait_new();
        {
          const float* sp = smem_c + ns * C::STAGE_FLOATS;
#pragma unroll
          for (int k = 0; k < YPT; ++k) q[(jj + 2 * R) % T][k] = ld2(sp + rowoff(R + k) + off[(R + k) & 1]);
        }
        adv(ns);
        if (ns == 0) nph ^= 1;
        const float* sc = smem_c + cs * C::STAGE_FLOATS;
        float2 col[M];
#pragma unroll
        for (int m = 0; m < M; ++m) col[m] = ld2(sc + rowoff(m) + off[m & 1]);
        float2 res[YPT][(OP == OP_GRAD) ? 3 : 1];
#pragma unroll
        for (int k = 0; k < YPT; ++k) {
          const float* rp = sc + rowoff(R + k) + off[(R + k) & 1];
          const float2 zl = ld2(rp - 2), zr = ld2(rp + 2), cc = col[k + R];
          const float2 zt[T] = {zl, make_float2(zl.y, cc.x), cc, make_float2(cc.y, zr.x), zr};
          if constexpr (C::LAPL) {
            float2 acc = M2(w2[0], q[jj % T][k]);
#pragma unroll
            for (int t = 1; t < T; ++t) acc = __fadd2_rn(acc, M2(w2[t], q[(jj + t) % T][k]));
#pragma unroll
            for (int t = 0; t < T; ++t) acc = __fadd2_rn(acc, M2(w2[t], col[k + t]));
#pragma unroll
            for (int t = 0; t < T; ++t) acc = __fadd2_rn(acc, M2(w2[t], zt[t]));
            res[k][0] = M2(al2, acc);
            if constexpr (OP == OP_HEAT) res[k][0] = __fadd2_rn(cc, M2(dt2, res[k][0]));  // u2 + dt*(alpha*L)
          } else {
            float2 ax = M2(w2[0], q[jj % T][k]), ay = M2(w2[0], col[k]), az = M2(w2[0], zt[0]);
#pragma unroll
            for (int t = 1; t < T; ++t) {
              ax = __fadd2_rn(ax, M2(w2[t], q[(jj + t) % T][k]));
              ay = __fadd2_rn(ay, M2(w2[t], col[k + t]));
              az = __fadd2_rn(az, M2(w2[t], zt[t]));
            }
            res[k][0] = M2(al2, ax);
            res[k][1] = M2(al2, ay);
            res[k][2] = M2(al2, az);
          }
        }
        if constexpr (OP == OP_GRAD) {
          // stage: the pair's floats 3z .. 3z+5 (x, y, z of each cell) at the row's line offset
          float* ob = obuf + (C::OBUFS == 2 ? (opc & 1) * (TY * C::OROW) : 0);
          const size_t rf0 = (((size_t)(xs + j) * P.Y + y0) * P.Z + z0) * 3;
          const int r0 = (obase + (int)(rf0 & 31u)) & 31;
#pragma unroll
          for (int k = 0; k < YPT; ++k) {
            const int t = row0 + k;
            float* sr = ob + t * C::OROW + ((r0 + t * dzr) & 31) + 6 * lane;
            if (st2) {  // even line offset: 8-byte stores
              *reinterpret_cast<float2*>(sr) = make_float2(res[k][0].x, res[k][1].x);
              *reinterpret_cast<float2*>(sr + 2) = make_float2(res[k][2].x, res[k][0].y);
              *reinterpret_cast<float2*>(sr + 4) = make_float2(res[k][1].y, res[k][2].y);
            } else {
              sr[0] = res[k][0].x; sr[1] = res[k][1].x; sr[2] = res[k][2].x;
              sr[3] = res[k][0].y; sr[4] = res[k][1].y; sr[5] = res[k][2].y;
            }
          }
          release(cs);  // the centre plane is not read again
          adv(cs);
          ++opc;
          s3_grad_rows<C, R, TZ, TY>(P, ob, rf0, r0, dzr, y0, z0);
        } else {
          release(cs);  // the centre plane is not read again
          adv(cs);
          float* op = optr + (size_t)j * oplane;
          if (all_rows) {
#pragma unroll
            for (int k = 0; k < YPT; ++k) *reinterpret_cast<float2*>(op + (size_t)k * P.Z) = res[k][0];
          } else {
#pragma unroll
            for (int k = 0; k < YPT; ++k) {
              if ((vm0 >> k) & 1u) op[(size_t)k * P.Z] = res[k][0].x;
              if ((vm1 >> k) & 1u) op[(size_t)k * P.Z + 1] = res[k][0].y;
            }
          }
        }
      });
    }
    // the last R planes were read only into the x-queue
#pragma unroll
    for (int i = 0; i < R; ++i) {
      release(cs);
      adv(cs);
    }
  }
  if constexpr (OP == OP_GRAD) bulk_wait();  // this lane's bulk stores are done before the block exits
}

// Register budget: two resident blocks per SM up to 320 threads, one above
// (a cap of two such blocks spilled at 56-72 registers).
// Work items are (chunk of planes, tile) pairs in chunk-major order, dealt
// round-robin to a persistent grid: the items in flight at any time share a
// plane range, so neighbouring tiles read each other's halo rows from L2.
// The stage ring and its barrier phases continue from one item to the next
// (running stage counters), so the producer prefetches across items.
template <int R, int OP, int CIN, int TZ, int TY, int YPT, int PREF, int MAPK, int MODE>
__global__ void __launch_bounds__(S3Cfg<R, OP, CIN, TZ, TY, YPT, PREF, MAPK, MODE>::THREADS,
                                   (S3Cfg<R, OP, CIN, TZ, TY, YPT, PREF, MAPK, MODE>::THREADS > 320 ? 1 : 2))
    stream3d_kernel(const __grid_constant__ CUtensorMap tmap, const S3Params P, const FastW FW) {
  using C = S3Cfg<R, OP, CIN, TZ, TY, YPT, PREF, MAPK, MODE>;
  constexpr bool PP0 = (MAPK != MAP_ROWS_GEN);
  constexpr int ROWS = C::ROWS, W = C::W, WP = C::WP, S = C::S, T = 2 * R + 1;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* smem = reinterpret_cast<float*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * C::STAGE_FLOATS);
  uint64_t* empty = full + S;
  float* obuf = reinterpret_cast<float*>(empty + S);

  if ((int)blockIdx.x >= P.nitems) return;  // block-uniform
  const int nx = P.X - 2 * P.g;
  const int tid = threadIdx.x;

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], C::NCW);
    }
    mbar_fence_init();
  }
  __syncthreads();

  if (tid >= C::NCONS) {
    // ---------------- producer warp ----------------
    const int wl = tid - C::NCONS;
    bool dead = false;
    int s = 0, ph = 0, issued = 0;  // stage, its use parity, planes issued
    for (int item = blockIdx.x; item < P.nitems; item += gridDim.x) {
      const int c = item / P.ntiles, tile = item - c * P.ntiles;
      const int xoff = c * P.chunk, len = min(P.chunk, nx - xoff);
      const int tz = tile % P.nz_tiles, ty = tile / P.nz_tiles;
      const int z0 = P.g + tz * TZ, y0 = P.g + ty * TY, xs = P.g + xoff;
      const int nplanes = len + 2 * R;
      int rowf = ((xs - R) * P.Y + (y0 - R)) * P.Z * CIN + (z0 - R) * CIN;  // row 0 of plane 0
      const int plane_f = P.Y * P.Z * CIN, row_f = P.Z * CIN;
      for (int i = 0; i < nplanes; ++i) {
        // plane `issued` reuses the stage of plane issued - S: wait for its release
        if (issued >= S && !dead && !mbar_wait_bounded(&empty[s], (uint32_t)(ph ^ 1), P.wait_ns, &g_err)) {
          dead = true;
          flag_error(PDE_ERR_TIMEOUT);
        }
        if (wl == 0) mbar_arrive_expect_tx(&full[s], ROWS * W * 4);
        __syncwarp();
        if constexpr (MAPK == MAP_PAIRS) {
          // even rows (p = 0) and odd rows (p = 1) of the tile: (y0 - R) is even
          if (wl < 2)
            tma_load_3d(smem + s * C::STAGE_FLOATS + wl * C::HALF, &tmap, (wl * row_f + (z0 - R) * CIN) & ~3,
                        (y0 - R) >> 1, xs - R + i, &full[s]);
        } else {
          for (int r = wl; r < ROWS; r += 32)
            tma_load_1d(smem + (s * ROWS + r) * WP, &tmap, (rowf + r * row_f) & ~3, &full[s]);
        }
        rowf += plane_f;
        ++issued;
        if (++s == S) { s = 0; ph ^= 1; }
      }
    }
    return;
  }

  // ---------------- consumer threads ----------------
  if constexpr (C::ZP) {
    s3_zpairs<R, OP, TZ, TY, YPT, PREF>(P, smem, full, empty, obuf);
  } else {
    const int lane = tid % C::LANES, yg = tid / C::LANES;
    const bool warp_leader = (tid & 31) == 0;
    const int cofs = C::LAPL ? (R * CIN + lane) : ((R + lane) * CIN);
    constexpr int qc = 0;                         // x taps: component 0 (DIV: u_x)
    constexpr int yc = (OP == OP_DIV) ? 1 : 0;    // y taps: DIV reads u_y
    constexpr int zcmp = (OP == OP_DIV) ? 2 : 0;  // z taps: DIV reads u_z
    constexpr int zstep = CIN;
    constexpr int M = YPT + 2 * R;                // centre-plane rows a thread reads
    const int row0 = yg * YPT;                    // first stage row of the thread's window
    // offset (floats) of window row m (stage row row0 + m) inside a stage, without its lead;
    // MAP_PAIRS: row0 is even (YPT even), so row0 + m has the parity of m
    static_assert(MAPK != MAP_PAIRS || (YPT % 2 == 0), "pairs need an even row count per thread");
    auto rowoff = [&](int m) -> int {
      if constexpr (MAPK == MAP_PAIRS) return (m & 1) * C::HALF + (m >> 1) * W;
      else return m * WP;
    };
    const float* smem_c = smem + ((MAPK == MAP_PAIRS) ? (row0 >> 1) * W : row0 * WP) + cofs;

    float w[T];
#pragma unroll
    for (int t = 0; t < T; ++t) w[t] = P.w[t];
    const float alpha = P.alpha;
    float2 w2[T];
#pragma unroll
    for (int t = 0; t < T; ++t) w2[t] = make_float2(w[t], w[t]);
    const float2 al2 = make_float2(alpha, alpha), nz2 = make_float2(P.negzero, P.negzero);

    bool dead = false;
    // consumer stage counters: the newest plane (ns, nph) and the centre plane (cs)
    int ns = 0, nph = 0, cs = 0;
    auto adv = [&](int& st) { if (++st == S) st = 0; };
    auto wait_new = [&]() {
      if (!dead && !mbar_wait_bounded(&full[ns], (uint32_t)nph, P.wait_ns, &g_err)) {
        dead = true;
        flag_error(PDE_ERR_TIMEOUT);
      }
    };
    auto release = [&](int st) {
      __syncwarp();
      if (warp_leader) mbar_arrive(&empty[st]);
    };

    int opc = 0;  // grad: planes stored so far (selects the staging buffer)
    const int obase = (int)((reinterpret_cast<uintptr_t>(P.out) >> 2) & 31u);  // grad: out's float offset in its line
    const int dzr = (3 * P.Z) & 31;  // grad: line offset step from one output row to the next

    const int zrow = P.Z * CIN;
    const int oplane = C::LAPL ? P.Y * zrow : P.Y * P.Z * ((OP == OP_GRAD) ? 3 : 1);
    const int orow = C::LAPL ? zrow : P.Z * ((OP == OP_GRAD) ? 3 : 1);

    for (int item = blockIdx.x; item < P.nitems; item += gridDim.x) {
      const int c = item / P.ntiles, tile = item - c * P.ntiles;
      const int xoff = c * P.chunk, len = min(P.chunk, nx - xoff);
      const int tz = tile % P.nz_tiles, ty = tile / P.nz_tiles;
      const int z0 = P.g + tz * TZ, y0 = P.g + ty * TY, xs = P.g + xoff;
      const int zc = (z0 - R) * CIN;

      // Lead of window row m in plane x: (x*pp + (y0-R+row0+m)*pr + zc) & 3 depends on
      // m only through m mod 4: off[cl] for class cl = m & 3.  MAP_PAIRS: the lead
      // of a row depends only on its parity (off[0], off[1]).
      const int phi = (y0 - R + row0) & 3;
      int off[4];
      auto offsets = [&](int x) {
        if constexpr (MAPK == MAP_PAIRS) {
#pragma unroll
          for (int cl = 0; cl < 4; ++cl) off[cl] = ((cl & 1) * P.Z * CIN + zc) & 3;
        } else {
          const int l = x * P.pp + zc;
#pragma unroll
          for (int cl = 0; cl < 4; ++cl) off[cl] = (l + (phi + cl) * P.pr) & 3;
        }
      };
      if constexpr (PP0) offsets(0);

      unsigned vmask = 0;
      const int zcell = C::LAPL ? (z0 + lane / CIN) : (z0 + lane);
#pragma unroll
      for (int k = 0; k < YPT; ++k)
        if (y0 + row0 + k < P.Y - P.g && zcell < P.Z - P.g) vmask |= 1u << k;
      const bool all_rows = vmask == (1u << YPT) - 1u;
      float* optr = P.out + (C::LAPL ? ((xs * P.Y + y0 + row0) * zrow + z0 * CIN + lane)
                                            : ((xs * P.Y + y0 + row0) * P.Z + zcell) * ((OP == OP_GRAD) ? 3 : 1));

      // x-queue: plane p (item-relative) lives in slot p % T
      float q[T][YPT];
#pragma unroll
      for (int i = 0; i < 2 * R; ++i) {
        wait_new();
        if constexpr (!PP0) offsets(xs - R + i);
        const float* sp = smem_c + ns * C::STAGE_FLOATS + qc;
#pragma unroll
        for (int k = 0; k < YPT; ++k) q[i][k] = sp[rowoff(R + k) + off[(R + k) & 3]];
        if (i < R) {  // planes below R are never a centre plane
          release(cs);
          adv(cs);
        }
        adv(ns);
        if (ns == 0) nph ^= 1;
      }

      for (int j0 = 0; j0 < len; j0 += T) {
        static_for<0, T>([&](auto JJ) {
          constexpr int jj = decltype(JJ)::value;
          const int j = j0 + jj;
          if (j >= len) return;
          wait_new();
          if constexpr (!PP0) offsets(xs + R + j);
          {
            const float* sp = smem_c + ns * C::STAGE_FLOATS + qc;
#pragma unroll
            for (int k = 0; k < YPT; ++k) q[(jj + 2 * R) % T][k] = sp[rowoff(R + k) + off[(R + k) & 3]];
          }
          adv(ns);
          if (ns == 0) nph ^= 1;
          if constexpr (!PP0) offsets(xs + j);
          const float* sc = smem_c + cs * C::STAGE_FLOATS;
          float col[M];
#pragma unroll
          for (int m = 0; m < M; ++m) col[m] = sc[rowoff(m) + off[m & 3] + yc];
          float res[YPT][(OP == OP_GRAD) ? 3 : 1];
          // grad: this plane's staging buffer; tile row t of the plane starts rf0 + 3 Z t
          // floats into the array, at float (r0 + dzr t) mod 32 of a 128-byte line
          [[maybe_unused]] float* ob = obuf + (C::OBUFS == 2 ? (opc & 1) * (TY * C::OROW) : 0);
          [[maybe_unused]] size_t rf0 = 0;
          [[maybe_unused]] int r0 = 0;
          if constexpr (OP == OP_GRAD) {
            rf0 = (((size_t)(xs + j) * P.Y + y0) * P.Z + z0) * 3;
            r0 = (obase + (int)(rf0 & 31u)) & 31;
          }
          if constexpr (MODE == MODE_EXACT) {
            // Two rows per lane pair: packed products (__ffma2_rn with a run-time -0
            // addend, the correctly rounded product) and sums (__fadd2_rn), each lane
            // the scalar operation of the reference order.
            static_assert(YPT % 2 == 0, "row pairs");
#pragma unroll
            for (int kp = 0; kp < YPT; kp += 2) {
              const float* rp0 = sc + rowoff(R + kp) + off[(R + kp) & 3] + zcmp;
              const float* rp1 = sc + rowoff(R + kp + 1) + off[(R + kp + 1) & 3] + zcmp;
              auto X2 = [&](int t) { return make_float2(q[(jj + t) % T][kp], q[(jj + t) % T][kp + 1]); };
              auto Y2 = [&](int t) { return make_float2(col[kp + t], col[kp + 1 + t]); };
              auto Z2 = [&](int t) {
                if (t == R && OP != OP_DIV) return make_float2(col[kp + R], col[kp + 1 + R]);
                return make_float2(rp0[(t - R) * zstep], rp1[(t - R) * zstep]);
              };
              auto M2 = [&](float2 a, float2 b) { return __ffma2_rn(a, b, nz2); };
              if constexpr (C::LAPL || OP == OP_DIV) {
                float2 acc = M2(w2[0], X2(0));
#pragma unroll
                for (int t = 1; t < T; ++t) acc = __fadd2_rn(acc, M2(w2[t], X2(t)));
#pragma unroll
                for (int t = 0; t < T; ++t) acc = __fadd2_rn(acc, M2(w2[t], Y2(t)));
#pragma unroll
                for (int t = 0; t < T; ++t) acc = __fadd2_rn(acc, M2(w2[t], Z2(t)));
                float2 r = M2(al2, acc);
                if constexpr (OP == OP_HEAT)  // u2 + dt*(alpha*L), the centre of each row
                  r = __fadd2_rn(make_float2(col[kp + R], col[kp + 1 + R]), M2(make_float2(P.dt, P.dt), r));
                res[kp][0] = r.x;
                res[kp + 1][0] = r.y;
              } else {
                float2 ax = M2(w2[0], X2(0)), ay = M2(w2[0], Y2(0)), az = M2(w2[0], Z2(0));
#pragma unroll
                for (int t = 1; t < T; ++t) {
                  ax = __fadd2_rn(ax, M2(w2[t], X2(t)));
                  ay = __fadd2_rn(ay, M2(w2[t], Y2(t)));
                  az = __fadd2_rn(az, M2(w2[t], Z2(t)));
                }
                const float2 rx = M2(al2, ax), ry = M2(al2, ay), rz = M2(al2, az);
                res[kp][0] = rx.x;
                res[kp + 1][0] = rx.y;
                res[kp][1] = ry.x;
                res[kp + 1][1] = ry.y;
                res[kp][2] = rz.x;
                res[kp + 1][2] = rz.y;
              }
            }
          } else {
#pragma unroll
            for (int k = 0; k < YPT; ++k) {
              const float* rowp = sc + rowoff(R + k) + off[(R + k) & 3] + zcmp;
              auto xq = [&](int t) { return q[(jj + t) % T][k]; };
              auto zt = [&](int t) { return (t == R && OP == OP_LAP) ? col[k + R] : rowp[(t - R) * zstep]; };
              if constexpr (OP == OP_LAP) {
                // alpha*(sum_t w[t]*(x,y,z taps)) = a[R]*centre + sum_{t<R} a[t]*(six mirrored taps)
                float acc = FW.a[R] * col[k + R];
#pragma unroll
                for (int t = 0; t < R; ++t) {
                  const float s6 = ((xq(t) + xq(T - 1 - t)) + (col[k + t] + col[k + T - 1 - t])) +
                                   (zt(t) + zt(T - 1 - t));
                  acc = fmaf(FW.a[t], s6, acc);
                }
                res[k][0] = acc;
              } else if constexpr (OP == OP_DIV) {
                // alpha*sum_a sum_{t>R} w[t]*(u_a[+] - u_a[-])
                float acc = 0.0f;
#pragma unroll
                for (int t = R + 1; t < T; ++t) {
                  const float d3 = ((xq(t) - xq(T - 1 - t)) + (col[k + t] - col[k + T - 1 - t])) +
                                   (zt(t) - zt(T - 1 - t));
                  acc = (t == R + 1) ? FW.a[t - R - 1] * d3 : fmaf(FW.a[t - R - 1], d3, acc);
                }
                res[k][0] = acc;
              } else {
                float ax = 0.0f, ay = 0.0f, az = 0.0f;
#pragma unroll
                for (int t = R + 1; t < T; ++t) {
                  const float a = FW.a[t - R - 1];
                  const bool first = (t == R + 1);
                  ax = first ? a * (xq(t) - xq(T - 1 - t)) : fmaf(a, xq(t) - xq(T - 1 - t), ax);
                  ay = first ? a * (col[k + t] - col[k + T - 1 - t]) : fmaf(a, col[k + t] - col[k + T - 1 - t], ay);
                  az = first ? a * (rowp[(t - R) * zstep] - rowp[(R - t) * zstep])
                             : fmaf(a, rowp[(t - R) * zstep] - rowp[(R - t) * zstep], az);
                }
                res[k][0] = ax;
                res[k][1] = ay;
                res[k][2] = az;
              }
            }
          }
          if constexpr (OP == OP_GRAD) {  // staged: the rows' results need no registers after this
#pragma unroll
            for (int k = 0; k < YPT; ++k) {
              const int t = row0 + k;
              float* sr = ob + t * C::OROW + ((r0 + t * dzr) & 31) + 3 * lane;
              sr[0] = res[k][0];
              sr[1] = res[k][1];
              sr[2] = res[k][2];
            }
          }
          release(cs);  // the centre plane is not read again
          adv(cs);
          [[maybe_unused]] float* op = optr + j * oplane;  // this thread's first output (LAP, DIV)
          if constexpr (OP == OP_GRAD) {
            ++opc;
            s3_grad_rows<C, R, TZ, TY>(P, ob, rf0, r0, dzr, y0, z0);
          } else if (all_rows) {
#pragma unroll
            for (int k = 0; k < YPT; ++k) op[k * orow] = res[k][0];
          } else {
#pragma unroll
            for (int k = 0; k < YPT; ++k) {
              if (!((vmask >> k) & 1u)) continue;
              op[k * orow] = res[k][0];
            }
          }
        });
      }
      // the last R planes were read only into the x-queue
#pragma unroll
      for (int i = 0; i < R; ++i) {
        release(cs);
        adv(cs);
      }
    }
    if constexpr (OP == OP_GRAD && R >= 2) bulk_wait();  // this lane's bulk stores are done before the block exits
  }
}

}  // namespace pde
