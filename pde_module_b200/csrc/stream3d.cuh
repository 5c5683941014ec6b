// 2.5D streaming stencils for 3D grids with TMA-staged halo tiles.
//
// A block owns a (TY x TZ) tile of interior (y, z) columns and marches along
// X (the slowest axis) over a chunk of planes.  Each input plane of the tile
// (TY + 2R rows, each TZ + 2R cells plus alignment lead) is brought into a
// ring of S shared-memory stages by 1D TMA bulk-tensor copies (one per row:
// the array's row pitch is arbitrary, e.g. 514 floats, so a 3D tensor map's
// 16-byte stride rule cannot be met) completing on one mbarrier per stage.
// Loads run S - 2R - 1 planes ahead of the plane being computed.  X-direction
// taps come from a register queue of the thread's own column; Y and Z taps
// come from the centre stage.  Every product and sum is rounded separately,
// in the reference's order (axes ascending, taps low to high, alpha last), so
// the results are bit-identical to the general kernels.
#pragma once
#include "common.cuh"
#include "tma.cuh"

namespace pde {

enum { OP_LAP = 0, OP_GRAD = 1, OP_DIV = 2 };

struct S3Params {
  int X, Y, Z, g;
  int chunk;            // output planes per block
  int ny_tiles, nz_tiles;
  int pp, pr;           // (Y*Z*CIN) mod 4, (Z*CIN) mod 4: row alignment lead
  float w[5];
  float alpha;
  float* out;
};

__host__ __device__ constexpr int round4(int v) { return (v + 3) & ~3; }

template <int R, int OP, int CIN, int TZ, int TY, int YPT, int PREF>
struct S3Cfg {
  static constexpr int LANES = (OP == OP_LAP) ? TZ * CIN : TZ;
  static constexpr int TYG = TY / YPT;
  static constexpr int THREADS = LANES * TYG;
  static constexpr int ROWS = TY + 2 * R;
  static constexpr int W = round4(3 + (TZ + 2 * R) * CIN);  // TMA box (floats)
  static constexpr int WP = (W + 31) & ~31;  // smem row pitch: TMA destinations are 128-byte aligned
  static constexpr int S = 2 * R + 1 + PREF;
  static constexpr int STAGE_FLOATS = ROWS * WP;
  // + 128: the base is rounded up to a 128-byte boundary at run time
  static constexpr size_t SMEM = (size_t)S * STAGE_FLOATS * 4 + (size_t)S * 8 + 128;
  static_assert(ROWS <= 32, "one warp issues the row copies of a stage");
  static_assert(W <= 256, "TMA box extent");
  static_assert(TY % YPT == 0, "rows per thread");
};

template <int R, int OP, int CIN, int TZ, int TY, int YPT, int PREF>
__global__ void __launch_bounds__(S3Cfg<R, OP, CIN, TZ, TY, YPT, PREF>::THREADS)
    stream3d_kernel(const __grid_constant__ CUtensorMap tmap, const S3Params P) {
  using C = S3Cfg<R, OP, CIN, TZ, TY, YPT, PREF>;
  constexpr int ROWS = C::ROWS, W = C::W, WP = C::WP, S = C::S, T = 2 * R + 1;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* smem = reinterpret_cast<float*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u));
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + S * C::STAGE_FLOATS);

  int bid = blockIdx.x;
  const int tz = bid % P.nz_tiles;
  bid /= P.nz_tiles;
  const int ty = bid % P.ny_tiles;
  bid /= P.ny_tiles;
  const int z0 = P.g + tz * TZ, y0 = P.g + ty * TY;
  const int xs = P.g + bid * P.chunk;
  const int xe = min(xs + P.chunk, P.X - P.g);
  if (xs >= xe) return;  // block-uniform
  const int nout = xe - xs;
  const int nplanes = nout + 2 * R;
  const int lane = threadIdx.x, yg = threadIdx.y;
  const int tid = yg * C::LANES + lane;
  const int warp = tid >> 5, wl = tid & 31;
  const int zc = (z0 - R) * CIN;  // float offset of the tile start within a row

  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
    mbar_fence_init();
  }
  __syncthreads();

  // warp 0 brings plane i (x = xs - R + i) into stage i % S.
  auto issue = [&](int i) {
    const int s = i % S;
    const int x = xs - R + i;
    if (wl == 0) mbar_arrive_expect_tx(&bar[s], ROWS * W * 4);
    __syncwarp();
    if (wl < ROWS) {
      const int y = y0 - R + wl;
      const int f0 = (x * P.Y + y) * P.Z * CIN + zc;
      tma_load_1d(smem + (s * ROWS + wl) * WP, &tmap, f0 & ~3, &bar[s]);
    }
  };
  bool dead = false;
  auto wait_plane = [&](int i) {
    if (!dead && !mbar_wait_bounded(&bar[i % S], (uint32_t)((i / S) & 1))) {
      dead = true;
      flag_error(PDE_ERR_TIMEOUT);
    }
  };
  // position of the tile's first cell (z0 - R) inside a staged row.
  auto lead = [&](int x, int y) { return (x * P.pp + y * P.pr + zc) & 3; };
  auto stage = [&](int i) -> const float* { return smem + (i % S) * C::STAGE_FLOATS; };

  if (warp == 0) {
    const int pre = nplanes < S ? nplanes : S;
    for (int i = 0; i < pre; ++i) issue(i);
  }

  // Offset (floats) of this thread's centre value inside a staged row,
  // excluding the row lead.
  constexpr int zsel = (OP == OP_LAP) ? 0 : 1;
  const int cofs = (OP == OP_LAP) ? (R * CIN + lane) : ((R + lane) * CIN);
  // component read from the x-queue / y-column / z-row for each op.
  constexpr int qc = 0;                         // x taps: component 0 (DIV: u_x)
  constexpr int yc = (OP == OP_DIV) ? 1 : 0;    // y taps: DIV reads u_y
  constexpr int zcmp = (OP == OP_DIV) ? 2 : 0;  // z taps: DIV reads u_z
  constexpr int zstep = (OP == OP_LAP) ? CIN : CIN;
  (void)zsel;

  float q[T][YPT];
#pragma unroll
  for (int t = 0; t < T; ++t)
#pragma unroll
    for (int k = 0; k < YPT; ++k) q[t][k] = 0.0f;

  // Pre-load planes 0 .. 2R-1 into q[1 .. 2R].
#pragma unroll
  for (int i = 0; i < 2 * R; ++i) {
    wait_plane(i);
    const float* sp = stage(i);
    const int x = xs - R + i;
#pragma unroll
    for (int k = 0; k < YPT; ++k) {
      const int r = R + yg * YPT + k;
      q[i + 1][k] = sp[r * WP + lead(x, y0 - R + r) + cofs + qc];
    }
  }

  const float alpha = P.alpha;
  float w[T];
#pragma unroll
  for (int t = 0; t < T; ++t) w[t] = P.w[t];

  for (int j = 0; j < nout; ++j) {
    const int inew = j + 2 * R;
    wait_plane(inew);
#pragma unroll
    for (int t = 0; t < T - 1; ++t)
#pragma unroll
      for (int k = 0; k < YPT; ++k) q[t][k] = q[t + 1][k];
    {
      const float* sp = stage(inew);
      const int x = xs - R + inew;
#pragma unroll
      for (int k = 0; k < YPT; ++k) {
        const int r = R + yg * YPT + k;
        q[T - 1][k] = sp[r * WP + lead(x, y0 - R + r) + cofs + qc];
      }
    }
    const float* sc = stage(j + R);
    const int xc = xs + j;
    float col[YPT + 2 * R];
#pragma unroll
    for (int m = 0; m < YPT + 2 * R; ++m) {
      const int r = yg * YPT + m;
      col[m] = sc[r * WP + lead(xc, y0 - R + r) + cofs + yc];
    }
#pragma unroll
    for (int k = 0; k < YPT; ++k) {
      const int r = R + yg * YPT + k;
      const int yk = y0 - R + r;
      const float* rowp = sc + r * WP + lead(xc, yk) + cofs + zcmp;
      if constexpr (OP == OP_LAP || OP == OP_DIV) {
        float acc = 0.0f;
#pragma unroll
        for (int t = 0; t < T; ++t) acc = add(acc, mul(w[t], q[t][k]));
#pragma unroll
        for (int t = 0; t < T; ++t) acc = add(acc, mul(w[t], col[k + t]));
#pragma unroll
        for (int t = 0; t < T; ++t) acc = add(acc, mul(w[t], rowp[(t - R) * zstep]));
        const float res = mul(alpha, acc);
        if (OP == OP_LAP) {
          const int zcell = z0 + lane / CIN;
          if (yk < P.Y - P.g && zcell < P.Z - P.g)
            P.out[(xc * P.Y + yk) * P.Z * CIN + z0 * CIN + lane] = res;
        } else {
          const int zcell = z0 + lane;
          if (yk < P.Y - P.g && zcell < P.Z - P.g) P.out[(xc * P.Y + yk) * P.Z + zcell] = res;
        }
      } else {  // OP_GRAD: scalar in, (d/dx, d/dy, d/dz) out
        float ax = 0.0f, ay = 0.0f, az = 0.0f;
#pragma unroll
        for (int t = 0; t < T; ++t) ax = add(ax, mul(w[t], q[t][k]));
#pragma unroll
        for (int t = 0; t < T; ++t) ay = add(ay, mul(w[t], col[k + t]));
#pragma unroll
        for (int t = 0; t < T; ++t) az = add(az, mul(w[t], rowp[(t - R) * zstep]));
        const int zcell = z0 + lane;
        if (yk < P.Y - P.g && zcell < P.Z - P.g) {
          float* o = P.out + ((size_t)((xc * P.Y + yk) * P.Z + zcell)) * 3;
          o[0] = mul(alpha, ax);
          o[1] = mul(alpha, ay);
          o[2] = mul(alpha, az);
        }
      }
    }
    __syncthreads();  // every thread is done with plane j's stage
    if (warp == 0 && j + S < nplanes) issue(j + S);
  }
}

}  // namespace pde
