// Fused y-x-y pass of the FP32 H|psi> pipeline for k1 x k2 planes of the
// specialised shapes (x length NX = k1, y length NY = k2), one CTA per (band
// pair, z plane or two), one grid line per thread with the whole line in
// registers (compile-time-length FFTs of qx_regfft.cuh):
//   (1) backward y-FFT of each of the P1 sphere columns, read straight from
//       the z-transformed plane in bufA (rows outside the sphere are zero);
//   (2) per grid row: backward x-FFT (P1 non-zero inputs), times V_loc(r),
//       forward x-FFT, keep the P1 sphere columns;
//   (3) forward y-FFT of each column, the sphere rows written back to bufA.
// Between the steps the plane lives in shared memory as NY x P1 complex
// values.  This replaces k_ypass<+1>, k_xvx and k_ypass<-1> (hcnonloc's
// c2r -> V_loc * psi -> r2c, engrad.f90:484-571) and removes the two round
// trips of bufB through L2/HBM.
//
// This header holds the kernel templates and their per-shape launchers; each
// qx_fftplane_*.cu file instantiates a group of shapes and z lengths (so the
// groups compile in parallel), and qx_fftplane.cu dispatches on the grid.
#pragma once
#include "qx_fftplane.h"
#include "qx_regfft.cuh"

namespace qx {

// Resident CTAs per SM asked of the register allocator: 8 (128 registers)
// where that needs no spills.
constexpr int plane_minb(int n) { return n <= 54 ? 8 : 1; }

// Grid rows of the x phase, thread t of a 64-thread CTA: with two planes of
// at most 32 rows, warp w takes plane w's rows (both planes at once);
// otherwise thread t takes row t of each plane in turn.
template <int NY, int PL>
struct PlaneRows {
  static constexpr bool both = PL == 2 && NY <= 32;
  static constexpr int passes = both ? 1 : PL;
  __device__ static int plane(int t, int pass) { return both ? (t >> 5) : pass; }
  __device__ static int row(int t) { return both ? (t & 31) : t; }
};

template <int NX, int NY, int PL>
__global__ void __launch_bounds__(64, plane_minb(NX > NY ? NX : NY))
    k_plane(PipeParams P, float2 *__restrict__ bufA, const float *__restrict__ vloc) {
  using rf::out_pos;
  using Rows = PlaneRows<NY, PL>;
  // PL = 2: the CTA takes planes i3 and i3 + 1; the y phases give warp w the
  // columns of plane w (P1 <= 32).  PL = 1: one plane, the columns on
  // threads 0 .. P1 - 1.  NX = k1 (x, the sphere's P1 columns), NY = k2.
  const int i3b = blockIdx.x * PL;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= (P.npair_dev ? *P.npair_dev : P.npair)) return;
  const int P1 = P.P1, P2 = P.P2, m1 = P.m1, m2 = P.m2;
  const int npl_here = min(PL, P.k3 - i3b);   // planes this CTA owns (uniform)
  extern __shared__ float2 T[];   // [PL][NY][P1]
  const int t = threadIdx.x;
  const float2 zero = make_float2(0.f, 0.f);
  // column phases: plane and column of this thread
  const int cpl = (PL == 2) ? (t >> 5) : 0, col = (PL == 2) ? (t & 31) : t;
  const bool col_on = col < P1 && cpl < npl_here;
  float2 *A = bufA + ((long)pl * P.k3 + i3b + cpl) * P2 * P1;
  float2 *Tc = T + (long)cpl * NY * P1;

  // (1) y backward, thread = sphere column a of its plane
  if (col_on) {
    float2 x[NY];
#pragma unroll
    for (int i2 = 0; i2 < NY; ++i2) {
      const int j2 = (i2 <= m2) ? i2 + m2 : ((i2 >= NY - m2) ? i2 - NY + m2 : -1);
      float2 v = zero;
      if (j2 >= 0 && col >= P.row_lo[j2] && col <= P.row_hi[j2]) v = A[j2 * P1 + col];
      x[i2] = v;
    }
    rf::fft<float, +1, NY>(x);
    rf::static_for<0, NY>([&](auto ic) {
      constexpr int i2 = decltype(ic)::value, q = out_pos(NY, i2);
      Tc[i2 * P1 + col] = x[q];
    });
  }
  __syncthreads();
  // (2) x backward, * V, x forward; thread = grid row r of plane rp
  const int r = Rows::row(t);
  for (int pass = 0; pass < Rows::passes; ++pass) {
    const int rp = Rows::plane(t, pass);
    if (r < NY && rp < npl_here) {
      float2 x[NX];
      float2 *row = T + ((long)rp * NY + r) * P1;
#pragma unroll
      for (int i1 = 0; i1 < NX; ++i1) {
        float2 v = zero;
        if (i1 <= m1) v = row[i1 + m1];
        else if (i1 >= NX - m1) v = row[i1 - NX + m1];
        x[i1] = v;
      }
      rf::fft<float, +1, NX>(x);
      const float *V = vloc + ((long)(i3b + rp) * NY + r) * NX;
      float2 y[NX];
      rf::static_for<0, NX>([&](auto ic) {
        constexpr int i1 = decltype(ic)::value, q = out_pos(NX, i1);
        const float vv = V[i1];
        y[i1] = make_float2(x[q].x * vv, x[q].y * vv);
      });
      rf::fft<float, -1, NX>(y);
      rf::static_for<0, NX>([&](auto ic) {
        constexpr int i1 = decltype(ic)::value, q = out_pos(NX, i1);
        if (i1 <= m1) row[i1 + m1] = y[q];
        else if (i1 >= NX - m1) row[i1 - NX + m1] = y[q];
      });
    }
  }
  __syncthreads();
  // (3) y forward, thread = sphere column a of its plane; only rows inside the sphere are kept
  if (col_on) {
    float2 x[NY];
#pragma unroll
    for (int i2 = 0; i2 < NY; ++i2) x[i2] = Tc[i2 * P1 + col];
    rf::fft<float, -1, NY>(x);
    rf::static_for<0, NY>([&](auto ic) {
      constexpr int i2 = decltype(ic)::value, q = out_pos(NY, i2);
      const int j2 = (i2 <= m2) ? i2 + m2 : ((i2 >= NY - m2) ? i2 - NY + m2 : -1);
      if (j2 >= 0 && col >= P.row_lo[j2] && col <= P.row_hi[j2]) A[j2 * P1 + col] = x[q];
    });
  }
}

// ---------------------------------------------------------------------------
// The same fused y-x-y pass for longer lines (N = 2H, H a register-FFT length,
// N > 64), two threads per line: lanes 2l and 2l + 1 of a warp own line l.
// Backward transforms and the forward y transform by decimation in time:
// thread h holds the samples x[2j + h], transforms them (H points), and one
// butterfly exchange with its partner (shfl_xor 1) leaves it the outputs
// X[k + hH], k < H, at positions out_pos(H, k).  The forward x transform
// follows the potential multiply, when thread h holds the second half of the
// line (y[k + hH]), so it runs by decimation in frequency: the exchange
// stage first (a = y[k] + y[k+H] kept by h = 0, b = (y[k] - y[k+H]) w^k by
// h = 1), then the H-point transform gives the outputs Y[2j + h].  Whole
// warps run each phase (lanes without a line work on zeros and store
// nothing), so every shuffle has its full mask.
namespace pl2 {
template <int SIGN, int N>
__device__ __forceinline__ void dit_combine(float2 (&v)[N / 2], int h) {
  constexpr int H = N / 2;
  rf::static_for<0, H>([&](auto kc) {
    constexpr int k = decltype(kc)::value, pk = rf::out_pos(H, k);
    const float2 mine = v[pk];
    float2 other;
    other.x = __shfl_xor_sync(0xffffffffu, mine.x, 1);
    other.y = __shfl_xor_sync(0xffffffffu, mine.y, 1);
    const float2 e = h ? other : mine;
    const float2 t = rf::twiddle<float, SIGN, k, N>(h ? mine : other);
    v[pk] = h ? rf::sub(e, t) : rf::add(e, t);
  });
}
// v[out_pos(H, k)] = y[k + hH] in; u[k] (natural order) = a[k] (h = 0) or
// b[k] (h = 1) out, ready for the H-point transform.
template <int SIGN, int N>
__device__ __forceinline__ void dif_split(const float2 (&v)[N / 2], float2 (&u)[N / 2], int h) {
  constexpr int H = N / 2;
  rf::static_for<0, H>([&](auto kc) {
    constexpr int k = decltype(kc)::value, pk = rf::out_pos(H, k);
    const float2 mine = v[pk];
    float2 other;
    other.x = __shfl_xor_sync(0xffffffffu, mine.x, 1);
    other.y = __shfl_xor_sync(0xffffffffu, mine.y, 1);
    const float2 lo = h ? other : mine, hi = h ? mine : other;   // y[k], y[k + H]
    u[k] = h ? rf::twiddle<float, SIGN, k, N>(rf::sub(lo, hi)) : rf::add(lo, hi);
  });
}
}  // namespace pl2

template <int N>
__global__ void __launch_bounds__(2 * N) k_plane2(PipeParams P, float2 *__restrict__ bufA,
                                                 const float *__restrict__ vloc) {
  using rf::out_pos;
  constexpr int H = N / 2;
  const int i3 = blockIdx.x;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= (P.npair_dev ? *P.npair_dev : P.npair)) return;
  const int P1 = P.P1, P2 = P.P2, m1 = P.m1, m2 = P.m2;
  extern __shared__ float2 T[];   // [N][P1]
  float2 *A = bufA + ((long)pl * P.k3 + i3) * P2 * P1;
  const int t = threadIdx.x, l = t >> 1, h = t & 1;
  const bool warp_on_cols = (t & ~31) < 2 * P1;   // some lane of this warp owns a column
  const float2 zero = make_float2(0.f, 0.f);

  // (1) y backward, line = sphere column a = l
  if (warp_on_cols) {
    const bool on = l < P1;
    float2 x[H];
#pragma unroll
    for (int j = 0; j < H; ++j) {
      const int i2 = 2 * j + h;
      const int j2 = (i2 <= m2) ? i2 + m2 : ((i2 >= N - m2) ? i2 - N + m2 : -1);
      float2 v = zero;
      if (on && j2 >= 0 && l >= P.row_lo[j2] && l <= P.row_hi[j2]) v = A[j2 * P1 + l];
      x[j] = v;
    }
    rf::fft<float, +1, H>(x);
    pl2::dit_combine<+1, N>(x, h);
    if (on) {
      rf::static_for<0, H>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        T[(k + h * H) * P1 + l] = x[out_pos(H, k)];
      });
    }
  }
  __syncthreads();
  // (2) x backward, * V, x forward; line = grid row i2 = l (every thread has one)
  {
    float2 x[H];
    float2 *row = T + l * P1;
#pragma unroll
    for (int j = 0; j < H; ++j) {
      const int i1 = 2 * j + h;
      float2 v = zero;
      if (i1 <= m1) v = row[i1 + m1];
      else if (i1 >= N - m1) v = row[i1 - N + m1];
      x[j] = v;
    }
    rf::fft<float, +1, H>(x);
    pl2::dit_combine<+1, N>(x, h);
    const float *V = vloc + ((long)i3 * N + l) * N + h * H;
    rf::static_for<0, H>([&](auto kc) {
      constexpr int k = decltype(kc)::value, pk = out_pos(H, k);
      const float vv = V[k];
      x[pk] = make_float2(x[pk].x * vv, x[pk].y * vv);
    });
    float2 u[H];
    pl2::dif_split<-1, N>(x, u, h);
    rf::fft<float, -1, H>(u);
    __syncthreads();   // every thread has read its row before any row is rewritten
    rf::static_for<0, H>([&](auto jc) {
      constexpr int j = decltype(jc)::value;
      const int i1 = 2 * j + h;
      if (i1 <= m1) row[i1 + m1] = u[out_pos(H, j)];
      else if (i1 >= N - m1) row[i1 - N + m1] = u[out_pos(H, j)];
    });
  }
  __syncthreads();
  // (3) y forward, line = sphere column a = l; only rows inside the sphere are kept
  if (warp_on_cols) {
    const bool on = l < P1;
    float2 x[H];
#pragma unroll
    for (int j = 0; j < H; ++j) x[j] = on ? T[(2 * j + h) * P1 + l] : zero;
    rf::fft<float, -1, H>(x);
    pl2::dit_combine<-1, N>(x, h);
    if (on) {
      rf::static_for<0, H>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        const int i2 = k + h * H;
        const int j2 = (i2 <= m2) ? i2 + m2 : ((i2 >= N - m2) ? i2 - N + m2 : -1);
        if (j2 >= 0 && l >= P.row_lo[j2] && l <= P.row_hi[j2]) A[j2 * P1 + l] = x[out_pos(H, k)];
      });
    }
  }
}

// ---------------------------------------------------------------------------
// The z transforms of the FP32 pipeline, one sphere z-column (j2, a) of one
// band pair per thread with the whole line in registers (replacing the
// shared-memory k_zinv / k_zfwd for the specialised lengths).  The column's
// coefficients come from the z-column table (col_ig, i3-major, so a warp's
// lookups are one row); positions without a sphere entry are zero.
//   inverse: two real bands packed as c_A + i c_B (their +G and -G halves),
//            backward z-FFT, written to bufA[pair][i3][j2][a];
//   forward: read the column from bufA, forward z-FFT, scale by 1/N and
//            scatter to zsph as k_zfwd does.
constexpr int ZC_T = 64;

template <int N>
__global__ void __launch_bounds__(ZC_T) k_zcols_inv(PipeParams P, const float *__restrict__ cin, long ldc,
                                                     float2 *__restrict__ bufA) {
  using rf::out_pos;
  const int q = blockIdx.x * ZC_T + threadIdx.x;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= (P.npair_dev ? *P.npair_dev : P.npair) || q >= P.ncol) return;
  const int bA = P.pairs[2 * p], bB = P.pairs[2 * p + 1];
  const float *cA = cin + (long)bA * ldc;
  const float *cB = bB >= 0 ? cin + (long)bB * ldc : nullptr;
  float2 x[N];
#pragma unroll
  for (int i3 = 0; i3 < N; ++i3) {
    const int code = P.col_ig[i3 * P.ncol + q];
    float2 z = make_float2(0.f, 0.f);
    if (code != 0) {
      const int ig = (code > 0 ? code : -code) - 1;
      const float ra = cA[2 * ig], ia = ig ? cA[2 * ig + 1] : 0.f;
      const float rb = cB ? cB[2 * ig] : 0.f, ib = (cB && ig) ? cB[2 * ig + 1] : 0.f;
      if (code > 0) { z.x = ra - ib; z.y = ia + rb; }
      else          { z.x = ra + ib; z.y = rb - ia; }
    }
    x[i3] = z;
  }
  rf::fft<float, +1, N>(x);
  float2 *dst = bufA + (long)pl * N * P.P2 * P.P1 + P.col_ja[q];
  rf::static_for<0, N>([&](auto ic) {
    constexpr int i3 = decltype(ic)::value;
    dst[(long)i3 * P.P2 * P.P1] = x[out_pos(N, i3)];
  });
}

template <int N>
__global__ void __launch_bounds__(ZC_T) k_zcols_fwd(PipeParams P, const float2 *__restrict__ bufA,
                                                     float2 *__restrict__ zsph) {
  using rf::out_pos;
  const int q = blockIdx.x * ZC_T + threadIdx.x;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= (P.npair_dev ? *P.npair_dev : P.npair) || q >= P.ncol) return;
  const float2 *src = bufA + (long)pl * N * P.P2 * P.P1 + P.col_ja[q];
  float2 x[N];
#pragma unroll
  for (int i3 = 0; i3 < N; ++i3) x[i3] = src[(long)i3 * P.P2 * P.P1];
  rf::fft<float, -1, N>(x);
  const float s = (float)P.inv_n;
  float2 *Z = zsph + (long)pl * (P.nplw + 1) * 2;
  rf::static_for<0, N>([&](auto ic) {
    constexpr int i3 = decltype(ic)::value;
    const int code = P.col_ig[i3 * P.ncol + q];
    if (code != 0) {
      float2 z = x[out_pos(N, i3)];
      z.x *= s;
      z.y *= s;
      if (code > 0) {
        const int ig = code - 1;
        Z[2 * ig] = z;
        if (ig == 0) Z[1] = z;
      } else {
        Z[2 * (-code - 1) + 1] = z;
      }
    }
  });
}

// The inverse z pass for the two-lanes-a-line lengths (N = 2H > 64): lanes
// 2c and 2c + 1 own sphere z-column c, each gathers the coefficients of the
// even or odd i3 and transforms them (H points), and the butterfly exchange
// of k_plane2 completes the N-point transform.  Whole warps run (lanes past
// the last column work on zeros and store nothing).
template <int N>
__global__ void __launch_bounds__(ZC_T) k_zcols_inv2(PipeParams P, const float *__restrict__ cin, long ldc,
                                                      float2 *__restrict__ bufA) {
  using rf::out_pos;
  constexpr int H = N / 2;
  const int q = (int)((blockIdx.x * ZC_T + threadIdx.x) >> 1), h = threadIdx.x & 1;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= (P.npair_dev ? *P.npair_dev : P.npair)) return;   // uniform in the block
  const bool on = q < P.ncol;
  const int bA = P.pairs[2 * p], bB = P.pairs[2 * p + 1];
  const float *cA = cin + (long)bA * ldc;
  const float *cB = bB >= 0 ? cin + (long)bB * ldc : nullptr;
  float2 x[H];
#pragma unroll
  for (int j = 0; j < H; ++j) {
    const int i3 = 2 * j + h;
    const int code = on ? P.col_ig[i3 * P.ncol + q] : 0;
    float2 z = make_float2(0.f, 0.f);
    if (code != 0) {
      const int ig = (code > 0 ? code : -code) - 1;
      const float ra = cA[2 * ig], ia = ig ? cA[2 * ig + 1] : 0.f;
      const float rb = cB ? cB[2 * ig] : 0.f, ib = (cB && ig) ? cB[2 * ig + 1] : 0.f;
      if (code > 0) { z.x = ra - ib; z.y = ia + rb; }
      else          { z.x = ra + ib; z.y = rb - ia; }
    }
    x[j] = z;
  }
  rf::fft<float, +1, H>(x);
  pl2::dit_combine<+1, N>(x, h);
  if (on) {
    float2 *dst = bufA + (long)pl * N * P.P2 * P.P1 + P.col_ja[q];
    rf::static_for<0, H>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      dst[(long)(k + h * H) * P.P2 * P.P1] = x[out_pos(H, k)];
    });
  }
}

template <int N>
int zcols2_launch(const PipeParams &P, int npl, const float *cin, long ldc, float2 *bufA, bool inv,
                         cudaStream_t st) {
  if (!inv) return -1;   // the forward z pass stays on the shared-memory kernel
  dim3 g((2 * P.ncol + ZC_T - 1) / ZC_T, npl);
  k_zcols_inv2<N><<<g, ZC_T, 0, st>>>(P, cin, ldc, bufA);
  note_launch();
  return 0;
}

template <int N>
int zcols_launch(const PipeParams &P, int npl, const float *cin, long ldc, float2 *bufA, const float2 *src,
                        float2 *zsph, bool inv, cudaStream_t st) {
  dim3 g((P.ncol + ZC_T - 1) / ZC_T, npl);
  if (inv) k_zcols_inv<N><<<g, ZC_T, 0, st>>>(P, cin, ldc, bufA);
  else k_zcols_fwd<N><<<g, ZC_T, 0, st>>>(P, src, zsph);
  note_launch();
  return 0;
}

// Density for the same grids (softchg, chgdns.f90:388-454): per CTA one z
// plane and one group of band pairs; for each pair the backward y- and
// x-FFTs of the plane as above, then rho += occ_A/Omega psi_A(r)^2 +
// occ_B/Omega psi_B(r)^2 accumulated in FP64 in shared memory (each thread
// owns one grid row).  The group's partial plane goes to part[group]; a
// second kernel sums the groups in a fixed order, so the result is the same
// from run to run.
template <int NX, int NY, int PL>
__global__ void __launch_bounds__(64) k_rho_plane(PipeParams P, const float2 *__restrict__ bufA,
                                                  const double *__restrict__ wocc, double *__restrict__ part,
                                                  int npl, int per_group) {
  using rf::out_pos;
  using Rows = PlaneRows<NY, PL>;
  // PL = 2: planes i3 and i3 + 1, warp w taking plane w's columns in the y
  // phase (P1 <= 32); the x phase as in k_plane.
  const int i3b = blockIdx.x * PL, grp = blockIdx.y;
  const int P1 = P.P1, P2 = P.P2, m1 = P.m1, m2 = P.m2;
  const int npl_here = min(PL, P.k3 - i3b);
  constexpr int NP = NX * NY;
  extern __shared__ double accs[];            // [PL][NY][NX] FP64, then the [PL][NY][P1] complex tiles
  float2 *T = reinterpret_cast<float2 *>(accs + PL * NP);
  const int t = threadIdx.x;
  const float2 zero = make_float2(0.f, 0.f);
  const int cpl = (PL == 2) ? (t >> 5) : 0, col = (PL == 2) ? (t & 31) : t;
  const bool col_on = col < P1 && cpl < npl_here;
  float2 *Tc = T + (long)cpl * NY * P1;
  for (int i = t; i < PL * NP; i += blockDim.x) accs[i] = 0.0;
  const int np = min(npl, (P.npair_dev ? *P.npair_dev : P.npair) - P.pair0);
  const int pl0 = grp * per_group, pl1 = min(np, pl0 + per_group);
  const int r = Rows::row(t);
  for (int pl = pl0; pl < pl1; ++pl) {
    const int p = P.pair0 + pl;
    const float2 *A = bufA + ((long)pl * P.k3 + i3b + cpl) * P2 * P1;
    if (col_on) {
      float2 x[NY];
#pragma unroll
      for (int i2 = 0; i2 < NY; ++i2) {
        const int j2 = (i2 <= m2) ? i2 + m2 : ((i2 >= NY - m2) ? i2 - NY + m2 : -1);
        float2 v = zero;
        if (j2 >= 0 && col >= P.row_lo[j2] && col <= P.row_hi[j2]) v = A[j2 * P1 + col];
        x[i2] = v;
      }
      rf::fft<float, +1, NY>(x);
      rf::static_for<0, NY>([&](auto ic) {
        constexpr int i2 = decltype(ic)::value, q = out_pos(NY, i2);
        Tc[i2 * P1 + col] = x[q];
      });
    }
    __syncthreads();
    const int bA = P.pairs[2 * p], bB = P.pairs[2 * p + 1];
    const double fa = wocc[bA], fb = bB >= 0 ? wocc[bB] : 0.0;
    for (int pass = 0; pass < Rows::passes; ++pass) {
      const int rp = Rows::plane(t, pass);
      if (r < NY && rp < npl_here) {
        float2 x[NX];
        const float2 *row = T + ((long)rp * NY + r) * P1;
#pragma unroll
        for (int i1 = 0; i1 < NX; ++i1) {
          float2 v = zero;
          if (i1 <= m1) v = row[i1 + m1];
          else if (i1 >= NX - m1) v = row[i1 - NX + m1];
          x[i1] = v;
        }
        rf::fft<float, +1, NX>(x);
        double *a = accs + ((long)rp * NY + r) * NX;
        rf::static_for<0, NX>([&](auto ic) {
          constexpr int i1 = decltype(ic)::value, q = out_pos(NX, i1);
          const double re = x[q].x, im = x[q].y;
          a[i1] += fa * re * re + fb * im * im;
        });
      }
    }
    __syncthreads();
  }
  __syncthreads();
  for (int rp = 0; rp < npl_here; ++rp) {
    double *dst = part + ((long)grp * P.k3 + i3b + rp) * NP;
    for (int i = t; i < NP; i += blockDim.x) dst[i] = accs[(long)rp * NP + i];
  }
}

// The density pass for the two-threads-a-line lengths (see k_plane2): the
// y and x backward transforms by decimation in time, thread h of row l then
// adds the columns k + hH, k < H, of the row to the FP64 accumulation plane.
template <int N>
__global__ void __launch_bounds__(2 * N) k_rho_plane2(PipeParams P, const float2 *__restrict__ bufA,
                                                     const double *__restrict__ wocc, double *__restrict__ part,
                                                     int npl, int per_group) {
  using rf::out_pos;
  constexpr int H = N / 2;
  const int i3 = blockIdx.x, grp = blockIdx.y;
  const int P1 = P.P1, P2 = P.P2, m1 = P.m1, m2 = P.m2;
  extern __shared__ double accs[];            // [N][N] FP64, then the [N][P1] complex tile
  float2 *T = reinterpret_cast<float2 *>(accs + N * N);
  const int t = threadIdx.x, l = t >> 1, h = t & 1;
  const bool warp_on_cols = (t & ~31) < 2 * P1;
  const float2 zero = make_float2(0.f, 0.f);
  for (int i = t; i < N * N; i += 2 * N) accs[i] = 0.0;
  const int np = min(npl, (P.npair_dev ? *P.npair_dev : P.npair) - P.pair0);
  const int pl0 = grp * per_group, pl1 = min(np, pl0 + per_group);
  for (int pl = pl0; pl < pl1; ++pl) {
    const int p = P.pair0 + pl;
    const float2 *A = bufA + ((long)pl * P.k3 + i3) * P2 * P1;
    if (warp_on_cols) {
      const bool on = l < P1;
      float2 x[H];
#pragma unroll
      for (int j = 0; j < H; ++j) {
        const int i2 = 2 * j + h;
        const int j2 = (i2 <= m2) ? i2 + m2 : ((i2 >= N - m2) ? i2 - N + m2 : -1);
        float2 v = zero;
        if (on && j2 >= 0 && l >= P.row_lo[j2] && l <= P.row_hi[j2]) v = A[j2 * P1 + l];
        x[j] = v;
      }
      rf::fft<float, +1, H>(x);
      pl2::dit_combine<+1, N>(x, h);
      if (on) {
        rf::static_for<0, H>([&](auto kc) {
          constexpr int k = decltype(kc)::value;
          T[(k + h * H) * P1 + l] = x[out_pos(H, k)];
        });
      }
    }
    __syncthreads();
    {
      float2 x[H];
      const float2 *row = T + l * P1;
#pragma unroll
      for (int j = 0; j < H; ++j) {
        const int i1 = 2 * j + h;
        float2 v = zero;
        if (i1 <= m1) v = row[i1 + m1];
        else if (i1 >= N - m1) v = row[i1 - N + m1];
        x[j] = v;
      }
      rf::fft<float, +1, H>(x);
      pl2::dit_combine<+1, N>(x, h);
      const int bA = P.pairs[2 * p], bB = P.pairs[2 * p + 1];
      const double fa = wocc[bA], fb = bB >= 0 ? wocc[bB] : 0.0;
      double *a = accs + l * N + h * H;
      rf::static_for<0, H>([&](auto kc) {
        constexpr int k = decltype(kc)::value, q = out_pos(H, k);
        const double re = x[q].x, im = x[q].y;
        a[k] += fa * re * re + fb * im * im;
      });
    }
    __syncthreads();
  }
  __syncthreads();
  double *dst = part + ((long)grp * P.k3 + i3) * N * N;
  for (int i = t; i < N * N; i += 2 * N) dst[i] = accs[i];
}

template <int NX, int NY>
int rho_launch(const PipeParams &P, int npl, const float2 *bufA, const double *wocc, double *part, double *rho,
               int accumulate, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_rho_plane<NX, NY, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_rho_plane<NX, NY, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 192 * 1024);
    attr = true;
  }
  const int per_group = (npl + RHO_GROUPS - 1) / RHO_GROUPS;
  const size_t sm1 = sizeof(double) * (size_t)NX * NY + sizeof(float2) * (size_t)NY * P.P1;
  if (P.P1 <= 32 && plane_pairs_enabled() && 2 * sm1 <= 192 * 1024) {
    dim3 g((P.k3 + 1) / 2, RHO_GROUPS);
    k_rho_plane<NX, NY, 2><<<g, 64, 2 * sm1, st>>>(P, bufA, wocc, part, npl, per_group);
  } else {
    dim3 g(P.k3, RHO_GROUPS);
    k_rho_plane<NX, NY, 1><<<g, 64, sm1, st>>>(P, bufA, wocc, part, npl, per_group);
  }
  note_launch();
  const long n = (long)P.k1 * P.k2 * P.k3;
  rho_groups_launch(part, n, rho, accumulate, st);
  return 0;
}

template <int N>
int rho2_launch(const PipeParams &P, int npl, const float2 *bufA, const double *wocc, double *part, double *rho,
                       int accumulate, cudaStream_t st) {
  const size_t sm = sizeof(double) * (size_t)N * N + sizeof(float2) * (size_t)N * P.P1;
  if (sm > 200 * 1024) return -1;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_rho_plane2<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  const int per_group = (npl + RHO_GROUPS - 1) / RHO_GROUPS;
  dim3 g(P.k3, RHO_GROUPS);
  k_rho_plane2<N><<<g, 2 * N, sm, st>>>(P, bufA, wocc, part, npl, per_group);
  note_launch();
  const long n = (long)P.k1 * P.k2 * P.k3;
  rho_groups_launch(part, n, rho, accumulate, st);
  return 0;
}

template <int NX, int NY>
int plane_launch(const PipeParams &P, int npl, float2 *bufA, const float *vloc, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_plane<NX, NY, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    cudaFuncSetAttribute(k_plane<NX, NY, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    attr = true;
  }
  if (P.P1 <= 32 && plane_pairs_enabled()) {   // two planes a CTA: warp w takes plane w's columns
    const size_t sm = sizeof(float2) * 2 * (size_t)NY * P.P1;
    dim3 g((P.k3 + 1) / 2, npl);
    k_plane<NX, NY, 2><<<g, 64, sm, st>>>(P, bufA, vloc);
  } else {
    const size_t sm = sizeof(float2) * (size_t)NY * P.P1;
    dim3 g(P.k3, npl);
    k_plane<NX, NY, 1><<<g, 64, sm, st>>>(P, bufA, vloc);
  }
  note_launch();
  return 0;
}

template <int N>
int plane2_launch(const PipeParams &P, int npl, float2 *bufA, const float *vloc, cudaStream_t st) {
  const size_t sm = sizeof(float2) * (size_t)N * P.P1;
  if (2 * P.P1 > 2 * N || sm > 100 * 1024) return -1;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_plane2<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    attr = true;
  }
  dim3 g(P.k3, npl);
  k_plane2<N><<<g, 2 * N, sm, st>>>(P, bufA, vloc);
  note_launch();
  return 0;
}

// Explicit instantiation of the launchers of one k1 x k2 plane shape.
#define QX_PLANE_GRID(NX, NY)                                                                                    \
  template int plane_launch<NX, NY>(const PipeParams &, int, float2 *, const float *, cudaStream_t);             \
  template int rho_launch<NX, NY>(const PipeParams &, int, const float2 *, const double *, double *, double *,   \
                                  int, cudaStream_t);
// ... and of the z-column launcher of one k3.
#define QX_ZCOLS_LENGTH(N)                                                                                      \
  template int zcols_launch<N>(const PipeParams &, int, const float *, long, float2 *, const float2 *, float2 *, \
                               bool, cudaStream_t);
// The same for the two-lanes-a-line kernels.
#define QX_PLANE_LENGTH2(N)                                                                                     \
  template int plane2_launch<N>(const PipeParams &, int, float2 *, const float *, cudaStream_t);                \
  template int rho2_launch<N>(const PipeParams &, int, const float2 *, const double *, double *, double *, int,  \
                              cudaStream_t);                                                                    \
  template int zcols2_launch<N>(const PipeParams &, int, const float *, long, float2 *, bool, cudaStream_t);

}  // namespace qx
