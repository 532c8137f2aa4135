// Fused y-x-y pass of the FP32 H|psi> pipeline for grids with k1 == k2 == N,
// one CTA per (band pair, z plane), one grid line per thread with the whole
// line in registers (compile-time-length FFTs of qx_regfft.cuh):
//   (1) backward y-FFT of each of the P1 sphere columns, read straight from
//       the z-transformed plane in bufA (rows outside the sphere are zero);
//   (2) per grid row: backward x-FFT (P1 non-zero inputs), times V_loc(r),
//       forward x-FFT, keep the P1 sphere columns;
//   (3) forward y-FFT of each column, the sphere rows written back to bufA.
// Between the steps the plane lives in shared memory as N x P1 complex
// values.  This replaces k_ypass<+1>, k_xvx and k_ypass<-1> (hcnonloc's
// c2r -> V_loc * psi -> r2c, engrad.f90:484-571) and removes the two round
// trips of bufB through L2/HBM.
#include "qx_internal.h"
#include "qx_regfft.cuh"

namespace qx {

template <int N>
__global__ void __launch_bounds__(64) k_plane(PipeParams P, float2 *__restrict__ bufA, const float *__restrict__ vloc) {
  using rf::out_pos;
  const int i3 = blockIdx.x;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= (P.npair_dev ? *P.npair_dev : P.npair)) return;
  const int P1 = P.P1, P2 = P.P2, m1 = P.m1, m2 = P.m2;
  extern __shared__ float2 T[];   // [N][P1]
  float2 *A = bufA + ((long)pl * P.k3 + i3) * P2 * P1;
  const int t = threadIdx.x;
  const float2 zero = make_float2(0.f, 0.f);

  // (1) y backward, thread = sphere column a
  if (t < P1) {
    float2 x[N];
#pragma unroll
    for (int i2 = 0; i2 < N; ++i2) {
      const int j2 = (i2 <= m2) ? i2 + m2 : ((i2 >= N - m2) ? i2 - N + m2 : -1);
      float2 v = zero;
      if (j2 >= 0 && t >= P.row_lo[j2] && t <= P.row_hi[j2]) v = A[j2 * P1 + t];
      x[i2] = v;
    }
    rf::fft<float, +1, N>(x);
    rf::static_for<0, N>([&](auto ic) {
      constexpr int i2 = decltype(ic)::value, q = out_pos(N, i2);
      T[i2 * P1 + t] = x[q];
    });
  }
  __syncthreads();
  // (2) x backward, * V, x forward; thread = grid row i2
  if (t < N) {
    float2 x[N];
    float2 *row = T + t * P1;
#pragma unroll
    for (int i1 = 0; i1 < N; ++i1) {
      float2 v = zero;
      if (i1 <= m1) v = row[i1 + m1];
      else if (i1 >= N - m1) v = row[i1 - N + m1];
      x[i1] = v;
    }
    rf::fft<float, +1, N>(x);
    const float *V = vloc + ((long)i3 * N + t) * N;
    float2 y[N];
    rf::static_for<0, N>([&](auto ic) {
      constexpr int i1 = decltype(ic)::value, q = out_pos(N, i1);
      const float vv = V[i1];
      y[i1] = make_float2(x[q].x * vv, x[q].y * vv);
    });
    rf::fft<float, -1, N>(y);
    rf::static_for<0, N>([&](auto ic) {
      constexpr int i1 = decltype(ic)::value, q = out_pos(N, i1);
      if (i1 <= m1) row[i1 + m1] = y[q];
      else if (i1 >= N - m1) row[i1 - N + m1] = y[q];
    });
  }
  __syncthreads();
  // (3) y forward, thread = sphere column a; only rows inside the sphere are kept
  if (t < P1) {
    float2 x[N];
#pragma unroll
    for (int i2 = 0; i2 < N; ++i2) x[i2] = T[i2 * P1 + t];
    rf::fft<float, -1, N>(x);
    rf::static_for<0, N>([&](auto ic) {
      constexpr int i2 = decltype(ic)::value, q = out_pos(N, i2);
      const int j2 = (i2 <= m2) ? i2 + m2 : ((i2 >= N - m2) ? i2 - N + m2 : -1);
      if (j2 >= 0 && t >= P.row_lo[j2] && t <= P.row_hi[j2]) A[j2 * P1 + t] = x[q];
    });
  }
}

template <int N>
static int plane_launch(const PipeParams &P, int npl, float2 *bufA, const float *vloc, cudaStream_t st) {
  const size_t sm = sizeof(float2) * (size_t)N * P.P1;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_plane<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    attr = true;
  }
  dim3 g(P.k3, npl);
  k_plane<N><<<g, 64, sm, st>>>(P, bufA, vloc);
  note_launch();
  return 0;
}

// Launch the fused pass if this grid has a specialised length; -1 otherwise.
int launch_plane_f32(const PipeParams &P, int npl, float2 *bufA, const float *vloc, cudaStream_t st) {
  if (P.k1 != P.k2 || P.P1 > P.k1 || P.P2 > P.k2) return -1;
  switch (P.k1) {
    case 20: return plane_launch<20>(P, npl, bufA, vloc, st);
    case 24: return plane_launch<24>(P, npl, bufA, vloc, st);
    case 27: return plane_launch<27>(P, npl, bufA, vloc, st);
    case 30: return plane_launch<30>(P, npl, bufA, vloc, st);
    case 32: return plane_launch<32>(P, npl, bufA, vloc, st);
    case 36: return plane_launch<36>(P, npl, bufA, vloc, st);
    case 40: return plane_launch<40>(P, npl, bufA, vloc, st);
    case 45: return plane_launch<45>(P, npl, bufA, vloc, st);
    case 48: return plane_launch<48>(P, npl, bufA, vloc, st);
    case 54: return plane_launch<54>(P, npl, bufA, vloc, st);
    case 60: return plane_launch<60>(P, npl, bufA, vloc, st);
    case 64: return plane_launch<64>(P, npl, bufA, vloc, st);
    default: return -1;
  }
}

}  // namespace qx
