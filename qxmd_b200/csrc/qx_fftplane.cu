// Dispatch of the fused FFT plane passes of the FP32 H|psi> pipeline on the
// grid length: the kernels are in qx_fftplane_kern.cuh, their launchers are
// instantiated per length in the qx_fftplane_*.cu files.
#include "qx_fftplane.h"

namespace qx {

bool plane_pairs_enabled() {
  const char *e = getenv("QX_PLANE_PAIRS");
  return !(e && e[0] == '0');
}

// QX_ZCOLS=0 keeps the shared-memory z passes (read at every call).
static bool zcols_enabled() {
  const char *e = getenv("QX_ZCOLS");
  return !(e && e[0] == '0');
}

static int zcols_dispatch(const PipeParams &P, int npl, const float *cin, long ldc, float2 *bufA, const float2 *src,
                          float2 *zsph, bool inv, cudaStream_t st) {
  if (!zcols_enabled() || P.ncol <= 0) return -1;
  switch (P.k3) {
    case 20: return zcols_launch<20>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 21: return zcols_launch<21>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 24: return zcols_launch<24>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 25: return zcols_launch<25>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 27: return zcols_launch<27>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 30: return zcols_launch<30>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 32: return zcols_launch<32>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 36: return zcols_launch<36>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 40: return zcols_launch<40>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 42: return zcols_launch<42>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 45: return zcols_launch<45>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 48: return zcols_launch<48>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 49: return zcols_launch<49>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 54: return zcols_launch<54>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 60: return zcols_launch<60>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 64: return zcols_launch<64>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    case 96: return zcols2_launch<96>(P, npl, cin, ldc, bufA, inv, st);
    default: return -1;
  }
}

int launch_zcols_inv_f32(const PipeParams &P, int npl, const float *cin, long ldc, float2 *bufA, cudaStream_t st) {
  return zcols_dispatch(P, npl, cin, ldc, bufA, nullptr, nullptr, true, st);
}
int launch_zcols_fwd_f32(const PipeParams &P, int npl, const float2 *bufA, float2 *zsph, cudaStream_t st) {
  return zcols_dispatch(P, npl, nullptr, 0, nullptr, bufA, zsph, false, st);
}

// Sum of the RHO_GROUPS partial planes in group order (all loads of an
// element issued together).
__global__ void k_rho_groups(const double *__restrict__ part, long n, double *__restrict__ rho, int accumulate) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double v[RHO_GROUPS];
#pragma unroll
    for (int g = 0; g < RHO_GROUPS; ++g) v[g] = part[(long)g * n + i];
    double s = accumulate ? rho[i] : 0.0;
#pragma unroll
    for (int g = 0; g < RHO_GROUPS; ++g) s += v[g];
    rho[i] = s;
  }
}

void rho_groups_launch(const double *part, long n, double *rho, int accumulate, cudaStream_t st) {
  k_rho_groups<<<148 * 4, 256, 0, st>>>(part, n, rho, accumulate);
  note_launch();
}

// Density of one chunk of pairs through the plane kernel; -1 if the grid has
// no specialised length.  part: RHO_GROUPS * kfft0 doubles.
int launch_rho_plane_f32(const PipeParams &P, int npl, const float2 *bufA, const double *wocc, double *part,
                         double *rho, int accumulate, cudaStream_t st) {
  if (P.k1 != P.k2 || P.P1 > P.k1 || P.P2 > P.k2 || !part) return -1;
  switch (P.k1) {
    case 20: return rho_launch<20>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 21: return rho_launch<21>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 24: return rho_launch<24>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 25: return rho_launch<25>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 27: return rho_launch<27>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 30: return rho_launch<30>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 32: return rho_launch<32>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 36: return rho_launch<36>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 40: return rho_launch<40>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 42: return rho_launch<42>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 45: return rho_launch<45>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 48: return rho_launch<48>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 49: return rho_launch<49>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 54: return rho_launch<54>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 60: return rho_launch<60>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 64: return rho_launch<64>(P, npl, bufA, wocc, part, rho, accumulate, st);
    case 96: return rho2_launch<96>(P, npl, bufA, wocc, part, rho, accumulate, st);
    default: return -1;
  }
}

bool plane_length_supported(int k1, int k2) {
  if (k1 != k2) return false;
  switch (k1) {
    case 20: case 21: case 24: case 25: case 27: case 30: case 32: case 36: case 40: case 42: case 45: case 48:
    case 49: case 54: case 60: case 64: case 96:
      return true;
    default:
      return false;
  }
}

// Launch the fused pass if this grid has a specialised length; -1 otherwise.
int launch_plane_f32(const PipeParams &P, int npl, float2 *bufA, const float *vloc, cudaStream_t st) {
  if (P.k1 != P.k2 || P.P1 > P.k1 || P.P2 > P.k2) return -1;
  switch (P.k1) {
    case 20: return plane_launch<20>(P, npl, bufA, vloc, st);
    case 21: return plane_launch<21>(P, npl, bufA, vloc, st);
    case 24: return plane_launch<24>(P, npl, bufA, vloc, st);
    case 25: return plane_launch<25>(P, npl, bufA, vloc, st);
    case 27: return plane_launch<27>(P, npl, bufA, vloc, st);
    case 30: return plane_launch<30>(P, npl, bufA, vloc, st);
    case 32: return plane_launch<32>(P, npl, bufA, vloc, st);
    case 36: return plane_launch<36>(P, npl, bufA, vloc, st);
    case 40: return plane_launch<40>(P, npl, bufA, vloc, st);
    case 42: return plane_launch<42>(P, npl, bufA, vloc, st);
    case 45: return plane_launch<45>(P, npl, bufA, vloc, st);
    case 48: return plane_launch<48>(P, npl, bufA, vloc, st);
    case 49: return plane_launch<49>(P, npl, bufA, vloc, st);
    case 54: return plane_launch<54>(P, npl, bufA, vloc, st);
    case 60: return plane_launch<60>(P, npl, bufA, vloc, st);
    case 64: return plane_launch<64>(P, npl, bufA, vloc, st);
    case 96: return plane2_launch<96>(P, npl, bufA, vloc, st);
    default: return -1;
  }
}

}  // namespace qx
