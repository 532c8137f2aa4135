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
#define QX_CASE(N) \
  case N: return zcols_launch<N>(P, npl, cin, ldc, bufA, src, zsph, inv, st);
    QX_ZCOLS_LENGTHS(QX_CASE)
#undef QX_CASE
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
  if (P.P1 > P.k1 || P.P2 > P.k2 || !part) return -1;
  switch (plane_grid_key(P.k1, P.k2)) {
#define QX_CASE(NX, NY) \
  case plane_grid_key(NX, NY): return rho_launch<NX, NY>(P, npl, bufA, wocc, part, rho, accumulate, st);
    QX_PLANE_GRIDS(QX_CASE)
#undef QX_CASE
    case plane_grid_key(96, 96): return rho2_launch<96>(P, npl, bufA, wocc, part, rho, accumulate, st);
    default: return -1;
  }
}

bool plane_length_supported(int k1, int k2) {
  switch (plane_grid_key(k1, k2)) {
#define QX_CASE(NX, NY) case plane_grid_key(NX, NY):
    QX_PLANE_GRIDS(QX_CASE)
#undef QX_CASE
    case plane_grid_key(96, 96):
      return true;
    default:
      return false;
  }
}

// Launch the fused pass if this grid has a specialised length; -1 otherwise.
int launch_plane_f32(const PipeParams &P, int npl, float2 *bufA, const float *vloc, cudaStream_t st) {
  if (P.P1 > P.k1 || P.P2 > P.k2) return -1;
  switch (plane_grid_key(P.k1, P.k2)) {
#define QX_CASE(NX, NY) \
  case plane_grid_key(NX, NY): return plane_launch<NX, NY>(P, npl, bufA, vloc, st);
    QX_PLANE_GRIDS(QX_CASE)
#undef QX_CASE
    case plane_grid_key(96, 96): return plane2_launch<96>(P, npl, bufA, vloc, st);
    default: return -1;
  }
}

}  // namespace qx
