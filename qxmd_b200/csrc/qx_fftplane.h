// Launchers of the fused FFT plane kernels (qx_fftplane_kern.cuh), one per
// specialised plane shape or z length, explicitly instantiated in the
// qx_fftplane_*.cu files.  Each returns 0 after queuing its kernels on st,
// or -1 if the plane does not fit the kernel (the caller then takes the
// generic passes).
#pragma once
#include "qx_internal.h"

namespace qx {

// One grid line per thread: planes of NX = k1 by NY = k2 points (each at
// most 64), z columns of N = k3 points.
template <int NX, int NY>
int plane_launch(const PipeParams &P, int npl, float2 *bufA, const float *vloc, cudaStream_t st);
template <int NX, int NY>
int rho_launch(const PipeParams &P, int npl, const float2 *bufA, const double *wocc, double *part, double *rho,
               int accumulate, cudaStream_t st);
template <int N>
int zcols_launch(const PipeParams &P, int npl, const float *cin, long ldc, float2 *bufA, const float2 *src,
                 float2 *zsph, bool inv, cudaStream_t st);

// Two lanes a line (N = 96).
template <int N>
int plane2_launch(const PipeParams &P, int npl, float2 *bufA, const float *vloc, cudaStream_t st);
template <int N>
int rho2_launch(const PipeParams &P, int npl, const float2 *bufA, const double *wocc, double *part, double *rho,
                int accumulate, cudaStream_t st);
template <int N>
int zcols2_launch(const PipeParams &P, int npl, const float *cin, long ldc, float2 *bufA, bool inv,
                  cudaStream_t st);

// The k1 x k2 plane shapes with register kernels, X(k1, k2): the square
// grids of 20 to 64 points built from radices 2, 3, 5 and 7, and the
// elongated cells of the 48-cell batch (two or three primitive cells along
// x).  The same list drives the dispatch and the instantiation files.
#define QX_PLANE_GRIDS(X)                                                                              \
  X(20, 20) X(21, 21) X(24, 24) X(25, 25) X(27, 27) X(30, 30) X(32, 32) X(36, 36) X(40, 40) X(42, 42) \
  X(45, 45) X(48, 48) X(49, 49) X(54, 54) X(60, 60) X(64, 64)                                         \
  X(24, 25) X(25, 24) X(25, 27) X(27, 25) X(42, 21) X(45, 24) X(45, 42) X(48, 45) X(49, 25) X(54, 24) \
  X(54, 25) X(54, 27)
// The z lengths with register column kernels.
#define QX_ZCOLS_LENGTHS(X) \
  X(20) X(21) X(24) X(25) X(27) X(30) X(32) X(36) X(40) X(42) X(45) X(48) X(49) X(54) X(60) X(64)

constexpr int plane_grid_key(int k1, int k2) { return k1 * 1024 + k2; }

// QX_PLANE_PAIRS=0 keeps one z plane a CTA (read at every call).
bool plane_pairs_enabled();

// rho = [rho +] the sum of the RHO_GROUPS partial planes in part, in group order.
void rho_groups_launch(const double *part, long n, double *rho, int accumulate, cudaStream_t st);

}  // namespace qx
