// Launchers of the fused FFT plane kernels (qx_fftplane_kern.cuh), one per
// specialised grid length N, explicitly instantiated in the qx_fftplane_*.cu
// files.  Each returns 0 after queuing its kernels on st, or -1 if the plane
// does not fit the kernel (the caller then takes the generic passes).
#pragma once
#include "qx_internal.h"

namespace qx {

// One grid line per thread (N in 20..64).
template <int N>
int plane_launch(const PipeParams &P, int npl, float2 *bufA, const float *vloc, cudaStream_t st);
template <int N>
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

// QX_PLANE_PAIRS=0 keeps one z plane a CTA (read at every call).
bool plane_pairs_enabled();

// rho = [rho +] the sum of the RHO_GROUPS partial planes in part, in group order.
void rho_groups_launch(const double *part, long n, double *rho, int accumulate, cudaStream_t st);

}  // namespace qx
