// Launchers of the FP64 density-side kernels.
#pragma once
#include <cuda_runtime.h>

namespace qx {

constexpr int SCF_NBLK = 296;   // partial-sum blocks (2 per SM)

void grid_g2(int k1, int k2, int k3, const double *cross, double ecutdens, double *g2, cudaStream_t st);
void real_to_cplx(const double *r, const double *r2, double2 *z, long n, cudaStream_t st);
void hartree_g(double2 *z, const double *g2, long n, double half_vol, double *part, double *out, cudaStream_t st);
void kerker(double2 *z, const double *g2, long n, double q02, cudaStream_t st);
template <typename T>
void xc_glocal(const double *rho, const double *vloc, const double2 *vh, long n, double rdelv, double *glocal,
               T *glocal_t, double *part, double *out2, cudaStream_t st);
void mix(double *rho_in, const double *rho_out, const double2 *dfilt, long n, double beta, double rdelv, double *part,
         double *out, cudaStream_t st);
void band_energy(const double *w, const double *occ, int nb, double *out, cudaStream_t st);

}  // namespace qx
