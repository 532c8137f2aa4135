// Launchers of the FP64 density-side kernels.
#pragma once
#include <cuda_runtime.h>

namespace qx {

constexpr int SCF_NBLK = 296;   // partial-sum blocks (2 per SM)
constexpr int PULAY_MAX = 16;   // longest Pulay history

// Pulay mixing state on the device (see qx_scf.cu).
struct PulayDev {
  int cnt, slot, reset_next, pad;
  int order[PULAY_MAX];
  double coef[PULAY_MAX];
  double A[PULAY_MAX * PULAY_MAX];
};
struct PulayState {
  PulayDev *s;
  double2 *u, *d;   // itratn history slots of n complex values each
  int itratn;
  double q1;
};
void pulay_push(const PulayState &p, int reset, cudaStream_t st);
void pack2(const double *rin, const double *rout, double2 *z, long n, cudaStream_t st);
void pulay_store(const double2 *z, const double *g2, int k1, int k2, int k3, const PulayState &p, cudaStream_t st);
void pulay_coef(const double *g2, long n, const PulayState &p, double rvol, double *part, double *adot,
                cudaStream_t st);
void pulay_new(const double *g2, long n, const PulayState &p, double aslh, double bslh, double2 *z, cudaStream_t st);
void take_real(double *rho_in, const double *rho_out, const double2 *z, long n, double rdelv, double *part,
               double *out, cudaStream_t st);

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
