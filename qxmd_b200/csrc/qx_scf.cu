// Density-side kernels of one SCF iteration, all FP64: Hartree potential
// (harting, engrad.f90:1673-1743), Perdew-Zunger LDA (xclda/VXC,
// vxc.f90:961-1018, 2063-2108, with the reference's single-precision
// literals), glocal assembly (pwlda.f90:1984-2024) and Kerker-filtered
// linear density mixing.  Reductions write per-block partial sums that a
// single block adds in a fixed order, so results are deterministic.
#include "qx_internal.h"
#include "qx_scf.h"

namespace qx {

constexpr int RB = 256;

__device__ __forceinline__ double block_sum_rb(double v, double *red) { return block_sum(v, red); }

// |G|^2 of every grid point, or -1 outside the density sphere (and 0 at G=0).
__global__ void k_grid_g2(int k1, int k2, int k3, double c00, double c01, double c02, double c10, double c11,
                          double c12, double c20, double c21, double c22, double ecutdens, double *__restrict__ g2) {
  const long n = (long)k1 * k2 * k3;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int i1 = (int)(i % k1), i2 = (int)((i / k1) % k2), i3 = (int)(i / ((long)k1 * k2));
    const double d1 = i1 <= k1 / 2 ? i1 : i1 - k1;
    const double d2 = i2 <= k2 / 2 ? i2 : i2 - k2;
    const double d3 = i3 <= k3 / 2 ? i3 : i3 - k3;
    const double gx = c00 * d1 + c01 * d2 + c02 * d3;
    const double gy = c10 * d1 + c11 * d2 + c12 * d3;
    const double gz = c20 * d1 + c21 * d2 + c22 * d3;
    const double s = gx * gx + gy * gy + gz * gz;
    g2[i] = (s <= ecutdens) ? s : -1.0;
  }
}

__global__ void k_real_to_cplx(const double *__restrict__ r, const double *__restrict__ r2, double2 *__restrict__ z,
                               long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    z[i] = make_double2(r2 ? r[i] - r2[i] : r[i], 0.0);
}

// V_H(G) = 8 pi rho(G) / |G|^2 inside the density sphere; E_H partial sums
// (Omega/2) sum_G V_H(G) conj(rho(G)).
__global__ void __launch_bounds__(RB) k_hartree(double2 *__restrict__ z, const double *__restrict__ g2, long n,
                                                double half_vol, double *__restrict__ part) {
  __shared__ double red[RB / 32];
  double e = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double q = g2[i];
    double2 v = z[i];
    if (q > 0.0) {
      const double f = 8.0 * 3.14159265358979323846 / q;
      e += f * (v.x * v.x + v.y * v.y);
      v.x *= f; v.y *= f;
    } else {
      v.x = 0.0; v.y = 0.0;
    }
    z[i] = v;
  }
  e = block_sum_rb(e, red);
  if (threadIdx.x == 0) part[blockIdx.x] = e * half_vol;
}

// Kerker filter of a density difference in G space: d(G) *= G^2/(G^2+q0^2)
// inside the density sphere, 0 at G = 0 and outside.
__global__ void k_kerker(double2 *__restrict__ z, const double *__restrict__ g2, long n, double q02) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double q = g2[i];
    double2 v = z[i];
    const double f = (q > 0.0) ? q / (q + q02) : 0.0;
    v.x *= f; v.y *= f;
    z[i] = v;
  }
}

// PZ LDA on rho, glocal = vloc + Re(vh) + vxc; partial sums of
// eps_xc*rho and vxc*rho (times rdelv).
template <typename T>
__global__ void __launch_bounds__(RB) k_xc_glocal(const double *__restrict__ rho, const double *__restrict__ vloc,
                                                  const double2 *__restrict__ vh, long n, double rdelv,
                                                  double *__restrict__ glocal, T *__restrict__ glocal_t,
                                                  double *__restrict__ part) {
  __shared__ double red[RB / 32];
  const double pi4 = 12.56637061436;
  const double a1 = -0.4582, b1 = -0.1423, b2 = (double)1.0529f, b3 = (double)0.3334f;
  const double c1 = -0.0480, c2 = (double)0.0311f, c3 = (double)-0.0116f, c4 = (double)0.0020f;
  double sx = 0.0, sv = 0.0;
  for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < n; m += (long)gridDim.x * blockDim.x) {
    const double rh = rho[m];
    double vexc = 0.0, eexc = 0.0;
    if (rh >= 1e-30) {
      const double rs = cbrt(3.0 / (pi4 * rh));
      const double ex = a1 / rs, vx = 4.0 * ex / 3.0;
      double ec, vc;
      if (rs >= 1.0) {
        const double srs = sqrt(rs);
        const double bunb = 1.0 + b2 * srs + b3 * rs;
        ec = b1 / bunb;
        vc = ec * (1.0 + (b2 * srs / 6.0 + b3 * rs / 3.0) / bunb);
      } else {
        const double lr = log(rs);
        ec = c1 + c2 * lr + c3 * rs + c4 * rs * lr;
        vc = ec - (c2 + (c3 + c4) * rs + c4 * rs * lr) / 3.0;
      }
      vexc = 2.0 * (vx + vc);
      eexc = 2.0 * (ex + ec);
    }
    const double g = vloc[m] + vh[m].x + vexc;
    glocal[m] = g;
    glocal_t[m] = (T)g;
    sx += eexc * rh;
    sv += vexc * rh;
  }
  sx = block_sum_rb(sx, red);
  sv = block_sum_rb(sv, red);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sx * rdelv;
    part[2 * blockIdx.x + 1] = sv * rdelv;
  }
}

// rho_in += beta * Re(filtered difference); partial sums of the residual
// |rho_out - rho_in|^2 * rdelv taken before the update.
__global__ void __launch_bounds__(RB) k_mix(double *__restrict__ rho_in, const double *__restrict__ rho_out,
                                            const double2 *__restrict__ dfilt, long n, double beta, double rdelv,
                                            double *__restrict__ part) {
  __shared__ double red[RB / 32];
  double s = 0.0;
  for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < n; m += (long)gridDim.x * blockDim.x) {
    const double d = rho_out[m] - rho_in[m];
    s += d * d;
    rho_in[m] += beta * dfilt[m].x;
  }
  s = block_sum_rb(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s * rdelv;
}

// out[k] = sum over nblk partial sums with stride `stride` and offset k.
// One warp per output: lane-strided partial sums, then a shuffle tree (a fixed
// order, so the result does not change from run to run).
__global__ void k_reduce(const double *__restrict__ part, int nblk, int stride, int nk, double *__restrict__ out) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = w; k < nk; k += blockDim.x >> 5) {
    double s = 0.0;
    for (int b = lane; b < nblk; b += 32) s += part[(long)b * stride + k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[k] = s;
  }
}

// sum_b occ_b * w_b
__global__ void k_band_energy(const double *__restrict__ w, const double *__restrict__ occ, int nb,
                              double *__restrict__ out) {
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += occ[b] * w[b];
    *out = s;
  }
}

// ---- launchers -------------------------------------------------------------
void grid_g2(int k1, int k2, int k3, const double *cross, double ecutdens, double *g2, cudaStream_t st) {
  k_grid_g2<<<148 * 4, 256, 0, st>>>(k1, k2, k3, cross[0], cross[3], cross[6], cross[1], cross[4], cross[7],
                                    cross[2], cross[5], cross[8], ecutdens, g2); note_launch();
}

void real_to_cplx(const double *r, const double *r2, double2 *z, long n, cudaStream_t st) {
  k_real_to_cplx<<<148 * 4, 256, 0, st>>>(r, r2, z, n); note_launch();
}

void hartree_g(double2 *z, const double *g2, long n, double half_vol, double *part, double *out, cudaStream_t st) {
  k_hartree<<<SCF_NBLK, RB, 0, st>>>(z, g2, n, half_vol, part); note_launch();
  k_reduce<<<1, 32, 0, st>>>(part, SCF_NBLK, 1, 1, out); note_launch();
}

void kerker(double2 *z, const double *g2, long n, double q02, cudaStream_t st) {
  k_kerker<<<148 * 4, 256, 0, st>>>(z, g2, n, q02); note_launch();
}

template <typename T>
void xc_glocal(const double *rho, const double *vloc, const double2 *vh, long n, double rdelv, double *glocal,
               T *glocal_t, double *part, double *out2, cudaStream_t st) {
  k_xc_glocal<T><<<SCF_NBLK, RB, 0, st>>>(rho, vloc, vh, n, rdelv, glocal, glocal_t, part); note_launch();
  k_reduce<<<1, 64, 0, st>>>(part, SCF_NBLK, 2, 2, out2); note_launch();
}
template void xc_glocal<float>(const double *, const double *, const double2 *, long, double, double *, float *,
                               double *, double *, cudaStream_t);
template void xc_glocal<double>(const double *, const double *, const double2 *, long, double, double *, double *,
                                double *, double *, cudaStream_t);

void mix(double *rho_in, const double *rho_out, const double2 *dfilt, long n, double beta, double rdelv, double *part,
         double *out, cudaStream_t st) {
  k_mix<<<SCF_NBLK, RB, 0, st>>>(rho_in, rho_out, dfilt, n, beta, rdelv, part); note_launch();
  k_reduce<<<1, 32, 0, st>>>(part, SCF_NBLK, 1, 1, out); note_launch();
}

void band_energy(const double *w, const double *occ, int nb, double *out, cudaStream_t st) {
  k_band_energy<<<1, 32, 0, st>>>(w, occ, nb, out); note_launch();
}

}  // namespace qx
