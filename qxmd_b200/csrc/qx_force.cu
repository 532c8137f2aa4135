// Hellmann-Feynman forces of the Kohn-Sham state on the device:
//  * floc, the local pseudopotential in G space (flocal_g, nlkbpp.f90:1037-1120):
//      F_a = 2 sum_{G != 0, half sphere} G svco(G) (Re rho(G) sin(G.R_a) + Im rho(G) cos(G.R_a)),
//    with cos/sin(G.R_a) composed from per-dimension phase tables built by the
//    angle-addition recurrence of stscfn (bulk.f90:2086-2175);
//  * fnl, the G-space Kleinman-Bylander term (kbnlpp_frc2, nlkbpp.f90:1878-2130):
//      F_a = 4 sum_n occ_n sum_l vclalp_l P_{la,n} D_{la,n},
//    P = <beta|psi> with the KB metric and D = sum_{G != 0} G (beta_re psi_im - beta_im psi_re),
//    both as contractions over the half sphere (D through derivative tables
//    d(2g) = -G beta(2g+1), d(2g+1) = G beta(2g), built once per geometry).
// All sums in FP64 in a fixed order.
#include "qx_internal.h"

namespace qx {

constexpr int FT = 256;

// dcq/dsq[(a * 3 + dim) * ktot + koff[dim] + k + kmax[dim]] = cos/sin(2 pi k s_dim(a)),
// k = -kmax..kmax: the recurrence of stscfn.
__global__ void k_phase_tables(int natom, const double *__restrict__ satm, int km1, int km2, int km3, int ktot,
                               double *__restrict__ dcq, double *__restrict__ dsq) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * natom) return;
  const int a = t / 3, dim = t - 3 * a;
  const int km = dim == 0 ? km1 : (dim == 1 ? km2 : km3);
  const int off = dim == 0 ? 0 : (dim == 1 ? 2 * km1 + 1 : 2 * km1 + 2 * km2 + 2);
  double *c = dcq + (long)a * ktot + off + km, *s = dsq + (long)a * ktot + off + km;
  const double ph = satm[3 * a + dim] * (2.0 * 3.14159265358979323846);
  const double c1 = cos(ph), s1 = sin(ph);
  c[0] = 1.0;
  s[0] = 0.0;
  if (km >= 1) {
    c[1] = c1; s[1] = s1;
    c[-1] = c1; s[-1] = -s1;
  }
  double cp = c1, sp = s1;
  for (int k = 2; k <= km; ++k) {
    const double cn = c1 * cp - s1 * sp, sn = s1 * cp + c1 * sp;
    c[k] = cn; s[k] = sn;
    c[-k] = cn; s[-k] = -sn;
    cp = cn; sp = sn;
  }
}

// vlocal_g (nlkbpp.f90:862-1036): V(G) = (1/Omega) sum_a svco(G, type of a)
// (cos G.R_a, -sin G.R_a) on the density half sphere, written at +G and, as
// its conjugate, at -G of the full complex grid (zeroed before); one thread
// per G, atoms summed in order.
__global__ void k_vloc_g(int n5, int natom, const int *__restrict__ ijk5, const int *__restrict__ ngabc,
                         const double *__restrict__ svco, const int *__restrict__ ityp, const double *__restrict__ dcq,
                         const double *__restrict__ dsq, int km1, int km2, int km3, int ktot, double rvolr, int k1n,
                         int k2n, int k3n, double2 *__restrict__ zg) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n5) return;
  const int k1 = ngabc[3 * g], k2 = ngabc[3 * g + 1], k3 = ngabc[3 * g + 2];
  double re = 0.0, im = 0.0;
  for (int a = 0; a < natom; ++a) {
    const double *c1 = dcq + (long)a * ktot + km1, *s1 = dsq + (long)a * ktot + km1;
    const double *c2 = dcq + (long)a * ktot + 2 * km1 + 1 + km2, *s2 = dsq + (long)a * ktot + 2 * km1 + 1 + km2;
    const double *c3 = dcq + (long)a * ktot + 2 * km1 + 2 * km2 + 2 + km3,
                 *s3 = dsq + (long)a * ktot + 2 * km1 + 2 * km2 + 2 + km3;
    const double cc12 = c1[k1] * c2[k2] - s1[k1] * s2[k2];
    const double sc12 = s1[k1] * c2[k2] + c1[k1] * s2[k2];
    const double zc = cc12 * c3[k3] - sc12 * s3[k3];
    const double zs = sc12 * c3[k3] + cc12 * s3[k3];
    const double sv = svco[(long)ityp[a] * n5 + g] * rvolr;
    re += sv * zc;
    im -= sv * zs;
  }
  zg[ijk5[g]] = make_double2(re, im);
  if (g > 0) {
    const int m1 = (k1n - k1 % k1n) % k1n, m2 = (k2n - k2 % k2n) % k2n, m3 = (k3n - k3 % k3n) % k3n;
    zg[m1 + (long)k1n * (m2 + (long)k2n * m3)] = make_double2(re, -im);
  }
}

__global__ void k_real_part(const double2 *__restrict__ z, double *__restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = z[i].x;
}

void real_part(const double2 *z, double *out, long n, cudaStream_t st) {
  k_real_part<<<4 * 148, 256, 0, st>>>(z, out, n);
  note_launch();
}

void vloc_g(int n5, int natom, const int *ijk5, const int *ngabc, const double *svco, const int *ityp,
            const double *dcq, const double *dsq, int km1, int km2, int km3, int ktot, double rvol, int k1, int k2,
            int k3, double2 *zg, cudaStream_t st) {
  k_vloc_g<<<(n5 + 255) / 256, 256, 0, st>>>(n5, natom, ijk5, ngabc, svco, ityp, dcq, dsq, km1, km2, km3, ktot,
                                             1.0 / rvol, k1, k2, k3, zg);
  note_launch();
}

// One block per atom: the three components of floc, G = 0 excluded.
__global__ void __launch_bounds__(FT) k_floc(int n5, const int *__restrict__ ijk5, const int *__restrict__ ngabc,
                                             const double *__restrict__ gvec5, const double *__restrict__ svco,
                                             const int *__restrict__ ityp, const double2 *__restrict__ rhog,
                                             const double *__restrict__ dcq, const double *__restrict__ dsq,
                                             int km1, int km2, int km3, int ktot, double *__restrict__ floc) {
  __shared__ double red[FT / 32];
  const int a = blockIdx.x;
  const double *c1 = dcq + (long)a * ktot + km1, *s1 = dsq + (long)a * ktot + km1;
  const double *c2 = dcq + (long)a * ktot + 2 * km1 + 1 + km2, *s2 = dsq + (long)a * ktot + 2 * km1 + 1 + km2;
  const double *c3 = dcq + (long)a * ktot + 2 * km1 + 2 * km2 + 2 + km3,
               *s3 = dsq + (long)a * ktot + 2 * km1 + 2 * km2 + 2 + km3;
  const double *sv = svco + (long)ityp[a] * n5;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (int g = 1 + threadIdx.x; g < n5; g += FT) {
    const int k1 = ngabc[3 * g], k2 = ngabc[3 * g + 1], k3 = ngabc[3 * g + 2];
    const double cc12 = c1[k1] * c2[k2] - s1[k1] * s2[k2];
    const double sc12 = s1[k1] * c2[k2] + c1[k1] * s2[k2];
    const double zc = cc12 * c3[k3] - sc12 * s3[k3];
    const double zs = sc12 * c3[k3] + cc12 * s3[k3];
    const double2 r = rhog[ijk5[g]];
    const double f = sv[g] * (r.x * zs + r.y * zc);
    fx += f * gvec5[3 * g];
    fy += f * gvec5[3 * g + 1];
    fz += f * gvec5[3 * g + 2];
  }
  fx = block_sum(fx, red);
  fy = block_sum(fy, red);
  fz = block_sum(fz, red);
  if (threadIdx.x == 0) {
    floc[3 * a] = 2.0 * fx;
    floc[3 * a + 1] = 2.0 * fy;
    floc[3 * a + 2] = 2.0 * fz;
  }
}

// Derivative tables dtab[dim][j][.] from kbg[j][.] (both [nproj][nplwex]):
// entries of G index g >= 1: d(2g) = -G_dim(g) beta(2g+1), d(2g+1) = G_dim(g) beta(2g); G = 0 gives 0.
template <typename T>
__global__ void k_dtab(int nproj, int nplw, const T *__restrict__ kbg, const double *__restrict__ gw,
                       T *__restrict__ dtab) {
  const long ne = 2L * (nplw + 1);
  const long tot = (long)nproj * (nplw + 1);
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < tot; q += (long)gridDim.x * blockDim.x) {
    const int j = (int)(q / (nplw + 1)), g = (int)(q - (long)j * (nplw + 1));
    const double br = (double)kbg[j * ne + 2 * g], bi = (double)kbg[j * ne + 2 * g + 1];
#pragma unroll
    for (int dim = 0; dim < 3; ++dim) {
      const double gd = (g == 0) ? 0.0 : gw[3 * g + dim];
      T *d = dtab + ((long)dim * nproj + j) * ne;
      d[2 * g] = (T)(-gd * bi);
      d[2 * g + 1] = (T)(gd * br);
    }
  }
}

// One block per atom: fnl(dim, a) = 4 sum_n occ_n sum_l vclalp_l P(la, n) D(dim, la, n).
// P: nproj x nb (column n at P + n * nproj); D: 3 nproj x nb (row dim * nproj + j).
template <typename T>
__global__ void __launch_bounds__(FT) k_fnl(int lmx, int nproj, int nb, const T *__restrict__ P,
                                            const T *__restrict__ D, const T *__restrict__ vclalp,
                                            const double *__restrict__ occ, double *__restrict__ fnl) {
  __shared__ double red[FT / 32];
  const int a = blockIdx.x;
  double f[3] = {0.0, 0.0, 0.0};
  for (int q = threadIdx.x; q < lmx * nb; q += FT) {
    const int n = q / lmx, l = q - n * lmx, j = l + lmx * a;
    const double w = occ[n] * (double)vclalp[j] * (double)P[(long)n * nproj + j];
#pragma unroll
    for (int dim = 0; dim < 3; ++dim) f[dim] += w * (double)D[(long)n * 3 * nproj + dim * nproj + j];
  }
#pragma unroll
  for (int dim = 0; dim < 3; ++dim) {
    const double s = block_sum(f[dim], red);
    if (threadIdx.x == 0) fnl[3 * a + dim] = 4.0 * s;
  }
}

// ---- launchers ---------------------------------------------------------------
void phase_tables(int natom, const double *satm, int km1, int km2, int km3, int ktot, double *dcq, double *dsq,
                  cudaStream_t st) {
  k_phase_tables<<<(3 * natom + 127) / 128, 128, 0, st>>>(natom, satm, km1, km2, km3, ktot, dcq, dsq);
  note_launch();
}
void floc_g(int natom, int n5, const int *ijk5, const int *ngabc, const double *gvec5, const double *svco,
            const int *ityp, const double2 *rhog, const double *dcq, const double *dsq, int km1, int km2, int km3,
            int ktot, double *floc, cudaStream_t st) {
  k_floc<<<natom, FT, 0, st>>>(n5, ijk5, ngabc, gvec5, svco, ityp, rhog, dcq, dsq, km1, km2, km3, ktot, floc);
  note_launch();
}
template <typename T>
void dtab_build(int nproj, int nplw, const T *kbg, const double *gw, T *dtab, cudaStream_t st) {
  k_dtab<T><<<148 * 4, 256, 0, st>>>(nproj, nplw, kbg, gw, dtab);
  note_launch();
}
template <typename T>
void fnl_reduce(int natom, int lmx, int nproj, int nb, const T *P, const T *D, const T *vclalp, const double *occ,
                double *fnl, cudaStream_t st) {
  k_fnl<T><<<natom, FT, 0, st>>>(lmx, nproj, nb, P, D, vclalp, occ, fnl);
  note_launch();
}
template void dtab_build<float>(int, int, const float *, const double *, float *, cudaStream_t);
template void dtab_build<double>(int, int, const double *, const double *, double *, cudaStream_t);
template void fnl_reduce<float>(int, int, int, int, const float *, const float *, const float *, const double *,
                                double *, cudaStream_t);
template void fnl_reduce<double>(int, int, int, int, const double *, const double *, const double *,
                                 const double *, double *, cudaStream_t);

}  // namespace qx
