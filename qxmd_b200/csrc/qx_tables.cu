// Geometry-dependent G-space KB projector tables built on the device, so that
// an MD step rebuilds eqlmr_ without a host round trip:
//  * k_setqlm, once per cell (setqlm, nlkbpp.f90:2196-2247): the radial table
//    tbqlm(0:mxqlm) of each (channel, species), step dlqlm, interpolated at |G|
//    by the three-point forward-difference formula
//      m = 2 int(|G| / (2 dl)), d = (|G| / dl - m) / 2,
//      f = d ((d - 1) a_m + t_{m+2} - t_m) + t_m,  a_m = 2 (t_m + t_{m+2} - 2 t_{m+1})
//    (a_m is tbqlma, ppkb.f90:3228-3236), times the angular factor qlm(G)
//    of the channel;
//  * k_setbgq, once per geometry (setbgq, nlkbpp.f90:2135-2187): with the
//    structure phases cos/sin(G.R_a) composed from the per-dimension
//    recurrence tables of stscfn_pw (pwlda.f90:5711-5850),
//      even l: eqlmr_(2g+1) =  cos f,  eqlmr_(2g+2) = -sin f
//      odd l:  eqlmr_(2g+1) = -sin f,  eqlmr_(2g+2) = -cos f
//    written straight into the context's projector table (and its padded
//    FP32 copy) together with the per-projector KB energies.
#include "qx_internal.h"

namespace qx {

__global__ void k_setqlm(int nplw1, int nchan, int lmx, int mxqlm, const double *__restrict__ dlqlm,
                         const double *__restrict__ tbqlm, const double *__restrict__ qlm,
                         const int *__restrict__ lmidx, const double *__restrict__ dk, double *__restrict__ zzz) {
  const long tot = (long)nplw1 * nchan;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < tot; q += (long)gridDim.x * blockDim.x) {
    const int ch = (int)(q / nplw1), g = (int)(q - (long)ch * nplw1);
    const int it = ch / lmx;
    const double dl = dlqlm[it];
    const double ag = sqrt(dk[2 * g]);
    const int m = 2 * (int)(ag / (2.0 * dl));
    const double d = 0.5 * (ag / dl - (double)m);
    const double *t = tbqlm + (long)ch * (mxqlm + 1);
    const double t0 = t[m], t1 = t[m + 1], t2 = t[m + 2];
    const double a = 2.0 * (t0 + t2 - 2.0 * t1);
    const double f = d * ((d - 1.0) * a + t2 - t0) + t0;
    zzz[q] = f * qlm[(long)lmidx[ch] * nplw1 + g];
  }
}

// blockIdx.y = atom; one half-sphere G per thread, all lmx projectors of the atom.
template <typename T>
__global__ void k_setbgq(int nplw1, int ne, int lmx, const int *__restrict__ ityp, const int *__restrict__ ngabc,
                         const double *__restrict__ dcq, const double *__restrict__ dsq, int km1, int km2, int km3,
                         int ktot, const double *__restrict__ zzz, const int *__restrict__ even,
                         const double *__restrict__ vcl_type, T *__restrict__ kbg, float *__restrict__ kbgp, long ldp,
                         T *__restrict__ vcl) {
  const int a = blockIdx.y;
  const int it = ityp[a];
  const double *cq = dcq + (long)a * ktot, *sq = dsq + (long)a * ktot;
  const int o2 = 2 * km1 + 1, o3 = 2 * km1 + 2 * km2 + 2;
  if (blockIdx.x == 0 && threadIdx.x < lmx) vcl[threadIdx.x + lmx * a] = (T)vcl_type[threadIdx.x + lmx * it];
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nplw1; g += gridDim.x * blockDim.x) {
    const int k1 = ngabc[3 * g], k2 = ngabc[3 * g + 1], k3 = ngabc[3 * g + 2];
    const double c1 = cq[km1 + k1], s1 = sq[km1 + k1];
    const double c2 = cq[o2 + km2 + k2], s2 = sq[o2 + km2 + k2];
    const double c3 = cq[o3 + km3 + k3], s3 = sq[o3 + km3 + k3];
    const double c12 = c1 * c2 - s1 * s2, s12 = s1 * c2 + c1 * s2;
    const double yc = c12 * c3 - s12 * s3, ys = s12 * c3 + c12 * s3;
    for (int l = 0; l < lmx; ++l) {
      const double f = zzz[(long)(l + lmx * it) * nplw1 + g];
      double re, im;
      if (even[l + lmx * it]) { re = yc * f; im = -ys * f; }
      else { re = -ys * f; im = -yc * f; }
      const long p = l + (long)lmx * a;
      if constexpr (sizeof(T) == 8) {
        reinterpret_cast<double2 *>(kbg + p * ne)[g] = make_double2(re, im);
      } else {
        const float2 v = make_float2((float)re, (float)im);
        reinterpret_cast<float2 *>(kbg + p * ne)[g] = v;
        if (kbgp) reinterpret_cast<float2 *>(kbgp + p * ldp)[g] = v;
      }
    }
  }
}

void setqlm(int nplw1, int nchan, int lmx, int mxqlm, const double *dlqlm, const double *tbqlm, const double *qlm,
            const int *lmidx, const double *dk, double *zzz, cudaStream_t st) {
  const long tot = (long)nplw1 * nchan;
  k_setqlm<<<(unsigned)std::min<long>(148 * 8, (tot + 255) / 256), 256, 0, st>>>(nplw1, nchan, lmx, mxqlm, dlqlm,
                                                                                tbqlm, qlm, lmidx, dk, zzz);
  note_launch();
}

template <typename T>
void setbgq(int natom, int nplw1, int ne, int lmx, const int *ityp, const int *ngabc, const double *dcq,
            const double *dsq, int km1, int km2, int km3, int ktot, const double *zzz, const int *even,
            const double *vcl_type, T *kbg, float *kbgp, long ldp, T *vcl, cudaStream_t st) {
  const unsigned gx = (unsigned)std::max(1, std::min((nplw1 + 255) / 256, std::max(1, 148 * 8 / natom)));
  k_setbgq<T><<<dim3(gx, natom), 256, 0, st>>>(nplw1, ne, lmx, ityp, ngabc, dcq, dsq, km1, km2, km3, ktot, zzz,
                                              even, vcl_type, kbg, kbgp, ldp, vcl);
  note_launch();
}
template void setbgq<float>(int, int, int, int, const int *, const int *, const double *, const double *, int, int,
                            int, int, const double *, const int *, const double *, float *, float *, long, float *,
                            cudaStream_t);
template void setbgq<double>(int, int, int, int, const int *, const int *, const double *, const double *, int, int,
                             int, int, const double *, const int *, const double *, double *, float *, long,
                             double *, cudaStream_t);

}  // namespace qx
