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
//    FP32 copy) together with the per-projector KB energies;
//  * real-space tables, once per geometry (setnlc, nlkbppr.f90:1010-1560):
//    the grid points within the projector radius of each atom (the box of
//    grid points around the atom's nearest grid point, periodic wrap), in
//    box order (x fastest), with the projector values interpolated from the
//    radial table by the same three-point formula times a real solid
//    harmonic polynomial of the displacement, then the x-line index (points
//    of each grid line, ordered by point) that the real-space KB kernels of
//    the FFT pipeline read.
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
    const int m = min(2 * (int)(ag / (2.0 * dl)), mxqlm - 2);
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

// ---- real-space tables ---------------------------------------------------
__device__ __forceinline__ int kbr_wrap(int n, int k) {
  n %= k;
  return n < 0 ? n + k : n;
}

// Box point q of atom a: wrapped grid index and displacement r - R_a (bohr).
__device__ __forceinline__ void kbr_point(const KbrGeom &G, const double *s, long q, int &mesh, double &dx,
                                          double &dy, double &dz) {
  const int w1 = 2 * G.nd[0] + 1, w2 = 2 * G.nd[1] + 1;
  const int o1 = (int)(q % w1) - G.nd[0];
  const int o2 = (int)((q / w1) % w2) - G.nd[1];
  const int o3 = (int)(q / ((long)w1 * w2)) - G.nd[2];
  const int n1 = (int)floor(s[0] * G.k[0] + 0.5) + o1, n2 = (int)floor(s[1] * G.k[1] + 0.5) + o2,
            n3 = (int)floor(s[2] * G.k[2] + 0.5) + o3;
  const double f1 = (double)n1 / G.k[0] - s[0], f2 = (double)n2 / G.k[1] - s[1], f3 = (double)n3 / G.k[2] - s[2];
  dx = G.rba[0] * f1 + G.rba[1] * f2 + G.rba[2] * f3;
  dy = G.rba[3] * f1 + G.rba[4] * f2 + G.rba[5] * f3;
  dz = G.rba[6] * f1 + G.rba[7] * f2 + G.rba[8] * f3;
  mesh = kbr_wrap(n1, G.k[0]) + G.k[0] * (kbr_wrap(n2, G.k[1]) + G.k[1] * kbr_wrap(n3, G.k[2]));
}

// real solid-harmonic polynomials of degree <= 2 (normalisation in the table)
__device__ __forceinline__ double kbr_poly(int c, double x, double y, double z) {
  switch (c) {
    case 0: return 1.0;
    case 1: return x;
    case 2: return y;
    case 3: return z;
    case 4: return x * y;
    case 5: return y * z;
    case 6: return z * x;
    case 7: return x * x - y * y;
    default: return 3.0 * z * z - (x * x + y * y + z * z);
  }
}

__global__ void k_kbr_count(KbrGeom G, const int *__restrict__ ityp, const double *__restrict__ satm,
                            const double *__restrict__ rcut, int *__restrict__ cnt) {
  const int a = blockIdx.x;
  const double *s = satm + 3 * a;
  const double rc2 = rcut[ityp[a]] * rcut[ityp[a]];
  const long nbox = (long)(2 * G.nd[0] + 1) * (2 * G.nd[1] + 1) * (2 * G.nd[2] + 1);
  int c = 0;
  for (long q = threadIdx.x; q < nbox; q += blockDim.x) {
    int m;
    double dx, dy, dz;
    kbr_point(G, s, q, m, dx, dy, dz);
    c += (dx * dx + dy * dy + dz * dz <= rc2) ? 1 : 0;
  }
  __shared__ int red[32];
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    cnt[a] = t;
  }
}

// Exclusive scan of n counts by one block of 1024 threads: out[0..n],
// out[n] = total.  If cursor is given, it receives out[0..n-1] too.
__global__ void __launch_bounds__(1024) k_scan1(const int *__restrict__ in, long n, int *__restrict__ out,
                                                int *__restrict__ cursor) {
  __shared__ int part[1024];
  const int t = threadIdx.x;
  const long per = (n + 1023) / 1024, lo = std::min<long>(n, t * per), hi = std::min<long>(n, lo + per);
  int sum = 0;
  for (long i = lo; i < hi; ++i) sum += in[i];
  part[t] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - sum;
  for (long i = lo; i < hi; ++i) {
    out[i] = run;
    if (cursor) cursor[i] = run;
    run += in[i];
  }
  if (t == 1023) out[n] = part[1023];
}

// gradient of the polynomial of kbr_poly
__device__ __forceinline__ void kbr_dpoly(int c, double x, double y, double z, double &gx, double &gy, double &gz) {
  gx = gy = gz = 0.0;
  switch (c) {
    case 0: break;
    case 1: gx = 1.0; break;
    case 2: gy = 1.0; break;
    case 3: gz = 1.0; break;
    case 4: gx = y; gy = x; break;
    case 5: gy = z; gz = y; break;
    case 6: gx = z; gz = x; break;
    case 7: gx = 2.0 * x; gy = -2.0 * y; break;
    default: gx = -2.0 * x; gy = -2.0 * y; gz = 4.0 * z; break;
  }
}

__device__ __forceinline__ double kbr_interp(const double *tb, int mm, double d) {
  const double t0 = tb[mm], t1 = tb[mm + 1], t2 = tb[mm + 2];
  const double av = 2.0 * (t0 + t2 - 2.0 * t1);
  return d * ((d - 1.0) * av + t2 - t0) + t0;
}

// dvnl (optional): the gradient of each projector with respect to the point,
// grad (g(r) P(d)) = (g'(r)/r) P(d) d + g(r) grad P(d), from the table
// dtabnl of g'(r)/r; dvnl[(i * lmx + l) * 3 + dim].  rcl[l + lmx * it]: the
// radius of projector l's angular channel (rmxnlc of setnlc,
// nlkbppr.f90:1405-1431); the atom's points are those within the species
// radius rcut (the largest channel's), and a projector is zero, value and
// gradient, at the points beyond its own channel's radius, so each channel
// sums over exactly the points of its own list in setnlc.
template <typename T>
__global__ void k_kbr_fill(KbrGeom G, int lmx, const int *__restrict__ ityp, const double *__restrict__ satm,
                           const double *__restrict__ rcut, const double *__restrict__ rcl,
                           const double *__restrict__ dltnl,
                           const double *__restrict__ tabnl, const double *__restrict__ dtabnl, int mxnl,
                           const int *__restrict__ poly, const int *__restrict__ off, int natom, long cap,
                           int *__restrict__ mesh, int *__restrict__ ptatom, T *__restrict__ vnl,
                           T *__restrict__ dvnl) {
  if (off[natom] > cap) return;   // the host grows the buffers and launches again
  const int a = blockIdx.x, it = ityp[a];
  const double *s = satm + 3 * a;
  const double rc2 = rcut[it] * rcut[it], dl = dltnl[it];
  const long nbox = (long)(2 * G.nd[0] + 1) * (2 * G.nd[1] + 1) * (2 * G.nd[2] + 1);
  __shared__ int wsum[32];
  __shared__ int base;
  if (threadIdx.x == 0) base = off[a];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (long q0 = 0; q0 < nbox; q0 += blockDim.x) {
    const long q = q0 + threadIdx.x;
    int m = 0;
    double dx = 0, dy = 0, dz = 0;
    bool in = false;
    if (q < nbox) {
      kbr_point(G, s, q, m, dx, dy, dz);
      in = dx * dx + dy * dy + dz * dz <= rc2;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, in);
    if (lane == 0) wsum[warp] = __popc(bal);
    __syncthreads();
    int wo = 0, tot = 0;
    for (int w = 0; w < nw; ++w) {
      wo += w < warp ? wsum[w] : 0;
      tot += wsum[w];
    }
    const long i = base + wo + __popc(bal & ((1u << lane) - 1u));
    if (in && i < off[a + 1]) {
      mesh[i] = m;
      ptatom[i] = a;
      const double r = sqrt(dx * dx + dy * dy + dz * dz);
      const int mm = min(2 * (int)(r / (2.0 * dl)), mxnl - 2);
      const double d = 0.5 * (r / dl - (double)mm);
      const double r2 = dx * dx + dy * dy + dz * dz;
      for (int l = 0; l < lmx; ++l) {
        const int ch = l + lmx * it;
        const bool inl = r2 <= rcl[ch] * rcl[ch];
        const double f = inl ? kbr_interp(tabnl + (long)ch * (mxnl + 1), mm, d) : 0.0;
        const double pv = kbr_poly(poly[ch], dx, dy, dz);
        vnl[i * lmx + l] = (T)(f * pv);
        if (dvnl) {
          const double fd = inl ? kbr_interp(dtabnl + (long)ch * (mxnl + 1), mm, d) : 0.0;
          double gx, gy, gz;
          kbr_dpoly(poly[ch], dx, dy, dz, gx, gy, gz);
          dvnl[(i * lmx + l) * 3 + 0] = (T)(fd * pv * dx + f * gx);
          dvnl[(i * lmx + l) * 3 + 1] = (T)(fd * pv * dy + f * gy);
          dvnl[(i * lmx + l) * 3 + 2] = (T)(fd * pv * dz + f * gz);
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) base += tot;
    __syncthreads();
  }
}

__global__ void k_kbr_line_count(const int *__restrict__ off, int natom, const int *__restrict__ mesh, int k1,
                                 int *__restrict__ lcnt) {
  const long tot = off[natom];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x)
    atomicAdd(&lcnt[mesh[i] / k1], 1);
}

__global__ void k_kbr_line_fill(const int *__restrict__ off, int natom, const int *__restrict__ mesh,
                                const int *__restrict__ ptatom, int k1, int *__restrict__ cursor,
                                int4 *__restrict__ lent) {
  const long tot = off[natom];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x) {
    const int m = mesh[i];
    const int pos = atomicAdd(&cursor[m / k1], 1);
    lent[pos] = make_int4(m % k1, (int)i, ptatom[i], 0);
  }
}

// One block per line: entries ordered by point index.  Up to LSORT_MAX
// entries go to shared memory and each lands at its rank (the count of
// smaller point indices; indices are unique); a longer line is sorted by one
// thread in place (insertion sort).
constexpr int LSORT_MAX = 1024;
__global__ void __launch_bounds__(128) k_kbr_line_sort(const int *__restrict__ loff, long nlines,
                                                       int4 *__restrict__ lent) {
  __shared__ int4 e[LSORT_MAX];
  for (long l = blockIdx.x; l < nlines; l += gridDim.x) {
    const int lo = loff[l], hi = loff[l + 1], m = hi - lo;
    if (m <= 1) continue;   // uniform across the block
    if (m <= LSORT_MAX) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) e[i] = lent[lo + i];
      __syncthreads();
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int key = e[i].y;
        int r = 0;
        for (int j = 0; j < m; ++j) r += e[j].y < key ? 1 : 0;
        lent[lo + r] = e[i];
      }
      __syncthreads();
    } else if (threadIdx.x == 0) {
      for (int i = lo + 1; i < hi; ++i) {
        const int4 v = lent[i];
        int j = i - 1;
        while (j >= lo && lent[j].y > v.y) {
          lent[j + 1] = lent[j];
          --j;
        }
        lent[j + 1] = v;
      }
    }
  }
}

void kbr_count(const KbrGeom &G, int natom, const int *ityp, const double *satm, const double *rcut, int *cnt,
               int *off, cudaStream_t st) {
  k_kbr_count<<<natom, 256, 0, st>>>(G, ityp, satm, rcut, cnt);
  note_launch();
  k_scan1<<<1, 1024, 0, st>>>(cnt, natom, off, nullptr);
  note_launch();
}

template <typename T>
void kbr_fill(const KbrGeom &G, int natom, int lmx, const int *ityp, const double *satm, const double *rcut,
              const double *rcl, const double *dltnl, const double *tabnl, const double *dtabnl, int mxnl,
              const int *poly, const int *off, long cap, int *mesh, int *ptatom, T *vnl, T *dvnl, cudaStream_t st) {
  k_kbr_fill<T><<<natom, 256, 0, st>>>(G, lmx, ityp, satm, rcut, rcl, dltnl, tabnl, dtabnl, mxnl, poly, off, natom,
                                       cap, mesh, ptatom, vnl, dtabnl ? dvnl : nullptr);
  note_launch();
}
template void kbr_fill<float>(const KbrGeom &, int, int, const int *, const double *, const double *, const double *,
                              const double *, const double *, const double *, int, const int *, const int *, long,
                              int *, int *, float *, float *, cudaStream_t);
template void kbr_fill<double>(const KbrGeom &, int, int, const int *, const double *, const double *, const double *,
                               const double *, const double *, const double *, int, const int *, const int *, long,
                               int *, int *, double *, double *, cudaStream_t);

int kbr_lines(const int *off, int natom, const int *mesh, const int *ptatom, int k1, long nlines, int *lcnt,
              int *loff, int *cursor, int4 *lent, cudaStream_t st) {
  if (cudaMemsetAsync(lcnt, 0, sizeof(int) * nlines, st) != cudaSuccess) return 1;
  k_kbr_line_count<<<148 * 4, 256, 0, st>>>(off, natom, mesh, k1, lcnt);
  note_launch();
  k_scan1<<<1, 1024, 0, st>>>(lcnt, nlines, loff, cursor);
  note_launch();
  k_kbr_line_fill<<<148 * 4, 256, 0, st>>>(off, natom, mesh, ptatom, k1, cursor, lent);
  note_launch();
  k_kbr_line_sort<<<(unsigned)std::min<long>(148 * 16, nlines), 128, 0, st>>>(loff, nlines, lent);
  note_launch();
  return 0;
}

}  // namespace qx
