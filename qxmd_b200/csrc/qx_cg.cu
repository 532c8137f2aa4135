// Batched BKL conjugate-gradient band update (eigen_BKL, eigen.f90:199-938,
// preconditioner prpcg eigen.f90:1093-1113, subgs4 engrad.f90:1196-1248).
// All bands iterate together; band ib is projected against the entry
// snapshot of bands < ib (subgs3, done as two GEMMs by the caller), which is
// the reference's result with one band per rank.  One CTA per band; every
// reduction is accumulated in FP64.  Per-band state lives on the device, so a
// CG sweep needs no host round trip.
#include "qx_internal.h"
#include "qx_cg.h"

namespace qx {

// One CTA per band; 1024 threads give each SM enough loads in flight for
// these bandwidth-bound sweeps over a band.
constexpr int CGT = 1024;

template <typename T>
__device__ __forceinline__ double ld(const T *p, long i) { return (double)p[i]; }

// Gamma-point inner product of two bands, block-wide.
template <typename T>
__device__ double bdot(const T *x, const T *y, int ne, double *red) {
  double s = 0.0;
  for (int i = threadIdx.x; i < ne; i += blockDim.x) s += ld(x, i) * ld(y, i);
  s = block_sum(s, red);
  return 2.0 * s - ld(x, 0) * ld(y, 0);
}

template <typename T>
__global__ void __launch_bounds__(CGT) k_cg_init(int ne, long ldx, const T *__restrict__ x,
                                                         const T *__restrict__ hx, T *__restrict__ g, CgState s) {
  __shared__ double red[CGT / 32];
  const int b = blockIdx.x;
  const T *xb = x + b * ldx, *hb = hx + b * ldx;
  T *gb = g + b * ldx;
  const double e = bdot(xb, hb, ne, red);
  double z = 0.0;
  for (int i = threadIdx.x; i < ne; i += blockDim.x) {
    const T v = (T)e * xb[i] - hb[i];
    gb[i] = v;
    z += (double)v * (double)v;
  }
  z = block_sum(z, red);
  z = 2.0 * z - ld(gb, 0) * ld(gb, 0);
  if (threadIdx.x == 0) {
    s.eig[b] = e;
    s.zansa[b] = z;
    s.zansab[b] = z;
    s.z000re[b] = z;
    s.x000re[b] = 1.0e10;
    s.eigb[b] = e;
    s.dinnerx[b] = 0.0;
    s.betk[b] = 0.0;
    s.izcnt[b] = 0;
    s.lreset[b] = 1;
    s.iter[b] = 0;
    s.active[b] = 1;
  }
}

// g <- prcd * g; zansap = <g|g>; h <- g + beta*h (h <- g on reset).
template <typename T>
__global__ void __launch_bounds__(CGT) k_cg_prec(int ne, long ldx, T *__restrict__ g, T *__restrict__ h,
                                                         const double *__restrict__ dk, CgState s,
                                                         const int *__restrict__ cur, int nb) {
  __shared__ double red[CGT / 32];
  const int b = cur ? *cur : blockIdx.x;
  if (b >= nb || !s.active[b]) return;
  T *gb = g + b * ldx, *hb = h + b * ldx;
  const double e15 = 1.5 * s.ekib[b];
  double z = 0.0;
  for (int i = threadIdx.x; i < ne; i += blockDim.x) {
    const double x = dk[i] / e15;
    double t = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x));
    const double x2 = x * x, x4 = x2 * x2;
    t = t / (t + 16.0 * x4);
    const T v = (T)((double)gb[i] * (t * 2.0 / e15));
    gb[i] = v;
    z += (double)v * (double)v;
  }
  z = block_sum(z, red);
  const double zansap = 2.0 * z - ld(gb, 0) * ld(gb, 0);
  const int reset = s.lreset[b];
  const double beta = reset ? 0.0 : zansap / s.betk[b];
  for (int i = threadIdx.x; i < ne; i += blockDim.x) {
    const T hv = reset ? (T)0 : hb[i];
    hb[i] = gb[i] + (T)beta * hv;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s.lreset[b] = 0;
    s.betk[b] = zansap;
    s.iter[b] += 1;
  }
}

// Mask for subgs3: M(j,i) = P(j,i) if j < i and band i is active, else 0.
template <typename T>
__global__ void k_cg_mask(int nb, T *__restrict__ Pm, CgState s) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= (long)nb * nb) return;
  const int i = (int)(e / nb), j = (int)(e - (long)i * nb);
  if (!(j < i && s.active[i])) Pm[e] = (T)0;
}

// subgs4: h -= <x|h> x; cai = <h|hx>.
template <typename T>
__global__ void __launch_bounds__(CGT) k_cg_orth(int ne, long ldx, const T *__restrict__ x,
                                                         const T *__restrict__ hx, T *__restrict__ h, CgState s,
                                                         const int *__restrict__ cur, int nb) {
  __shared__ double red[CGT / 32];
  const int b = cur ? *cur : blockIdx.x;
  if (b >= nb || !s.active[b]) return;
  const T *xb = x + b * ldx, *hxb = hx + b * ldx;
  T *hb = h + b * ldx;
  const double hhx = bdot(xb, (const T *)hb, ne, red);
  double c = 0.0;
  for (int i = threadIdx.x; i < ne; i += blockDim.x) {
    const T v = hb[i] - (T)hhx * xb[i];
    hb[i] = v;
    c += (double)v * (double)hxb[i];
  }
  c = block_sum(c, red);
  if (threadIdx.x == 0) s.cai[b] = 2.0 * c - ld(hb, 0) * ld(hxb, 0);
}

// Active-band list and the band pairs of the FFT pipeline: one warp compacts
// 32 bands per round with a ballot and a population-count prefix.
__global__ void k_cg_list(int nb, CgState s) {
  const int lane = threadIdx.x & 31;
  int n = 0;
  for (int b0 = 0; b0 < nb; b0 += 32) {
    const int b = b0 + lane;
    const bool act = (b < nb) && s.active[b];
    const unsigned m = __ballot_sync(0xffffffffu, act);
    if (act) s.list[n + __popc(m & ((1u << lane) - 1u))] = b;
    n += __popc(m);
  }
  __syncwarp();
  for (int p = lane; p < (n + 1) / 2; p += 32) {
    s.pairs[2 * p] = s.list[2 * p];
    s.pairs[2 * p + 1] = (2 * p + 1 < n) ? s.list[2 * p + 1] : -1;
  }
  if (lane == 0) {
    *s.nact = n;
    *s.npair = (n + 1) / 2;
  }
}

// BKL 2x2 step (eigen.f90:593-622), line minimisation fallback (624-695),
// x/hx update (698-709), residual and convergence test (731-764).
// SEQ: one CTA on band *q.cur; when the band stops, its final vector becomes
// its snapshot column (cgjr(:,ib) = gdcr(:,ibb), eigen.f90:699, real*4 when
// q.ccreal4) and the next band starts.
// All bands at once: two CTAs per SM (at most 32 registers), so that 160
// bands fit one wave on 148 SMs.
template <typename T, bool SEQ>
__global__ void __launch_bounds__(CGT, SEQ ? 1 : 2) k_cg_update(int ne, long ldx, T *__restrict__ x, T *__restrict__ hx,
                                                           T *__restrict__ g, const T *__restrict__ h,
                                                           const T *__restrict__ gh, CgState s, CgParm pm,
                                                           SeqArgs q) {
  __shared__ double red[CGT / 32];
  __shared__ int stop_sh;
  const int b = SEQ ? *q.cur : blockIdx.x;
  if (SEQ && b >= q.nb) {
    if (threadIdx.x == 0) cudaGraphSetConditional(q.handle, 0);
    return;
  }
  if (!SEQ && !s.active[b]) return;
  T *xb = x + b * ldx, *hxb = hx + b * ldx, *gb = g + b * ldx;
  const T *hb = h + b * ldx, *ghb = gh + b * ldx;
  const double dinx = s.dinnerx[b];   // read before thread 0 may update it
  double cb = 0.0, hh = 0.0;
  for (int i = threadIdx.x; i < ne; i += blockDim.x) {
    const double hv = (double)hb[i];
    cb += hv * (double)ghb[i];
    hh += hv * hv;
  }
  cb = block_sum(cb, red);
  hh = block_sum(hh, red);
  const double h0 = ld(hb, 0);
  const double cbi = 2.0 * cb - h0 * ld(ghb, 0);
  const double hhi = 2.0 * hh - h0 * h0;
  const double cai = s.cai[b];
  double e = s.eig[b];
  double dtnew, alpsq;
  if (hhi > 0.0) {
    const double h11 = e, h12 = cai / sqrt(hhi), h21 = h12, h22 = cbi / hhi;
    const double enew = 0.5 * (h11 + h22 - sqrt((h11 + h22) * (h11 + h22) - 4.0 * (h11 * h22 - h12 * h21)));
    dtnew = (enew - h11) / h12 / sqrt(hhi);
    const double alpsq2 = 1.0 / (1.0 + dtnew * (0.0 + dtnew * hhi));
    alpsq = sqrt(alpsq2);
    e = enew;
  } else {
    double hx2 = 0.0;
    for (int i = threadIdx.x; i < ne; i += blockDim.x) hx2 += (double)hb[i] * (double)xb[i];
    hx2 = block_sum(hx2, red);
    const double hhx = 2.0 * hx2 - h0 * ld(xb, 0);
    const double c0 = e, c1 = cai, c2 = cbi, c3 = hhi, c4 = 2.0 * hhx;
    const double s0 = c0 * c4 - c1, s1 = c0 * c3 - c2, s2 = c1 * c3 - c2 * c4;
    const double sr = s1 * s1 - s2 * s0;
    dtnew = (sr > 0.0) ? (-s1 - sqrt(sr)) / s2 : -1.0;
    if (dtnew > 0.0) {
      const double dinner = sqrt(1.0 / (1.0 + dtnew * dtnew * hhi));
      if (dinner < pm.threinn) dtnew = 0.0;
      if (dinner < dinx * pm.wdinner) dtnew = 0.0;
      if (threadIdx.x == 0 && dinner > dinx) s.dinnerx[b] = dinner;
    }
    const double d2 = dtnew * dtnew;
    const double alpsq2 = 1.0 / (1.0 + dtnew * c4 + d2 * c3);
    e = (c0 + dtnew * c1 + d2 * c2) * alpsq2;
    alpsq = sqrt(alpsq2);
  }
  const T a = (T)alpsq, dt = (T)dtnew, et = (T)e;
  double z = 0.0;
  for (int i = threadIdx.x; i < ne; i += blockDim.x) {
    const T xn = a * (xb[i] + dt * hb[i]);
    const T hn = a * (hxb[i] + dt * ghb[i]);
    xb[i] = xn;
    hxb[i] = hn;
    const T gv = et * xn - hn;
    gb[i] = gv;
    z += (double)gv * (double)gv;
  }
  z = block_sum(z, red);
  const double zansa = 2.0 * z - ld(gb, 0) * ld(gb, 0);
  if (threadIdx.x == 0) {
    const int iter = s.iter[b];
    const double eigb = s.eigb[b];
    const double de = fabs(eigb - e);
    const int stop = (b < pm.noband && iter >= pm.itermx) || (b >= pm.noband && iter >= pm.iteremx) ||
                     zansa < pm.tolera || de < pm.tolera || zansa < s.z000re[b] * pm.roughfzan ||
                     (iter > 1 && de < s.x000re[b] * pm.roughfeig);
    s.eig[b] = e;
    s.zansa[b] = zansa;
    if (stop) {
      s.active[b] = 0;
    } else {
      if (iter == 1) s.x000re[b] = de;
      if (zansa > s.zansab[b]) {
        if (++s.izcnt[b] > 20) { s.izcnt[b] = 0; s.lreset[b] = 1; }
      }
      s.zansab[b] = zansa;
      s.eigb[b] = e;
    }
    stop_sh = stop;
  }
  if constexpr (SEQ) {
    __syncthreads();
    if (stop_sh) {
      // each thread reads back the elements of x it wrote above
      T *sb = (T *)q.snap + b * ldx;
      for (int i = threadIdx.x; i < ne; i += blockDim.x) {
        const T v = xb[i];
        sb[i] = q.ccreal4 ? (T)(float)v : v;
      }
      if (threadIdx.x == 0) {
        const int nx = b + 1;
        *q.cur = nx;
        q.pairs[0] = nx;
        q.pairs[1] = -1;
        q.list[0] = nx;
        if (nx >= q.nb) cudaGraphSetConditional(q.handle, 0);
      }
    }
  }
}

__global__ void k_seq_reset(SeqArgs q) {
  *q.cur = 0;
  q.pairs[0] = 0;
  q.pairs[1] = -1;
  q.list[0] = 0;
}

// Band-space dot products against band *cur: one CTA per vector j.
template <typename T>
__global__ void __launch_bounds__(256) k_seq_dots(int nmax, const int *__restrict__ n_dev, int ne,
                                                  const T *__restrict__ V, long ldv, const T *__restrict__ Y, long ldy,
                                                  const int *__restrict__ cur, int gamma, const T *__restrict__ scale,
                                                  double *__restrict__ out) {
  __shared__ double red[8];
  const int j = blockIdx.x;
  const int n = n_dev ? min(nmax, *n_dev) : nmax;
  if (j >= n) return;
  const T *v = V + j * ldv, *y = Y + (long)*cur * ldy;
  double sum = 0.0;
  for (int i = threadIdx.x; i < ne; i += blockDim.x) sum += (double)v[i] * (double)y[i];
  sum = block_sum(sum, red);
  if (threadIdx.x == 0) {
    double r = 2.0 * sum - (double)v[0] * (double)y[0];
    if (gamma == 2) r -= 2.0 * (double)v[1] * (double)y[1];
    if (scale) r *= (double)scale[j];
    out[j] = r;
  }
}

// Y_cur[i] += sign * sum_j coef[j] V_j[i]: a CTA owns 32 consecutive rows (one
// per lane); warp w takes j = w, w+8, ..., and the eight partial sums are added
// in a fixed order.
template <typename T>
__global__ void __launch_bounds__(256) k_seq_axpy(int nmax, const int *__restrict__ n_dev, int ne,
                                                  const T *__restrict__ V, long ldv, const double *__restrict__ coef,
                                                  double sign, T *__restrict__ Y, long ldy,
                                                  const int *__restrict__ cur) {
  __shared__ double part[8][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = blockIdx.x * 32 + lane;
  const int n = n_dev ? min(nmax, *n_dev) : nmax;
  double acc = 0.0;
  if (i < ne) {
    int j = w;
    for (; j + 24 < n; j += 32) {
      const T a0 = V[(long)j * ldv + i], a1 = V[(long)(j + 8) * ldv + i];
      const T a2 = V[(long)(j + 16) * ldv + i], a3 = V[(long)(j + 24) * ldv + i];
      acc += coef[j] * (double)a0;
      acc += coef[j + 8] * (double)a1;
      acc += coef[j + 16] * (double)a2;
      acc += coef[j + 24] * (double)a3;
    }
    for (; j < n; j += 8) acc += coef[j] * (double)V[(long)j * ldv + i];
  }
  part[w][lane] = acc;
  __syncthreads();
  if (w == 0 && i < ne) {
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) t += part[q][lane];
    T *y = Y + (long)*cur * ldy;
    y[i] = (T)((double)y[i] + sign * t);
  }
}

// ekinetic2 (engrad.f90:75-127): ekib(b) = 2*<c|T|c>, and sum occ*<c|T|c>
// into *ekin (one CTA per band writes its term; summed by k_sum_occ).
template <typename T>
__global__ void __launch_bounds__(CGT) k_ekin(int ne, long ldx, const T *__restrict__ x,
                                                      const double *__restrict__ dk, double *__restrict__ ekib) {
  __shared__ double red[CGT / 32];
  const int b = blockIdx.x;
  const T *xb = x + b * ldx;
  double s = 0.0;
  for (int i = threadIdx.x; i < ne; i += blockDim.x) s += dk[i] * ld(xb, i) * ld(xb, i);
  s = block_sum(s, red);
  if (threadIdx.x == 0) ekib[b] = 2.0 * (2.0 * s - dk[0] * ld(xb, 0) * ld(xb, 0));
}

// gradresnv (engrad.f90:1013-1067): per-band |eig*c - hc|^2 (Gamma metric).
template <typename T>
__global__ void __launch_bounds__(CGT) k_gradres(int ne, long ldx, const T *__restrict__ x,
                                                         const T *__restrict__ hx, const double *__restrict__ eig,
                                                         double *__restrict__ prod) {
  __shared__ double red[CGT / 32];
  const int b = blockIdx.x;
  const T *xb = x + b * ldx, *hb = hx + b * ldx;
  const double e = eig[b];
  double s = 0.0;
  for (int i = threadIdx.x; i < ne; i += blockDim.x) {
    const double r = e * ld(xb, i) - ld(hb, i);
    s += r * r;
  }
  s = block_sum(s, red);
  const double r0 = e * ld(xb, 0) - ld(hb, 0);
  if (threadIdx.x == 0) prod[b] = 2.0 * s - r0 * r0;
}

// Device-side summaries for a sync-free SCF iteration: out[0] = max_b prod,
// out[1] = sum_b occ_b prod_b (gradresnv's zmax and occupation-weighted sum).
__global__ void k_gradres_stats(const double *__restrict__ prod, const double *__restrict__ occ, int nb,
                                double *__restrict__ out) {
  const int lane = threadIdx.x;
  double m = 0.0, s = 0.0;
  for (int b = lane; b < nb; b += 32) {
    m = fmax(m, prod[b]);
    if (occ) s += occ[b] * prod[b];
  }
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    s += __shfl_xor_sync(0xffffffffu, s, o);
  }
  if (lane == 0) { out[0] = m; out[1] = s; }
}

// *out = sum of the per-band CG iteration counts (H|psi> band applications).
__global__ void k_iter_sum(const int *__restrict__ iter, int nb, int *__restrict__ out) {
  const int lane = threadIdx.x;
  int s = 0;
  for (int b = lane; b < nb; b += 32) s += iter[b];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) *out = s;
}

// Row scaling of the projection matrix P (nproj x ncol, column-major, columns
// through colmap): P(j, n) *= v(j).
template <typename T>
__global__ void k_scale_rows(int nproj, int ncol, T *__restrict__ P, long ldp, const T *__restrict__ v,
                             const int *__restrict__ colmap, const int *__restrict__ ncol_dev) {
  const int nc = ncol_dev ? min(ncol, *ncol_dev) : ncol;
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= (long)nproj * nc) return;
  const int n = (int)(e / nproj), j = (int)(e - (long)n * nproj);
  const long cn = colmap ? colmap[n] : n;
  P[cn * ldp + j] *= v[j];
}

// ---- launchers -------------------------------------------------------------
template <typename T> void cg_init(int nb, int ne, long ldx, const T *x, const T *hx, T *g, const CgState &s, cudaStream_t st) {
  k_cg_init<T><<<nb, CGT, 0, st>>>(ne, ldx, x, hx, g, s); note_launch();
}
template <typename T> void cg_prec(int nb, int ne, long ldx, T *g, T *h, const double *dk, const CgState &s, cudaStream_t st,
                                   const int *cur) {
  k_cg_prec<T><<<cur ? 1 : nb, CGT, 0, st>>>(ne, ldx, g, h, dk, s, cur, nb); note_launch();
}
template <typename T> void cg_mask(int nb, T *Pm, const CgState &s, cudaStream_t st) {
  const long nn = (long)nb * nb;
  k_cg_mask<T><<<(int)((nn + 255) / 256), 256, 0, st>>>(nb, Pm, s); note_launch();
}
template <typename T> void cg_orth(int nb, int ne, long ldx, const T *x, const T *hx, T *h, const CgState &s, cudaStream_t st,
                                   const int *cur) {
  k_cg_orth<T><<<cur ? 1 : nb, CGT, 0, st>>>(ne, ldx, x, hx, h, s, cur, nb); note_launch();
}
void cg_list(int nb, const CgState &s, cudaStream_t st) { k_cg_list<<<1, 32, 0, st>>>(nb, s); note_launch(); }
void gradres_stats(const double *prod, const double *occ, int nb, double *out, cudaStream_t st) {
  k_gradres_stats<<<1, 32, 0, st>>>(prod, occ, nb, out); note_launch();
}
void iter_sum(const int *iter, int nb, int *out, cudaStream_t st) { k_iter_sum<<<1, 32, 0, st>>>(iter, nb, out); note_launch(); }
template <typename T> void cg_update(int nb, int ne, long ldx, T *x, T *hx, T *g, const T *h, const T *gh,
                                     const CgState &s, const CgParm &pm, cudaStream_t st) {
  k_cg_update<T, false><<<nb, CGT, 0, st>>>(ne, ldx, x, hx, g, h, gh, s, pm, SeqArgs{}); note_launch();
}
template <typename T> void cg_update_seq(int ne, long ldx, T *x, T *hx, T *g, const T *h, const T *gh, const CgState &s,
                                         const CgParm &pm, const SeqArgs &q, cudaStream_t st) {
  k_cg_update<T, true><<<1, CGT, 0, st>>>(ne, ldx, x, hx, g, h, gh, s, pm, q); note_launch();
}
void seq_reset(const SeqArgs &q, cudaStream_t st) { k_seq_reset<<<1, 1, 0, st>>>(q); note_launch(); }
template <typename T> void seq_dots(int nmax, const int *n_dev, int ne, const T *V, long ldv, const T *Y, long ldy,
                                    const int *cur, int gamma, const T *scale, double *out, cudaStream_t st) {
  if (nmax <= 0) return;
  k_seq_dots<T><<<nmax, 256, 0, st>>>(nmax, n_dev, ne, V, ldv, Y, ldy, cur, gamma, scale, out); note_launch();
}
template <typename T> void seq_axpy(int nmax, const int *n_dev, int ne, const T *V, long ldv, const double *coef,
                                    double sign, T *Y, long ldy, const int *cur, cudaStream_t st) {
  k_seq_axpy<T><<<(ne + 31) / 32, 256, 0, st>>>(nmax, n_dev, ne, V, ldv, coef, sign, Y, ldy, cur); note_launch();
}
template <typename T> void ekin(int nb, int ne, long ldx, const T *x, const double *dk, double *ekib, cudaStream_t st) {
  k_ekin<T><<<nb, CGT, 0, st>>>(ne, ldx, x, dk, ekib); note_launch();
}
template <typename T> void gradres(int nb, int ne, long ldx, const T *x, const T *hx, const double *eig, double *prod,
                                   cudaStream_t st) {
  k_gradres<T><<<nb, CGT, 0, st>>>(ne, ldx, x, hx, eig, prod); note_launch();
}
template <typename T> void scale_rows(int nproj, int ncol, T *P, long ldp, const T *v, const int *colmap,
                                      const int *ncol_dev, cudaStream_t st) {
  const long n = (long)nproj * ncol;
  k_scale_rows<T><<<(int)((n + 255) / 256), 256, 0, st>>>(nproj, ncol, P, ldp, v, colmap, ncol_dev); note_launch();
}

#define QX_INST(T)                                                                                          \
  template void cg_init<T>(int, int, long, const T *, const T *, T *, const CgState &, cudaStream_t);        \
  template void cg_prec<T>(int, int, long, T *, T *, const double *, const CgState &, cudaStream_t,          \
                           const int *);                                                                    \
  template void cg_mask<T>(int, T *, const CgState &, cudaStream_t);                                         \
  template void cg_orth<T>(int, int, long, const T *, const T *, T *, const CgState &, cudaStream_t,         \
                           const int *);                                                                    \
  template void cg_update_seq<T>(int, long, T *, T *, T *, const T *, const T *, const CgState &,            \
                                 const CgParm &, const SeqArgs &, cudaStream_t);                            \
  template void seq_dots<T>(int, const int *, int, const T *, long, const T *, long, const int *, int,      \
                            const T *, double *, cudaStream_t);                                             \
  template void seq_axpy<T>(int, const int *, int, const T *, long, const double *, double, T *, long,      \
                            const int *, cudaStream_t);                                                     \
  template void cg_update<T>(int, int, long, T *, T *, T *, const T *, const T *, const CgState &,            \
                             const CgParm &, cudaStream_t);                                                  \
  template void ekin<T>(int, int, long, const T *, const double *, double *, cudaStream_t);                  \
  template void gradres<T>(int, int, long, const T *, const T *, const double *, double *, cudaStream_t);    \
  template void scale_rows<T>(int, int, T *, long, const T *, const int *, const int *, cudaStream_t);
QX_INST(float)
QX_INST(double)

}  // namespace qx
