// Batched, sphere-pruned 3D FFT pipeline for the Gamma-point H|psi> product.
//
// Replaces wvg2r (engrad.f90:1492-1559), the V_loc multiply and real-space KB
// add of hcnonloc (engrad.f90:484-530), rfft3 (fft3.f90:113-232), the gather
// at ijkgd (engrad.f90:564-571) and the kinetic term (eigen.f90:335,516).
//
// Two real bands A, B share one complex transform: Z(G) = cA(G) + i cB(G).
// Grid index n1 + (n2 + n3*k2)*k1.  The wavefunction sphere spans
// |n1| <= m1, |n2| <= m2 (compact indices a = n1 + m1 < P1, j2 = n2 + m2 < P2),
// so the pipeline keeps only what is non-zero between passes:
//   zinv : gather sphere -> z-FFT backward, per grid row j2   -> bufA[p][i3][j2][a]
//   y<+1>: y-FFT backward per (p, i3) plane                   -> bufB[p][i3][i2][a]
//   xvx  : x-FFT backward, * V(r), x-FFT forward per line     -> bufB (in place)
//   y<-1>: y-FFT forward                                      -> bufA rows j2
//   zfwd : z-FFT forward, 1/N, pick +G and -G                 -> zsph[p][ig][2]
//   unpack: split the two bands, add kinetic, write H|psi>
// Real-space KB (calnlc, nlkbppr.f90:1773-1900) splits xvx into xinv_r,
// nlproj and xfwd_r.  Density (softchg, chgdns.f90:388-454) uses zinv, y<+1>
// and xrho.
#include <algorithm>
#include <cmath>
#include <cstdlib>

#include <mutex>

#include "qx_internal.h"

// --------------------------------------------------------------------------
// Small DFTs in registers.  Roots of unity w_R^m = exp(-2 pi i m / R) for
// R = 2..9 live in constant memory (row R, column m), written once per
// device by init_fft_roots().  SIGN = -1 forward, +1 backward (conjugate roots).
__constant__ float2 c_root32[10 * 16];
__constant__ double2 c_root64[10 * 16];

template <typename T> __device__ __forceinline__ typename c2t<T>::type root(int R, int m);
template <> __device__ __forceinline__ float2 root<float>(int R, int m) { return c_root32[R * 16 + m]; }
template <> __device__ __forceinline__ double2 root<double>(int R, int m) { return c_root64[R * 16 + m]; }

template <typename T, int SIGN>
__device__ __forceinline__ typename c2t<T>::type rootS(int R, int m) {
  typename c2t<T>::type w = root<T>(R, m);
  if (SIGN > 0) w.y = -w.y;
  return w;
}

// multiply by SIGN * i
template <int SIGN, typename C> __device__ __forceinline__ C mul_si(C d) {
  C r;
  if (SIGN < 0) { r.x = d.y; r.y = -d.x; } else { r.x = -d.y; r.y = d.x; }
  return r;
}

template <typename T, int SIGN, int R>
struct Dft;

template <typename T, int SIGN> struct Dft<T, SIGN, 1> {
  typedef typename c2t<T>::type C;
  static __device__ __forceinline__ void run(const C *v, int sv, C *o, int so) { o[0] = v[0]; }
};
template <typename T, int SIGN> struct Dft<T, SIGN, 2> {
  typedef typename c2t<T>::type C;
  static __device__ __forceinline__ void run(const C *v, int sv, C *o, int so) {
    const C a = v[0], b = v[sv];
    o[0] = cadd(a, b);
    o[so] = csub(a, b);
  }
};
template <typename T, int SIGN> struct Dft<T, SIGN, 3> {
  typedef typename c2t<T>::type C;
  static __device__ __forceinline__ void run(const C *v, int sv, C *o, int so) {
    const T hs = (T)0.86602540378443864676;   // sqrt(3)/2
    const C v0 = v[0], t1 = cadd(v[sv], v[2 * sv]), d = csub(v[sv], v[2 * sv]);
    C t2;
    t2.x = v0.x - (T)0.5 * t1.x;
    t2.y = v0.y - (T)0.5 * t1.y;
    C hd; hd.x = hs * d.x; hd.y = hs * d.y;
    const C jd = mul_si<SIGN>(hd);
    o[0] = cadd(v0, t1);
    o[so] = cadd(t2, jd);
    o[2 * so] = csub(t2, jd);
  }
};
template <typename T, int SIGN> struct Dft<T, SIGN, 4> {
  typedef typename c2t<T>::type C;
  static __device__ __forceinline__ void run(const C *v, int sv, C *o, int so) {
    const C s0 = cadd(v[0], v[2 * sv]), d0 = csub(v[0], v[2 * sv]);
    const C s1 = cadd(v[sv], v[3 * sv]), d1 = csub(v[sv], v[3 * sv]);
    const C jd1 = mul_si<SIGN>(d1);
    o[0] = cadd(s0, s1);
    o[2 * so] = csub(s0, s1);
    o[so] = cadd(d0, jd1);
    o[3 * so] = csub(d0, jd1);
  }
};
// Direct DFT for the prime radices 5 and 7.
template <typename T, int SIGN, int R> struct DftDirect {
  typedef typename c2t<T>::type C;
  static __device__ __forceinline__ void run(const C *v, int sv, C *o, int so) {
    C x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = v[r * sv];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      C acc = x[0];
#pragma unroll
      for (int r = 1; r < R; ++r) acc = cadd(acc, cmul(x[r], rootS<T, SIGN>(R, (r * q) % R)));
      o[q * so] = acc;
    }
  }
};
template <typename T, int SIGN> struct Dft<T, SIGN, 5> : DftDirect<T, SIGN, 5> {};
template <typename T, int SIGN> struct Dft<T, SIGN, 7> : DftDirect<T, SIGN, 7> {};
// Two-factor radices R = P*Q: input r = a + P*c, output k = k1 + Q*k2:
// X[k1 + Q k2] = sum_a w_R^{a k1} w_P^{a k2} sum_c v[a + P c] w_Q^{c k1}.
template <typename T, int SIGN, int P, int Q> struct DftPQ {
  typedef typename c2t<T>::type C;
  static __device__ __forceinline__ void run(const C *v, int sv, C *o, int so) {
    C t[P * Q];
#pragma unroll
    for (int a = 0; a < P; ++a) Dft<T, SIGN, Q>::run(v + a * sv, P * sv, t + a * Q, 1);
#pragma unroll
    for (int a = 1; a < P; ++a)
#pragma unroll
      for (int k1 = 1; k1 < Q; ++k1) t[a * Q + k1] = cmul(t[a * Q + k1], rootS<T, SIGN>(P * Q, a * k1));
#pragma unroll
    for (int k1 = 0; k1 < Q; ++k1) Dft<T, SIGN, P>::run(t + k1, Q, o + k1 * so, Q * so);
  }
};
template <typename T, int SIGN> struct Dft<T, SIGN, 6> : DftPQ<T, SIGN, 2, 3> {};
template <typename T, int SIGN> struct Dft<T, SIGN, 8> : DftPQ<T, SIGN, 2, 4> {};
template <typename T, int SIGN> struct Dft<T, SIGN, 9> : DftPQ<T, SIGN, 3, 3> {};

// One Stockham stage of radix R over `nl` lines (element-major layout).
template <typename T, int SIGN, int R>
__device__ __forceinline__ void fft_stage(const typename c2t<T>::type *a, typename c2t<T>::type *b, int nr, int ns,
                                          int ld, int l, int j0, int jstep, const typename c2t<T>::type *st,
                                          const int *ob) {
  typedef typename c2t<T>::type C;
  for (int j = j0; j < nr; j += jstep) {
    C v[R], o[R];
    v[0] = a[j * ld + l];
#pragma unroll
    for (int r = 1; r < R; ++r) {
      C t = st[j * (R - 1) + r - 1];
      if (SIGN > 0) t.y = -t.y;
      v[r] = cmul(a[(j + r * nr) * ld + l], t);
    }
    Dft<T, SIGN, R>::run(v, 1, o, 1);
    const int base = ob[j];
#pragma unroll
    for (int q = 0; q < R; ++q) b[(base + q * ns) * ld + l] = o[q];
  }
}

// Batched in-shared-memory Stockham FFT (decimation in time, natural order
// in and out).  `nl` lines of length L.n, element-major: element e of line l
// at buf[e * ld + l].  Ping-pongs between buf and tmp; returns the buffer
// holding the result.  SIGN = -1 forward, +1 backward (unscaled).  stw/sob:
// the stage tables in shared memory.  Thread t works on line t % nl (needs
// nl <= blockDim.x).  Called by all threads; ends with a __syncthreads.
template <typename T, int SIGN>
__device__ typename c2t<T>::type *smem_fft(typename c2t<T>::type *buf, typename c2t<T>::type *tmp, int nl, int ld,
                                           const FftLen &L, const typename c2t<T>::type *tw,
                                           const typename c2t<T>::type *stw, const int *sob) {
  typedef typename c2t<T>::type C;
  (void)tw;
  const int n = L.n;
  const int l = threadIdx.x % nl;
  const int j0 = threadIdx.x / nl;
  const int jstep = blockDim.x / nl;
  const bool act = threadIdx.x < jstep * nl;
  int ns = 1;
  C *a = buf, *b = tmp;
  for (int s = 0; s < L.nstage; ++s) {
    const int R = L.radix[s];
    const int nr = n / R;
    const C *st = stw + L.st_off[s];
    const int *ob = sob + L.ob_off[s];
    if (act) {
      switch (R) {
        case 2: fft_stage<T, SIGN, 2>(a, b, nr, ns, ld, l, j0, jstep, st, ob); break;
        case 3: fft_stage<T, SIGN, 3>(a, b, nr, ns, ld, l, j0, jstep, st, ob); break;
        case 4: fft_stage<T, SIGN, 4>(a, b, nr, ns, ld, l, j0, jstep, st, ob); break;
        case 5: fft_stage<T, SIGN, 5>(a, b, nr, ns, ld, l, j0, jstep, st, ob); break;
        case 6: fft_stage<T, SIGN, 6>(a, b, nr, ns, ld, l, j0, jstep, st, ob); break;
        case 7: fft_stage<T, SIGN, 7>(a, b, nr, ns, ld, l, j0, jstep, st, ob); break;
        case 8: fft_stage<T, SIGN, 8>(a, b, nr, ns, ld, l, j0, jstep, st, ob); break;
        default: fft_stage<T, SIGN, 9>(a, b, nr, ns, ld, l, j0, jstep, st, ob); break;
      }
    }
    __syncthreads();
    C *t = a; a = b; b = t;
    ns *= R;
  }
  return a;
}

__device__ __forceinline__ int pair_count(const PipeParams &P) {
  return P.npair_dev ? *P.npair_dev : P.npair;
}

// Device copies of one length's FFT tables (see FftLen).
template <typename T>
struct FftTabs {
  const typename c2t<T>::type *tw, *stw;
  const int *sob;
};

// Shared-memory layout of a kernel: [tw | stw | sob | pad] then the tiles.
template <typename T>
struct SmTabs {
  typename c2t<T>::type *tw, *stw;
  int *sob;
  typename c2t<T>::type *tiles;
};

__host__ __device__ __forceinline__ size_t tab_bytes(const FftLen &L, size_t cs) {
  size_t b = (size_t)(L.n + L.nst) * cs + (size_t)L.nob * 4;
  return (b + 15) & ~(size_t)15;
}

template <typename T>
__device__ __forceinline__ SmTabs<T> load_tabs(unsigned char *sm, const FftLen &L, const FftTabs<T> &g) {
  typedef typename c2t<T>::type C;
  SmTabs<T> t;
  t.tw = reinterpret_cast<C *>(sm);
  t.stw = t.tw + L.n;
  t.sob = reinterpret_cast<int *>(t.stw + L.nst);
  t.tiles = reinterpret_cast<C *>(sm + tab_bytes(L, sizeof(C)));
  for (int i = threadIdx.x; i < L.n; i += blockDim.x) t.tw[i] = g.tw[i];
  for (int i = threadIdx.x; i < L.nst; i += blockDim.x) t.stw[i] = g.stw[i];
  for (int i = threadIdx.x; i < L.nob; i += blockDim.x) t.sob[i] = g.sob[i];
  return t;
}

// --------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(QX_THREADS) k_zinv(PipeParams P, const T *__restrict__ cin, long ldc,
                                                      typename c2t<T>::type *__restrict__ bufA,
                                                      FftTabs<T> gt3) {
  typedef typename c2t<T>::type C;
  const int j2 = blockIdx.x;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= pair_count(P)) return;
  const int lo = P.row_lo[j2], hi = P.row_hi[j2];
  if (lo > hi) return;
  const int W = hi - lo + 1, ld = W | 1, k3 = P.k3;
  extern __shared__ unsigned char smraw[];
  SmTabs<T> tb = load_tabs<T>(smraw, P.L3, gt3);
  C *t0 = tb.tiles;
  C *t1 = t0 + k3 * ld;
  const C zero = mk2<T>(0, 0);
  for (int i = threadIdx.x; i < k3 * ld; i += blockDim.x) t0[i] = zero;
  __syncthreads();
  const int bA = P.pairs[2 * p], bB = P.pairs[2 * p + 1];
  const T *cA = cin + (long)bA * ldc;
  const T *cB = bB >= 0 ? cin + (long)bB * ldc : nullptr;
  for (int e = P.row_off[j2] + threadIdx.x; e < P.row_off[j2 + 1]; e += blockDim.x) {
    const int4 en = P.row_ent[e];
    const int ig = en.z;
    T ra = cA[2 * ig], ia = ig ? cA[2 * ig + 1] : T(0);
    T rb = cB ? cB[2 * ig] : T(0), ib = (cB && ig) ? cB[2 * ig + 1] : T(0);
    C z;
    if (en.w > 0) { z.x = ra - ib; z.y = ia + rb; }
    else          { z.x = ra + ib; z.y = rb - ia; }
    t0[en.y * ld + en.x] = z;
  }
  __syncthreads();
  C *res = smem_fft<T, +1>(t0, t1, W, ld, P.L3, tb.tw, tb.stw, tb.sob);
  C *dst = bufA + ((long)pl * k3) * P.P2 * P.P1 + (long)j2 * P.P1 + lo;
  for (int i = threadIdx.x; i < k3 * W; i += blockDim.x) {
    const int i3 = i / W, l = i - i3 * W;
    dst[(long)i3 * P.P2 * P.P1 + l] = res[i3 * ld + l];
  }
}

// y pass.  SIGN=+1: bufA (rows j2, sphere ranges) -> bufB (all i2).
//          SIGN=-1: bufB -> bufA (rows j2, sphere ranges).
template <typename T, int SIGN>
__global__ void __launch_bounds__(QX_THREADS) k_ypass(PipeParams P, typename c2t<T>::type *__restrict__ bufA,
                                                       typename c2t<T>::type *__restrict__ bufB,
                                                       FftTabs<T> gt2) {
  typedef typename c2t<T>::type C;
  const int i3 = blockIdx.x;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= pair_count(P)) return;
  const int k2 = P.k2, P1 = P.P1, P2 = P.P2, ld = P1;   // P1 is odd
  extern __shared__ unsigned char smraw[];
  SmTabs<T> tb = load_tabs<T>(smraw, P.L2, gt2);
  C *t0 = tb.tiles;
  C *t1 = t0 + k2 * ld;
  C *A = bufA + ((long)pl * P.k3 + i3) * P2 * P1;
  C *B = bufB + ((long)pl * P.k3 + i3) * k2 * P1;
  if (SIGN > 0) {
    const C zero = mk2<T>(0, 0);
    for (int i = threadIdx.x; i < k2 * ld; i += blockDim.x) t0[i] = zero;
    __syncthreads();
    for (int i = threadIdx.x; i < P2 * P1; i += blockDim.x) {
      const int j2 = i / P1, a = i - j2 * P1;
      if (a >= P.row_lo[j2] && a <= P.row_hi[j2]) {
        int i2 = j2 - P.m2; if (i2 < 0) i2 += k2;
        t0[i2 * ld + a] = A[i];
      }
    }
    __syncthreads();
    C *res = smem_fft<T, +1>(t0, t1, P1, ld, P.L2, tb.tw, tb.stw, tb.sob);
    for (int i = threadIdx.x; i < k2 * P1; i += blockDim.x) B[i] = res[i];
  } else {
    for (int i = threadIdx.x; i < k2 * P1; i += blockDim.x) t0[i] = B[i];
    __syncthreads();
    C *res = smem_fft<T, -1>(t0, t1, P1, ld, P.L2, tb.tw, tb.stw, tb.sob);
    for (int i = threadIdx.x; i < P2 * P1; i += blockDim.x) {
      const int j2 = i / P1, a = i - j2 * P1;
      if (a >= P.row_lo[j2] && a <= P.row_hi[j2]) {
        int i2 = j2 - P.m2; if (i2 < 0) i2 += k2;
        A[i] = res[i2 * ld + a];
      }
    }
  }
}

__device__ __forceinline__ int a_to_i1(int a, int m1, int k1) {
  int i1 = a - m1;
  return i1 < 0 ? i1 + k1 : i1;
}

// x pass fused with the local potential: backward x-FFT of the pruned line,
// multiply by V(r), forward x-FFT, keep the pruned part.  One CTA handles
// `nlines` consecutive i2 lines of plane i3.
template <typename T>
__global__ void __launch_bounds__(QX_THREADS) k_xvx(PipeParams P, typename c2t<T>::type *__restrict__ bufB,
                                                     const T *__restrict__ vloc, int nlines, int nchunk,
                                                     FftTabs<T> gt1) {
  typedef typename c2t<T>::type C;
  const int i3 = blockIdx.x / nchunk, ch = blockIdx.x - i3 * nchunk;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= pair_count(P)) return;
  const int k1 = P.k1, k2 = P.k2, P1 = P.P1;
  const int i20 = ch * nlines;
  const int nl = min(nlines, k2 - i20);
  const int ld = nl | 1;
  extern __shared__ unsigned char smraw[];
  SmTabs<T> tb = load_tabs<T>(smraw, P.L1, gt1);
  C *t0 = tb.tiles;
  C *t1 = t0 + k1 * ld;
  const C zero = mk2<T>(0, 0);
  for (int i = threadIdx.x; i < k1 * ld; i += blockDim.x) t0[i] = zero;
  __syncthreads();
  C *B = bufB + (((long)pl * P.k3 + i3) * k2 + i20) * P1;
  for (int i = threadIdx.x; i < nl * P1; i += blockDim.x) {
    const int l = i / P1, a = i - l * P1;
    t0[a_to_i1(a, P.m1, k1) * ld + l] = B[i];
  }
  __syncthreads();
  C *r = smem_fft<T, +1>(t0, t1, nl, ld, P.L1, tb.tw, tb.stw, tb.sob);
  C *o = (r == t0) ? t1 : t0;
  const T *V = vloc + ((long)i3 * k2 + i20) * k1;
  for (int i = threadIdx.x; i < nl * k1; i += blockDim.x) {
    const int l = i / k1, i1 = i - l * k1;
    const T v = V[i];
    C z = r[i1 * ld + l];
    z.x *= v; z.y *= v;
    r[i1 * ld + l] = z;
  }
  __syncthreads();
  C *res = smem_fft<T, -1>(r, o, nl, ld, P.L1, tb.tw, tb.stw, tb.sob);
  for (int i = threadIdx.x; i < nl * P1; i += blockDim.x) {
    const int l = i / P1, a = i - l * P1;
    B[i] = res[a_to_i1(a, P.m1, k1) * ld + l];
  }
}

// z pass forward + pick: writes Z(+G) to slot 0 and Z(-G) to slot 1 of zsph.
template <typename T>
__global__ void __launch_bounds__(QX_THREADS) k_zfwd(PipeParams P, const typename c2t<T>::type *__restrict__ bufA,
                                                      typename c2t<T>::type *__restrict__ zsph,
                                                      FftTabs<T> gt3) {
  typedef typename c2t<T>::type C;
  const int j2 = blockIdx.x;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= pair_count(P)) return;
  const int lo = P.row_lo[j2], hi = P.row_hi[j2];
  if (lo > hi) return;
  const int W = hi - lo + 1, ld = W | 1, k3 = P.k3;
  extern __shared__ unsigned char smraw[];
  SmTabs<T> tb = load_tabs<T>(smraw, P.L3, gt3);
  C *t0 = tb.tiles;
  C *t1 = t0 + k3 * ld;
  const C *src = bufA + ((long)pl * k3) * P.P2 * P.P1 + (long)j2 * P.P1 + lo;
  for (int i = threadIdx.x; i < k3 * W; i += blockDim.x) {
    const int i3 = i / W, l = i - i3 * W;
    t0[i3 * ld + l] = src[(long)i3 * P.P2 * P.P1 + l];
  }
  __syncthreads();
  C *res = smem_fft<T, -1>(t0, t1, W, ld, P.L3, tb.tw, tb.stw, tb.sob);
  const T s = (T)P.inv_n;
  C *Z = zsph + (long)pl * (P.nplw + 1) * 2;
  for (int e = P.row_off[j2] + threadIdx.x; e < P.row_off[j2 + 1]; e += blockDim.x) {
    const int4 en = P.row_ent[e];
    C z = res[en.y * ld + en.x];
    z.x *= s; z.y *= s;
    if (en.w > 0) {
      Z[2 * en.z] = z;
      if (en.z == 0) Z[1] = z;
    } else {
      Z[2 * en.z + 1] = z;
    }
  }
}

// Split the two bands of each pair and write H|psi> = [acc ? out : 0]
// + dkgnrm*c (if dk != null) + FFT part.  Component 2 (Im c(G=0)) gets the
// exact 0 imaginary part of a real function's G=0 coefficient.
template <typename T>
__global__ void k_unpack(PipeParams P, const typename c2t<T>::type *__restrict__ zsph,
                         const T *__restrict__ cin, long ldc, T *__restrict__ out, long ldo,
                         const double *__restrict__ dk, int accumulate) {
  typedef typename c2t<T>::type C;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= pair_count(P)) return;
  const int ig = blockIdx.x * blockDim.x + threadIdx.x;
  if (ig > P.nplw) return;
  const C *Z = zsph + (long)pl * (P.nplw + 1) * 2;
  const C zp = Z[2 * ig], zm = Z[2 * ig + 1];
  const T h = (T)0.5;
  T har = h * (zp.x + zm.x), hai = h * (zp.y - zm.y);
  T hbr = h * (zp.y + zm.y), hbi = h * (zm.x - zp.x);
  if (ig == 0) { hai = 0; hbi = 0; }
  const int b[2] = {P.pairs[2 * p], P.pairs[2 * p + 1]};
  const T hr[2] = {har, hbr}, hi[2] = {hai, hbi};
  for (int s = 0; s < 2; ++s) {
    if (b[s] < 0) continue;
    T *o = out + (long)b[s] * ldo;
    const T *c = cin + (long)b[s] * ldc;
    T vr = hr[s], vi = hi[s];
    if (dk) { vr += (T)dk[2 * ig] * c[2 * ig]; vi += (T)dk[2 * ig + 1] * c[2 * ig + 1]; }
    if (accumulate) { vr += o[2 * ig]; vi += o[2 * ig + 1]; }
    o[2 * ig] = vr;
    o[2 * ig + 1] = vi;
  }
}

// --------------------------------------------------------------------------
// Real-space KB variant of the x pass.

// Backward x-FFT only: full real-space lines -> R[p][i3][i2][i1].
template <typename T>
__global__ void __launch_bounds__(QX_THREADS) k_xinv_r(PipeParams P, const typename c2t<T>::type *__restrict__ bufB,
                                                        typename c2t<T>::type *__restrict__ R, int nlines,
                                                        int nchunk, FftTabs<T> gt1) {
  typedef typename c2t<T>::type C;
  const int i3 = blockIdx.x / nchunk, ch = blockIdx.x - i3 * nchunk;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= pair_count(P)) return;
  const int k1 = P.k1, k2 = P.k2, P1 = P.P1;
  const int i20 = ch * nlines, nl = min(nlines, k2 - i20), ld = nl | 1;
  extern __shared__ unsigned char smraw[];
  SmTabs<T> tb = load_tabs<T>(smraw, P.L1, gt1);
  C *t0 = tb.tiles;
  C *t1 = t0 + k1 * ld;
  const C zero = mk2<T>(0, 0);
  for (int i = threadIdx.x; i < k1 * ld; i += blockDim.x) t0[i] = zero;
  __syncthreads();
  const C *B = bufB + (((long)pl * P.k3 + i3) * k2 + i20) * P1;
  for (int i = threadIdx.x; i < nl * P1; i += blockDim.x) {
    const int l = i / P1, a = i - l * P1;
    t0[a_to_i1(a, P.m1, k1) * ld + l] = B[i];
  }
  __syncthreads();
  C *r = smem_fft<T, +1>(t0, t1, nl, ld, P.L1, tb.tw, tb.stw, tb.sob);
  C *dst = R + (((long)pl * P.k3 + i3) * k2 + i20) * k1;
  for (int i = threadIdx.x; i < nl * k1; i += blockDim.x) {
    const int l = i / k1, i1 = i - l * k1;
    dst[i] = r[i1 * ld + l];
  }
}

// Real-space KB force of one (atom, band pair) (fnnlcl2, nlkbppr.f90:2024-3120):
// for each band b of the pair, P_l = rdelv sum_points vnl_l psi_b and
// D_l = rdelv sum_points grad vnl_l psi_b (gradient with respect to the
// point), then F_a += 2 occ_b / Omega sum_l clalp_l P_l D_l; one partial per
// pair in fpart[(pair * natom + atom) * 3 + dim] (summed over pairs in a
// fixed order afterwards).  wocc = occ / Omega.  lmx <= ML projectors per
// point (ML = 4: s, p; ML = 9: s, p, d).
template <typename T, int ML>
__global__ void __launch_bounds__(QX_THREADS) k_fnl_r(PipeParams P, const typename c2t<T>::type *__restrict__ R,
                                                       const int *__restrict__ off, const int *__restrict__ mesh,
                                                       const T *__restrict__ vnl, const T *__restrict__ dvnl,
                                                       const double *__restrict__ clalp, double rdelv, int natom,
                                                       int lmx, const double *__restrict__ wocc, int npl, int ppb,
                                                       double *__restrict__ fpart) {
  typedef typename c2t<T>::type C;
  constexpr int NQ = 8 * ML;   // P[band][l] (2 ML), then D[band][l][dim] (6 ML)
  const int at = blockIdx.x;
  // ppb pairs of the chunk per block, one after another, so that the atom's
  // table slice is read from cache after the first
  const int pend = min(npl, (int)(blockIdx.y + 1) * ppb);
  for (int pl = blockIdx.y * ppb; pl < pend; ++pl) {
  const int p = P.pair0 + pl;
  if (p >= pair_count(P)) break;   // uniform across the block
  const long n = (long)P.k1 * P.k2 * P.k3;
  const C *Rp = R + (long)pl * n;
  double acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
  for (int mm = off[at] + threadIdx.x; mm < off[at + 1]; mm += blockDim.x) {
    const C z = Rp[mesh[mm]];
#pragma unroll
    for (int l = 0; l < ML; ++l) {
      if (l >= lmx) break;   // uniform
      const double v = (double)vnl[(long)mm * lmx + l];
      acc[l] += v * (double)z.x;
      acc[ML + l] += v * (double)z.y;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double g = (double)dvnl[((long)mm * lmx + l) * 3 + d];
        acc[2 * ML + l * 3 + d] += g * (double)z.x;
        acc[5 * ML + l * 3 + d] += g * (double)z.y;
      }
    }
  }
  // the NQ sums: warp shuffles, then one pass over the warps' partials
  __shared__ double red[QX_THREADS / 32][NQ];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double v = acc[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][q] = v;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < NQ; q += blockDim.x) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][q];
    red[0][q] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double *s = red[0];
    const int b[2] = {P.pairs[2 * p], P.pairs[2 * p + 1]};
    double f[3] = {0.0, 0.0, 0.0};
    for (int h = 0; h < 2; ++h) {
      if (b[h] < 0) continue;
      const double w = 2.0 * wocc[b[h]] * rdelv * rdelv;
      for (int l = 0; l < lmx; ++l)
        for (int d = 0; d < 3; ++d) f[d] += w * clalp[l] * s[h * ML + l] * s[2 * ML + 3 * ML * h + l * 3 + d];
    }
    double *o = fpart + ((long)p * natom + at) * 3;
    o[0] = f[0];
    o[1] = f[1];
    o[2] = f[2];
  }
  __syncthreads();
  }
}

// fnl[atom * 3 + dim] = sum over pairs of fpart, in pair order
__global__ void k_fnl_r_sum(const double *__restrict__ fpart, int npair, int natom, double *__restrict__ fnl) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= natom * 3) return;
  double s = 0.0;
  for (int p = 0; p < npair; ++p) s += fpart[(long)p * natom * 3 + q];
  fnl[q] = s;
}

// sumr(l, atom) = rdelv * clalp_l * sum_points vnl_l * psi(point), both bands
// of the pair at once (real part band A, imaginary part band B); lmx <= ML
// projectors per point.
template <typename T, int ML>
__global__ void __launch_bounds__(QX_THREADS) k_nlproj(PipeParams P, const typename c2t<T>::type *__restrict__ R,
                                                        const int *__restrict__ off, const int *__restrict__ mesh,
                                                        const T *__restrict__ vnl, const double *__restrict__ clalp,
                                                        double rdelv, int natom, int lmx,
                                                        typename c2t<T>::type *__restrict__ sumr) {
  typedef typename c2t<T>::type C;
  const int at = blockIdx.x;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= pair_count(P)) return;
  const long n = (long)P.k1 * P.k2 * P.k3;
  const C *Rp = R + (long)pl * n;
  double acc[2 * ML];
#pragma unroll
  for (int q = 0; q < 2 * ML; ++q) acc[q] = 0.0;
  for (int mm = off[at] + threadIdx.x; mm < off[at + 1]; mm += blockDim.x) {
    const C z = Rp[mesh[mm]];
#pragma unroll
    for (int l = 0; l < ML; ++l) {
      if (l >= lmx) break;   // uniform
      const double v = (double)vnl[(long)mm * lmx + l];
      acc[2 * l] += v * (double)z.x;
      acc[2 * l + 1] += v * (double)z.y;
    }
  }
  __shared__ double red[QX_THREADS / 32];
  for (int l = 0; l < 2 * lmx; ++l) {
    const double s = block_sum(acc[l], red);
    if (threadIdx.x == 0) acc[l] = s;
  }
  if (threadIdx.x == 0) {
    C *o = sumr + ((long)pl * natom + at) * lmx;
    for (int l = 0; l < lmx; ++l) {
      const double f = rdelv * clalp[l];
      o[l] = mk2<T>((T)(acc[2 * l] * f), (T)(acc[2 * l + 1] * f));
    }
  }
}

// Forward x pass for the real-space KB mode: V*psi + sum vnl*sumr, forward
// x-FFT, keep the pruned part.  Line CSR `loff/lent` lists the projector
// points of each line (i3*k2 + i2): {i1, point index, atom}.
template <typename T, int ML>
__global__ void __launch_bounds__(QX_THREADS) k_xfwd_r(PipeParams P, const typename c2t<T>::type *__restrict__ R,
                                                        typename c2t<T>::type *__restrict__ bufB,
                                                        const T *__restrict__ vloc, const int *__restrict__ loff,
                                                        const int4 *__restrict__ lent, const T *__restrict__ vnl,
                                                        const typename c2t<T>::type *__restrict__ sumr, int natom,
                                                        int lmx, int nlines, int nchunk,
                                                        FftTabs<T> gt1) {
  typedef typename c2t<T>::type C;
  const int i3 = blockIdx.x / nchunk, ch = blockIdx.x - i3 * nchunk;
  const int pl = blockIdx.y, p = P.pair0 + pl;
  if (p >= pair_count(P)) return;
  const int k1 = P.k1, k2 = P.k2, P1 = P.P1;
  const int i20 = ch * nlines, nl = min(nlines, k2 - i20), ld = nl | 1;
  extern __shared__ unsigned char smraw[];
  SmTabs<T> tb = load_tabs<T>(smraw, P.L1, gt1);
  C *t0 = tb.tiles;
  C *t1 = t0 + k1 * ld;
  const C *src = R + (((long)pl * P.k3 + i3) * k2 + i20) * k1;
  const T *V = vloc + ((long)i3 * k2 + i20) * k1;
  for (int i = threadIdx.x; i < nl * k1; i += blockDim.x) {
    const int l = i / k1, i1 = i - l * k1;
    C z = src[i];
    const T v = V[i];
    z.x *= v; z.y *= v;
    t0[i1 * ld + l] = z;
  }
  __syncthreads();
  const C *S = sumr + (long)pl * natom * lmx;
  const int line0 = i3 * k2 + i20;
  for (int l = 0; l < nl; ++l) {
    for (int e = loff[line0 + l] + threadIdx.x; e < loff[line0 + l + 1]; e += blockDim.x) {
      const int4 en = lent[e];
      const C *s = S + (long)en.z * lmx;
      const T *v = vnl + (long)en.y * lmx;
      T ar = 0, ai = 0;
#pragma unroll
      for (int q = 0; q < ML; ++q) {
        if (q >= lmx) break;   // uniform
        ar += v[q] * s[q].x;
        ai += v[q] * s[q].y;
      }
      atomicAdd(&t0[en.x * ld + l].x, ar);
      atomicAdd(&t0[en.x * ld + l].y, ai);
    }
  }
  __syncthreads();
  C *res = smem_fft<T, -1>(t0, t1, nl, ld, P.L1, tb.tw, tb.stw, tb.sob);
  C *B = bufB + (((long)pl * P.k3 + i3) * k2 + i20) * P1;
  for (int i = threadIdx.x; i < nl * P1; i += blockDim.x) {
    const int l = i / P1, a = i - l * P1;
    B[i] = res[a_to_i1(a, P.m1, k1) * ld + l];
  }
}

// --------------------------------------------------------------------------
// Density: rho(r) += occ_A/Omega * psiA(r)^2 + occ_B/Omega * psiB(r)^2 over
// all pairs; one CTA owns `nlines` lines of a plane and loops over the pairs,
// so the sum is deterministic and needs no atomics.  accumulate=0 overwrites.
template <typename T>
__global__ void __launch_bounds__(QX_THREADS) k_xrho(PipeParams P, const typename c2t<T>::type *__restrict__ bufB,
                                                      const double *__restrict__ wocc, double *__restrict__ rho,
                                                      int nlines, int nchunk, int accumulate,
                                                      FftTabs<T> gt1) {
  typedef typename c2t<T>::type C;
  const int i3 = blockIdx.x / nchunk, ch = blockIdx.x - i3 * nchunk;
  const int k1 = P.k1, k2 = P.k2, P1 = P.P1;
  const int i20 = ch * nlines, nl = min(nlines, k2 - i20), ld = nl | 1;
  extern __shared__ unsigned char smraw[];
  SmTabs<T> tb = load_tabs<T>(smraw, P.L1, gt1);
  C *t0 = tb.tiles;
  C *t1 = t0 + k1 * ld;
  double *acc = reinterpret_cast<double *>(t1 + k1 * ld);
  for (int i = threadIdx.x; i < nl * k1; i += blockDim.x) acc[i] = 0.0;
  const int np = min(pair_count(P) - P.pair0, P.npair);
  const C zero = mk2<T>(0, 0);
  for (int pl = 0; pl < np; ++pl) {
    const int p = P.pair0 + pl;
    for (int i = threadIdx.x; i < k1 * ld; i += blockDim.x) t0[i] = zero;
    __syncthreads();
    const C *B = bufB + (((long)pl * P.k3 + i3) * k2 + i20) * P1;
    for (int i = threadIdx.x; i < nl * P1; i += blockDim.x) {
      const int l = i / P1, a = i - l * P1;
      t0[a_to_i1(a, P.m1, k1) * ld + l] = B[i];
    }
    __syncthreads();
    C *r = smem_fft<T, +1>(t0, t1, nl, ld, P.L1, tb.tw, tb.stw, tb.sob);
    const int bA = P.pairs[2 * p], bB = P.pairs[2 * p + 1];
    const double fa = wocc[bA], fb = bB >= 0 ? wocc[bB] : 0.0;
    for (int i = threadIdx.x; i < nl * k1; i += blockDim.x) {
      const int l = i / k1, i1 = i - l * k1;
      const C z = r[i1 * ld + l];
      acc[i] += fa * (double)z.x * (double)z.x + fb * (double)z.y * (double)z.y;
    }
    __syncthreads();
  }
  double *dst = rho + ((long)i3 * k2 + i20) * k1;
  for (int i = threadIdx.x; i < nl * k1; i += blockDim.x) dst[i] = accumulate ? dst[i] + acc[i] : acc[i];
}

// --------------------------------------------------------------------------
// Full-grid complex 3D FFT passes (density side, rfft3/fft3 drop-in).
template <typename T, int SIGN>
__global__ void __launch_bounds__(QX_THREADS) k_full_z(typename c2t<T>::type *__restrict__ g, int k1, int k2, int k3,
                                                        int tx, FftLen L3, FftTabs<T> gt3) {
  typedef typename c2t<T>::type C;
  const int nxc = (k1 + tx - 1) / tx;
  const int i2 = blockIdx.x / nxc, i10 = (blockIdx.x - i2 * nxc) * tx;
  const int nl = min(tx, k1 - i10), ld = nl | 1;
  extern __shared__ unsigned char smraw[];
  SmTabs<T> tb = load_tabs<T>(smraw, L3, gt3);
  C *t0 = tb.tiles;
  C *t1 = t0 + k3 * ld;
  for (int i = threadIdx.x; i < k3 * nl; i += blockDim.x) {
    const int i3 = i / nl, l = i - i3 * nl;
    t0[i3 * ld + l] = g[((long)i3 * k2 + i2) * k1 + i10 + l];
  }
  __syncthreads();
  C *r = smem_fft<T, SIGN>(t0, t1, nl, ld, L3, tb.tw, tb.stw, tb.sob);
  for (int i = threadIdx.x; i < k3 * nl; i += blockDim.x) {
    const int i3 = i / nl, l = i - i3 * nl;
    g[((long)i3 * k2 + i2) * k1 + i10 + l] = r[i3 * ld + l];
  }
}

template <typename T, int SIGN>
__global__ void __launch_bounds__(QX_THREADS) k_full_y(typename c2t<T>::type *__restrict__ g, int k1, int k2, int k3,
                                                        int tx, FftLen L2, FftTabs<T> gt2) {
  typedef typename c2t<T>::type C;
  const int nxc = (k1 + tx - 1) / tx;
  const int i3 = blockIdx.x / nxc, i10 = (blockIdx.x - i3 * nxc) * tx;
  const int nl = min(tx, k1 - i10), ld = nl | 1;
  extern __shared__ unsigned char smraw[];
  SmTabs<T> tb = load_tabs<T>(smraw, L2, gt2);
  C *t0 = tb.tiles;
  C *t1 = t0 + k2 * ld;
  C *base = g + (long)i3 * k2 * k1 + i10;
  for (int i = threadIdx.x; i < k2 * nl; i += blockDim.x) {
    const int i2 = i / nl, l = i - i2 * nl;
    t0[i2 * ld + l] = base[(long)i2 * k1 + l];
  }
  __syncthreads();
  C *r = smem_fft<T, SIGN>(t0, t1, nl, ld, L2, tb.tw, tb.stw, tb.sob);
  for (int i = threadIdx.x; i < k2 * nl; i += blockDim.x) {
    const int i2 = i / nl, l = i - i2 * nl;
    base[(long)i2 * k1 + l] = r[i2 * ld + l];
  }
}

template <typename T, int SIGN>
__global__ void __launch_bounds__(QX_THREADS) k_full_x(typename c2t<T>::type *__restrict__ g, int k1, int k2, int k3,
                                                        int nlines, FftLen L1, FftTabs<T> gt1,
                                                        double scale) {
  typedef typename c2t<T>::type C;
  const int nch = (k2 + nlines - 1) / nlines;
  const int i3 = blockIdx.x / nch, i20 = (blockIdx.x - i3 * nch) * nlines;
  const int nl = min(nlines, k2 - i20), ld = nl | 1;
  extern __shared__ unsigned char smraw[];
  SmTabs<T> tb = load_tabs<T>(smraw, L1, gt1);
  C *t0 = tb.tiles;
  C *t1 = t0 + k1 * ld;
  C *base = g + ((long)i3 * k2 + i20) * k1;
  for (int i = threadIdx.x; i < nl * k1; i += blockDim.x) {
    const int l = i / k1, i1 = i - l * k1;
    t0[i1 * ld + l] = base[i];
  }
  __syncthreads();
  C *r = smem_fft<T, SIGN>(t0, t1, nl, ld, L1, tb.tw, tb.stw, tb.sob);
  const T s = (T)scale;
  for (int i = threadIdx.x; i < nl * k1; i += blockDim.x) {
    const int l = i / k1, i1 = i - l * k1;
    C z = r[i1 * ld + l];
    z.x *= s; z.y *= s;
    base[i] = z;
  }
}

// --------------------------------------------------------------------------
// Host-side launchers (called from qx_api.cu).

namespace qx {

static size_t fft_smem(const FftLen &L, int ld, size_t cs) { return tab_bytes(L, cs) + 2 * (size_t)L.n * ld * cs; }

template <typename T>
static FftTabs<T> tabs(const Plan &pl, int d) {
  Bufs<T> &bf = pl.bufs<T>();
  FftTabs<T> t;
  t.tw = bf.tw + pl.tw_off[d];
  t.stw = bf.stw + pl.stw_off[d];
  t.sob = pl.d_sob + pl.sob_off[d];
  return t;
}

// The fused register-FFT plane pass is on unless QX_PLANE=0 (kept to compare
// against the shared-memory passes; read at every launch).
static bool plane_enabled() {
  const char *e = getenv("QX_PLANE");
  return !(e && e[0] == '0');
}

// Forward z pass one sphere column a thread (k_zcols_fwd) for columns of at
// most 32 points, where it measured faster than the shared-memory pass (the
// 48-cell batch, z lengths 21-27: 9365 -> 9735 cell-iter/s); at 54 points
// (Si64) it measured 2.5 % slower.  QX_ZCOLS_FWD=0 / 1 forces either (read at
// every call).
static bool zcols_fwd_enabled(int k3) {
  const char *e = getenv("QX_ZCOLS_FWD");
  if (e && (e[0] == '0' || e[0] == '1')) return e[0] == '1';
  return k3 <= 32;
}

template <typename T>
int launch_hpsi_chunk(const Plan &pl, const PipeParams &P, int npl, const T *cin, long ldc, T *out, long ldo,
                      const double *dk, int accumulate, int nlmode, cudaStream_t st, cudaEvent_t before_unpack) {
  typedef typename c2t<T>::type C;
  const size_t cs = sizeof(C);
  Bufs<T> &bf = pl.bufs<T>();
  const FftTabs<T> g1 = tabs<T>(pl, 0), g2 = tabs<T>(pl, 1), g3 = tabs<T>(pl, 2);
  dim3 gz(P.P2, npl);
  const size_t smz = fft_smem(P.L3, P.P1 | 1, cs);
  const bool zc = sizeof(T) == sizeof(float) &&
                  launch_zcols_inv_f32(P, npl, (const float *)cin, ldc, (float2 *)bf.bufA, st) == 0;
  if (!zc) { k_zinv<T><<<gz, QX_THREADS, smz, st>>>(P, cin, ldc, bf.bufA, g3); note_launch(); }
  auto zfwd = [&]() {
    if (sizeof(T) == sizeof(float) && zcols_fwd_enabled(P.k3) &&
        launch_zcols_fwd_f32(P, npl, (const float2 *)bf.bufA, (float2 *)bf.zsph, st) == 0)
      return;
    k_zfwd<T><<<gz, QX_THREADS, smz, st>>>(P, bf.bufA, bf.zsph, g3); note_launch();
  };
  dim3 gy(P.k3, npl);
  const size_t smy = fft_smem(P.L2, P.P1, cs);
  if (sizeof(T) == sizeof(float) && nlmode != 2 && pl.use_plane && plane_enabled() &&
      launch_plane_f32(P, npl, (float2 *)bf.bufA, (const float *)bf.vloc, st) == 0) {
    dim3 gu((P.nplw + 1 + 127) / 128, npl);
    zfwd();
    if (before_unpack) cudaStreamWaitEvent(st, before_unpack, 0);
    k_unpack<T><<<gu, 128, 0, st>>>(P, bf.zsph, cin, ldc, out, ldo, dk, accumulate); note_launch();
    return 0;
  }
  k_ypass<T, +1><<<gy, QX_THREADS, smy, st>>>(P, bf.bufA, bf.bufB, g2); note_launch();
  const int nlines = pl.xlines<T>();
  const int nch = (P.k2 + nlines - 1) / nlines;
  dim3 gx(P.k3 * nch, npl);
  const size_t smx = fft_smem(P.L1, nlines | 1, cs);
  if (nlmode == 2) {
    k_xinv_r<T><<<gx, QX_THREADS, smx, st>>>(P, bf.bufB, bf.bufR, nlines, nch, g1); note_launch();
    dim3 ga(pl.natom, npl);
    if (pl.kb_lmx <= 4) {
      k_nlproj<T, 4><<<ga, QX_THREADS, 0, st>>>(P, bf.bufR, pl.d_kb_off, pl.d_kb_mesh, bf.kb_vnl, pl.d_kb_clalp,
                                                pl.rdelv, pl.natom, pl.kb_lmx, bf.sumr); note_launch();
      k_xfwd_r<T, 4><<<gx, QX_THREADS, smx, st>>>(P, bf.bufR, bf.bufB, bf.vloc, pl.d_line_off, pl.d_line_ent,
                                                  bf.kb_vnl, bf.sumr, pl.natom, pl.kb_lmx, nlines, nch, g1);
      note_launch();
    } else {
      k_nlproj<T, 9><<<ga, QX_THREADS, 0, st>>>(P, bf.bufR, pl.d_kb_off, pl.d_kb_mesh, bf.kb_vnl, pl.d_kb_clalp,
                                                pl.rdelv, pl.natom, pl.kb_lmx, bf.sumr); note_launch();
      k_xfwd_r<T, 9><<<gx, QX_THREADS, smx, st>>>(P, bf.bufR, bf.bufB, bf.vloc, pl.d_line_off, pl.d_line_ent,
                                                  bf.kb_vnl, bf.sumr, pl.natom, pl.kb_lmx, nlines, nch, g1);
      note_launch();
    }
  } else {
    k_xvx<T><<<gx, QX_THREADS, smx, st>>>(P, bf.bufB, bf.vloc, nlines, nch, g1); note_launch();
  }
  k_ypass<T, -1><<<gy, QX_THREADS, smy, st>>>(P, bf.bufA, bf.bufB, g2); note_launch();
  zfwd();
  dim3 gu((P.nplw + 1 + 127) / 128, npl);
  if (before_unpack) cudaStreamWaitEvent(st, before_unpack, 0);
  k_unpack<T><<<gu, 128, 0, st>>>(P, bf.zsph, cin, ldc, out, ldo, dk, accumulate); note_launch();
  return 0;
}

template <typename T>
int launch_rho_chunk(const Plan &pl, const PipeParams &P, int npl, const T *cin, long ldc, const double *wocc,
                     double *rho, int accumulate, cudaStream_t st) {
  typedef typename c2t<T>::type C;
  const size_t cs = sizeof(C);
  Bufs<T> &bf = pl.bufs<T>();
  const FftTabs<T> g1 = tabs<T>(pl, 0), g2 = tabs<T>(pl, 1), g3 = tabs<T>(pl, 2);
  dim3 gz(P.P2, npl);
  if (!(sizeof(T) == sizeof(float) &&
        launch_zcols_inv_f32(P, npl, (const float *)cin, ldc, (float2 *)bf.bufA, st) == 0)) {
    k_zinv<T><<<gz, QX_THREADS, fft_smem(P.L3, P.P1 | 1, cs), st>>>(P, cin, ldc, bf.bufA, g3); note_launch();
  }
  if (sizeof(T) == sizeof(float) && pl.use_plane && plane_enabled() && bf.rho_part &&
      launch_rho_plane_f32(P, npl, (const float2 *)bf.bufA, wocc, bf.rho_part, rho, accumulate, st) == 0)
    return 0;
  dim3 gy(P.k3, npl);
  k_ypass<T, +1><<<gy, QX_THREADS, fft_smem(P.L2, P.P1, cs), st>>>(P, bf.bufA, bf.bufB, g2); note_launch();
  const int nlines = pl.rholines;
  const int nch = (P.k2 + nlines - 1) / nlines;
  const size_t sm = fft_smem(P.L1, nlines | 1, cs) + sizeof(double) * nlines * P.k1;
  k_xrho<T><<<P.k3 * nch, QX_THREADS, sm, st>>>(P, bf.bufB, wocc, rho, nlines, nch, accumulate, g1); note_launch();
  return 0;
}

// psi(r) of a chunk of band pairs (z, y, x inverse passes into bufR) and the
// real-space KB force partials of every (atom, pair).
template <typename T>
int launch_fnl_r_chunk(const Plan &pl, const PipeParams &P, int npl, const T *cin, long ldc, const T *dvnl,
                       const double *wocc, double *fpart, cudaStream_t st) {
  typedef typename c2t<T>::type C;
  const size_t cs = sizeof(C);
  Bufs<T> &bf = pl.bufs<T>();
  const FftTabs<T> g1 = tabs<T>(pl, 0), g2 = tabs<T>(pl, 1), g3 = tabs<T>(pl, 2);
  dim3 gz(P.P2, npl);
  if (!(sizeof(T) == sizeof(float) &&
        launch_zcols_inv_f32(P, npl, (const float *)cin, ldc, (float2 *)bf.bufA, st) == 0)) {
    k_zinv<T><<<gz, QX_THREADS, fft_smem(P.L3, P.P1 | 1, cs), st>>>(P, cin, ldc, bf.bufA, g3); note_launch();
  }
  dim3 gy(P.k3, npl);
  k_ypass<T, +1><<<gy, QX_THREADS, fft_smem(P.L2, P.P1, cs), st>>>(P, bf.bufA, bf.bufB, g2); note_launch();
  const int nlines = pl.xlines<T>();
  const int nch = (P.k2 + nlines - 1) / nlines;
  dim3 gx(P.k3 * nch, npl);
  k_xinv_r<T><<<gx, QX_THREADS, fft_smem(P.L1, nlines | 1, cs), st>>>(P, bf.bufB, bf.bufR, nlines, nch, g1);
  note_launch();
  // about four blocks per SM: pairs split over gy groups of ppb
  const int gyf = std::max(1, std::min(npl, (4 * 148 + pl.natom - 1) / pl.natom));
  const int ppb = (npl + gyf - 1) / gyf;
  dim3 ga(pl.natom, (npl + ppb - 1) / ppb);
  if (pl.kb_lmx <= 4)
    k_fnl_r<T, 4><<<ga, QX_THREADS, 0, st>>>(P, bf.bufR, pl.d_kb_off, pl.d_kb_mesh, bf.kb_vnl, dvnl, pl.d_kb_clalp,
                                             pl.rdelv, pl.natom, pl.kb_lmx, wocc, npl, ppb, fpart);
  else
    k_fnl_r<T, 9><<<ga, QX_THREADS, 0, st>>>(P, bf.bufR, pl.d_kb_off, pl.d_kb_mesh, bf.kb_vnl, dvnl, pl.d_kb_clalp,
                                             pl.rdelv, pl.natom, pl.kb_lmx, wocc, npl, ppb, fpart);
  note_launch();
  return 0;
}

void fnl_r_sum(const double *fpart, int npair, int natom, double *fnl, cudaStream_t st) {
  k_fnl_r_sum<<<(natom * 3 + 127) / 128, 128, 0, st>>>(fpart, npair, natom, fnl);
  note_launch();
}

template <typename T>
int launch_full_fft(const Plan &pl, typename c2t<T>::type *g, int sign, double scale, cudaStream_t st) {
  typedef typename c2t<T>::type C;
  const size_t cs = sizeof(C);
  const FftTabs<T> g1 = tabs<T>(pl, 0), g2 = tabs<T>(pl, 1), g3 = tabs<T>(pl, 2);
  const int k1 = pl.k1, k2 = pl.k2, k3 = pl.k3;
  const int tx = 16;
  const int nxc = (k1 + tx - 1) / tx;
  const int nlines = pl.xlines<T>();
  const int nch = (k2 + nlines - 1) / nlines;
  const FftLen &L1 = pl.L[0], &L2 = pl.L[1], &L3 = pl.L[2];
  // FP64 lines of at most 32 points: one line per thread in registers (the
  // x pass applies the scale)
  auto lines = [&](int axis) {
    return sizeof(T) == sizeof(double) &&
           launch_full_lines_f64((double2 *)g, k1, k2, k3, axis, sign, scale, st) == 0;
  };
  if (sign > 0) {
    if (!lines(2)) { k_full_z<T, +1><<<k2 * nxc, QX_THREADS, fft_smem(L3, tx | 1, cs), st>>>(g, k1, k2, k3, tx, L3, g3); note_launch(); }
    if (!lines(1)) { k_full_y<T, +1><<<k3 * nxc, QX_THREADS, fft_smem(L2, tx | 1, cs), st>>>(g, k1, k2, k3, tx, L2, g2); note_launch(); }
    if (!lines(0)) { k_full_x<T, +1><<<k3 * nch, QX_THREADS, fft_smem(L1, nlines | 1, cs), st>>>(g, k1, k2, k3, nlines, L1, g1, scale); note_launch(); }
  } else {
    if (!lines(2)) { k_full_z<T, -1><<<k2 * nxc, QX_THREADS, fft_smem(L3, tx | 1, cs), st>>>(g, k1, k2, k3, tx, L3, g3); note_launch(); }
    if (!lines(1)) { k_full_y<T, -1><<<k3 * nxc, QX_THREADS, fft_smem(L2, tx | 1, cs), st>>>(g, k1, k2, k3, tx, L2, g2); note_launch(); }
    if (!lines(0)) { k_full_x<T, -1><<<k3 * nch, QX_THREADS, fft_smem(L1, nlines | 1, cs), st>>>(g, k1, k2, k3, nlines, L1, g1, scale); note_launch(); }
  }
  return 0;
}

// Roots of unity of the register DFTs, on the current device.
int init_fft_roots() {
  float2 h32[10 * 16];
  double2 h64[10 * 16];
  const double tp = 2.0 * 3.14159265358979323846;
  for (int R = 0; R < 10; ++R)
    for (int m = 0; m < 16; ++m) {
      const double ang = (R > 0 && m < R) ? tp * m / R : 0.0;
      h64[R * 16 + m] = make_double2(std::cos(ang), -std::sin(ang));
      h32[R * 16 + m] = make_float2((float)std::cos(ang), (float)-std::sin(ang));
    }
  if (cudaMemcpyToSymbol(c_root32, h32, sizeof(h32)) != cudaSuccess) return 1;
  if (cudaMemcpyToSymbol(c_root64, h64, sizeof(h64)) != cudaSuccess) return 1;
  return 0;
}

// Largest dynamic shared memory any pipeline launch of this plan needs.
template <typename T>
size_t fft_smem_need(const Plan &pl) {
  const size_t cs = sizeof(typename c2t<T>::type);
  size_t need = 0;
  need = std::max(need, fft_smem(pl.L[2], pl.P1 | 1, cs));
  need = std::max(need, fft_smem(pl.L[1], pl.P1, cs));
  need = std::max(need, fft_smem(pl.L[0], pl.xlines<T>() | 1, cs));
  need = std::max(need, fft_smem(pl.L[0], pl.rholines | 1, cs) + sizeof(double) * pl.rholines * pl.k1);
  need = std::max(need, fft_smem(pl.L[2], 17, cs));
  need = std::max(need, fft_smem(pl.L[1], 17, cs));
  return need;
}
template size_t fft_smem_need<float>(const Plan &);
template size_t fft_smem_need<double>(const Plan &);

// Opt every kernel above into the shared-memory size the largest plan needs.
// The attribute is per process and contexts of different grids coexist, so
// it only ever grows.
template <typename T>
void set_fft_smem_limits(size_t bytes) {
  static std::mutex mu;
  static size_t cur = 0;
  std::lock_guard<std::mutex> lock(mu);
  if (bytes <= cur) return;
  cur = bytes;
  cudaFuncSetAttribute(k_zinv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_ypass<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_ypass<T, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_xvx<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_zfwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_xinv_r<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_xfwd_r<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_xfwd_r<T, 9>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_xrho<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_full_z<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_full_z<T, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_full_y<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_full_y<T, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_full_x<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_full_x<T, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template int launch_hpsi_chunk<float>(const Plan &, const PipeParams &, int, const float *, long, float *, long,
                                      const double *, int, int, cudaStream_t, cudaEvent_t);
template int launch_hpsi_chunk<double>(const Plan &, const PipeParams &, int, const double *, long, double *, long,
                                       const double *, int, int, cudaStream_t, cudaEvent_t);
template int launch_rho_chunk<float>(const Plan &, const PipeParams &, int, const float *, long, const double *,
                                     double *, int, cudaStream_t);
template int launch_rho_chunk<double>(const Plan &, const PipeParams &, int, const double *, long, const double *,
                                      double *, int, cudaStream_t);
template int launch_fnl_r_chunk<float>(const Plan &, const PipeParams &, int, const float *, long, const float *,
                                       const double *, double *, cudaStream_t);
template int launch_fnl_r_chunk<double>(const Plan &, const PipeParams &, int, const double *, long, const double *,
                                        const double *, double *, cudaStream_t);
template int launch_full_fft<float>(const Plan &, float2 *, int, double, cudaStream_t);
template int launch_full_fft<double>(const Plan &, double2 *, int, double, cudaStream_t);
template void set_fft_smem_limits<float>(size_t);
template void set_fft_smem_limits<double>(size_t);

}  // namespace qx
