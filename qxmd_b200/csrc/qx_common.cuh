// Shared definitions for the sm_100a Kohn-Sham hot-path kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define QX_THREADS 256

template <typename T> struct c2t;
template <> struct c2t<float> { typedef float2 type; };
template <> struct c2t<double> { typedef double2 type; };

template <typename T> __host__ __device__ __forceinline__ typename c2t<T>::type mk2(T x, T y) {
  typename c2t<T>::type r; r.x = x; r.y = y; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }

// One 1D transform length: radices (product = n) and the offset of its
// twiddle table w[t] = exp(-2 pi i t / n), t < n, in the plan's twiddle array.
struct FftLen {
  int n;
  int nstage;
  int radix[8];
  int tw_off;
};

// Batched in-shared-memory Stockham FFT (decimation in time, natural order
// in and out).  `nl` lines of length L.n, element-major: element e of line l
// at buf[e * ld + l].  Ping-pongs between buf and tmp; returns the buffer
// holding the result.  SIGN = -1 forward, +1 backward (unscaled).  `tw` is the
// length's twiddle table (in shared memory).  Must be called by all threads of
// the block; ends with a __syncthreads.
template <typename T, int SIGN>
__device__ typename c2t<T>::type *smem_fft(typename c2t<T>::type *buf, typename c2t<T>::type *tmp,
                                           int nl, int ld, const FftLen &L,
                                           const typename c2t<T>::type *tw) {
  typedef typename c2t<T>::type C;
  const int n = L.n;
  int ns = 1;
  C *a = buf, *b = tmp;
  for (int s = 0; s < L.nstage; ++s) {
    const int R = L.radix[s];
    const int nr = n / R;
    const int tstep = n / (ns * R);   // twiddle index step for k*r
    const int dstep = nr;             // DFT-constant index step for r*q
    const int work = nl * nr;
    for (int w = threadIdx.x; w < work; w += blockDim.x) {
      const int l = w % nl;
      const int j = w / nl;
      const int k = j % ns;
      C v[8];
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r < R) {
          C x = a[(j + r * nr) * ld + l];
          if (r > 0 && k > 0) {
            C t = tw[(k * r * tstep) % n];
            if (SIGN > 0) t.y = -t.y;
            x = cmul(x, t);
          }
          v[r] = x;
        }
      C o[8];
      if (R == 2) {
        o[0] = cadd(v[0], v[1]);
        o[1] = csub(v[0], v[1]);
      } else if (R == 4) {
        C s0 = cadd(v[0], v[2]), d0 = csub(v[0], v[2]);
        C s1 = cadd(v[1], v[3]), d1 = csub(v[1], v[3]);
        // multiply d1 by SIGN*i
        C jd1;
        if (SIGN < 0) { jd1.x = d1.y; jd1.y = -d1.x; } else { jd1.x = -d1.y; jd1.y = d1.x; }
        o[0] = cadd(s0, s1);
        o[2] = csub(s0, s1);
        o[1] = cadd(d0, jd1);
        o[3] = csub(d0, jd1);
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (q < R) {
            C acc = v[0];
#pragma unroll
            for (int r = 1; r < 8; ++r)
              if (r < R) {
                C t = tw[((r * q) % R) * dstep];
                if (SIGN > 0) t.y = -t.y;
                C p = cmul(v[r], t);
                acc = cadd(acc, p);
              }
            o[q] = acc;
          }
      }
      const int idx = (j / ns) * ns * R + k;
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (q < R) b[(idx + q * ns) * ld + l] = o[q];
    }
    __syncthreads();
    C *t = a; a = b; b = t;
    ns *= R;
  }
  return a;
}

// Block-wide sum of a double (all threads get the result).  `red` is a
// shared array of at least blockDim.x/32 doubles.
__device__ __forceinline__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  double r = 0.0;
  for (int i = 0; i < nw; ++i) r += red[i];
  __syncthreads();
  return r;
}
