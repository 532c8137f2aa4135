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

// One 1D transform length: radices (product = n), and offsets of its tables
// in the plan's arrays: the base twiddles w[t] = exp(-2 pi i t / n) (n
// entries), per stage the output base index of each butterfly
// ((j / ns) * ns * R + j % ns, n/R ints) and its R-1 input twiddles
// (w^{(j % ns) * r * n/(ns R)}, r = 1..R-1).
struct FftLen {
  int n;
  int nstage;
  int radix[8];
  int tw_off;
  int st_off[8];   // stage twiddles (complex), relative to the length's block
  int ob_off[8];   // stage output bases (int), relative to the length's block
  int nst;         // complex entries of all stage twiddles of this length
  int nob;         // ints of all stage output bases of this length
};

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
