// Register-resident FFTs of compile-time length for one line per thread.
//
// A length-N transform x[OFF + STR*j], j < N, of a register array is built by
// template recursion (decimation in time): N = R*M with R the first of the
// leaf radices 4, 3, 5, 7, 2 that divides N; the R sub-transforms of length M
// run in place on the strided subsets, then each output group k < M is
// twiddled by w_N^{r k} and put through an R-point leaf DFT.  Every index and
// twiddle is a compile-time constant, so the array stays in registers and the
// twiddles are immediates.  Outputs are left in digit-permuted positions:
// X[j] sits at position OFF + STR*out_pos<N>(j) (out_pos is a constexpr
// function), which callers use to address the result.
//
// Twiddles come from cos/sin evaluated at compile time by their Taylor series
// (argument reduced to [-pi/4, pi/4] by octant symmetry), accurate to double
// rounding and then rounded to the working precision.
#pragma once
#include <cuda_runtime.h>

#define QX_HD __host__ __device__ __forceinline__

namespace qx {
namespace rf {

constexpr double PI = 3.14159265358979323846264338327950288;

constexpr double cabs(double x) { return x < 0 ? -x : x; }
// Series terms are added until they drop below 1e-20 of the sum (|x| <= pi/4),
// which also keeps the compile-time evaluation clear of underflow.
constexpr double taylor_sin(double x) {
  double t = x, s = x;
  for (int n = 1; n < 14 && cabs(t) > 1e-20 * cabs(s); ++n) {
    t *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
    s += t;
  }
  return s;
}
constexpr double taylor_cos(double x) {
  double t = 1.0, s = 1.0;
  for (int n = 1; n < 14 && cabs(t) > 1e-20; ++n) {
    t *= -x * x / ((2.0 * n - 1.0) * (2.0 * n));
    s += t;
  }
  return s;
}
// cos and sin of 2*pi*p/q for integers 0 <= p < q, by octant reduction.
constexpr double cos2pi(long p, long q) {
  p %= q;
  if (p < 0) p += q;
  // angle = 2 pi p / q; octant o = floor(8 p / q)
  const long o = (8 * p) / q;
  const double a = 2.0 * PI * (double)p / (double)q;
  switch (o) {
    case 0: return taylor_cos(a);
    case 1: return taylor_sin(PI / 2 - a);
    case 2: return -taylor_sin(a - PI / 2);
    case 3: return -taylor_cos(PI - a);
    case 4: return -taylor_cos(a - PI);
    case 5: return -taylor_sin(3 * PI / 2 - a);
    case 6: return taylor_sin(a - 3 * PI / 2);
    default: return taylor_cos(2 * PI - a);
  }
}
constexpr double sin2pi(long p, long q) { return cos2pi(p * 4 - q, 4 * q); }   // sin t = cos(t - pi/2)

constexpr int leaf_radix(int n) {
  return (n % 4 == 0) ? 4 : (n % 3 == 0) ? 3 : (n % 5 == 0) ? 5 : (n % 7 == 0) ? 7 : (n % 2 == 0) ? 2 : n;
}
// Position (relative to the transform's base, in units of its stride) of
// output j of a length-n transform.
constexpr int out_pos(int n, int j) {
  if (n == 1) return 0;
  const int r = leaf_radix(n), m = n / r;
  const int k = j % m, q = j / m;
  return q + r * out_pos(m, k);
}

// Compile-time loop: f(IC<I>{}) for I = B .. E-1, so that loop indices can
// feed constant expressions (register-array subscripts through out_pos).
template <int I> struct IC { static constexpr int value = I; };
template <int B, int E, typename F> QX_HD void static_for(F &&f) {
  if constexpr (B < E) {
    f(IC<B>{});
    static_for<B + 1, E>(f);
  }
}

template <typename T> struct C2;
template <> struct C2<float> { typedef float2 t; };
template <> struct C2<double> { typedef double2 t; };

template <typename C> QX_HD C add(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> QX_HD C sub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
#if defined(__CUDA_ARCH__)
// FP32 pairs on the packed two-wide FP32 unit of sm_100: one instruction for
// both components (a - b as a + (-1) b, exact like the subtraction).
template <> __device__ __forceinline__ float2 add<float2>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 sub<float2>(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}
#endif

// x * exp(SIGN * 2 pi i p / q) with a compile-time root.
template <typename T, int SIGN, long P, long Q>
QX_HD typename C2<T>::t twiddle(typename C2<T>::t x) {
  if constexpr (P % Q == 0) {
    return x;
  } else {
    constexpr T c = (T)cos2pi(P, Q), s = (T)(SIGN * sin2pi(P, Q));
    typename C2<T>::t r;
    r.x = x.x * c - x.y * s;
    r.y = x.x * s + x.y * c;
    return r;
  }
}

// In-place R-point DFT of v[0..R) (natural order in and out).
template <typename T, int SIGN, int R> struct Leaf;

template <typename T, int SIGN> struct Leaf<T, SIGN, 2> {
  template <typename C> static QX_HD void run(C *v) {
    const C a = v[0], b = v[1];
    v[0] = add(a, b);
    v[1] = sub(a, b);
  }
};
template <typename T, int SIGN> struct Leaf<T, SIGN, 4> {
  template <typename C> static QX_HD void run(C *v) {
    const C s0 = add(v[0], v[2]), d0 = sub(v[0], v[2]);
    const C s1 = add(v[1], v[3]), d1 = sub(v[1], v[3]);
    C jd;   // SIGN * i * d1
    if (SIGN < 0) { jd.x = d1.y; jd.y = -d1.x; } else { jd.x = -d1.y; jd.y = d1.x; }
    v[0] = add(s0, s1);
    v[2] = sub(s0, s1);
    v[1] = add(d0, jd);
    v[3] = sub(d0, jd);
  }
};
template <typename T, int SIGN> struct Leaf<T, SIGN, 3> {
  template <typename C> static QX_HD void run(C *v) {
    constexpr T h = (T)0.86602540378443864676 * (T)SIGN;   // SIGN * sqrt(3)/2
    const C t1 = add(v[1], v[2]), d = sub(v[1], v[2]);
    C t2;
    t2.x = v[0].x - (T)0.5 * t1.x;
    t2.y = v[0].y - (T)0.5 * t1.y;
    C jd;   // SIGN * i * sqrt(3)/2 * d
    jd.x = -h * d.y;
    jd.y = h * d.x;
    v[0] = add(v[0], t1);
    v[1] = add(t2, jd);
    v[2] = sub(t2, jd);
  }
};
// Prime radices 5 and 7: direct sums with compile-time roots, pairing the
// conjugate-symmetric terms: with s_a = v_a + v_{R-a}, d_a = v_a - v_{R-a},
// X_q = v_0 + sum_a [cos(2 pi a q / R) s_a + i SIGN sin(2 pi a q / R) d_a]
// and X_{R-q} the same with the imaginary term negated.
template <typename T, int SIGN, int R, int Q, int A, typename C>
QX_HD void prime_acc(C &re, C &im, const C *s, const C *d) {
  if constexpr (A <= (R - 1) / 2) {
    constexpr T c = (T)cos2pi((long)A * Q, R), sn = (T)(SIGN * sin2pi((long)A * Q, R));
    re.x += c * s[A - 1].x;
    re.y += c * s[A - 1].y;
    im.x -= sn * d[A - 1].y;
    im.y += sn * d[A - 1].x;
    prime_acc<T, SIGN, R, Q, A + 1>(re, im, s, d);
  }
}
template <typename T, int SIGN, int R, int Q, typename C>
QX_HD void prime_out(const C &v0, const C *s, const C *d, C *o) {
  if constexpr (Q <= (R - 1) / 2) {
    C re = v0, im;
    im.x = 0;
    im.y = 0;
    prime_acc<T, SIGN, R, Q, 1>(re, im, s, d);
    o[Q] = add(re, im);
    o[R - Q] = sub(re, im);
    prime_out<T, SIGN, R, Q + 1>(v0, s, d, o);
  }
}
template <typename T, int SIGN, int R> struct LeafPrime {
  template <typename C> static QX_HD void run(C *v) {
    C o[R];
    C s[(R - 1) / 2], d[(R - 1) / 2];
#pragma unroll
    for (int a = 1; a <= (R - 1) / 2; ++a) { s[a - 1] = add(v[a], v[R - a]); d[a - 1] = sub(v[a], v[R - a]); }
    o[0] = v[0];
#pragma unroll
    for (int a = 0; a < (R - 1) / 2; ++a) o[0] = add(o[0], s[a]);
    prime_out<T, SIGN, R, 1>(v[0], s, d, o);
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = o[q];
  }
};
template <typename T, int SIGN> struct Leaf<T, SIGN, 5> : LeafPrime<T, SIGN, 5> {};
template <typename T, int SIGN> struct Leaf<T, SIGN, 7> : LeafPrime<T, SIGN, 7> {};

// Combine step for output group k (template recursion over k).
template <typename T, int SIGN, int N, int OFF, int STR, int TOT, int K>
QX_HD void combine(typename C2<T>::t (&x)[TOT]) {
  constexpr int R = leaf_radix(N), M = N / R;
  if constexpr (K < M) {
    constexpr int PK = out_pos(M, K);
    typename C2<T>::t v[R];
    // v[r] = X_r[K] * w_N^{r K}; X_r[K] at OFF + STR*(r + R*PK)
    if constexpr (R >= 1) v[0] = x[OFF + STR * (0 + R * PK)];
    if constexpr (R >= 2) v[1] = twiddle<T, SIGN, 1L * K, N>(x[OFF + STR * (1 + R * PK)]);
    if constexpr (R >= 3) v[2] = twiddle<T, SIGN, 2L * K, N>(x[OFF + STR * (2 + R * PK)]);
    if constexpr (R >= 4) v[3] = twiddle<T, SIGN, 3L * K, N>(x[OFF + STR * (3 + R * PK)]);
    if constexpr (R >= 5) v[4] = twiddle<T, SIGN, 4L * K, N>(x[OFF + STR * (4 + R * PK)]);
    if constexpr (R >= 6) v[5] = twiddle<T, SIGN, 5L * K, N>(x[OFF + STR * (5 + R * PK)]);
    if constexpr (R >= 7) v[6] = twiddle<T, SIGN, 6L * K, N>(x[OFF + STR * (6 + R * PK)]);
    Leaf<T, SIGN, R>::run(v);
    // X[K + q M] -> position q + R*PK
#pragma unroll
    for (int q = 0; q < R; ++q) x[OFF + STR * (q + R * PK)] = v[q];
    combine<T, SIGN, N, OFF, STR, TOT, K + 1>(x);
  }
}

template <typename T, int SIGN, int N, int OFF, int STR, int TOT>
QX_HD void rfft(typename C2<T>::t (&x)[TOT]);

template <typename T, int SIGN, int N, int OFF, int STR, int TOT, int Rr>
QX_HD void subffts(typename C2<T>::t (&x)[TOT]) {
  constexpr int R = leaf_radix(N), M = N / R;
  if constexpr (Rr < R) {
    rfft<T, SIGN, M, OFF + STR * Rr, STR * R, TOT>(x);
    subffts<T, SIGN, N, OFF, STR, TOT, Rr + 1>(x);
  }
}

template <typename T, int SIGN, int N, int OFF, int STR, int TOT>
QX_HD void rfft(typename C2<T>::t (&x)[TOT]) {
  static_assert(leaf_radix(N) <= 7, "lengths must be products of 2, 3, 5, 7");
  if constexpr (N > 1) {
    subffts<T, SIGN, N, OFF, STR, TOT, 0>(x);
    combine<T, SIGN, N, OFF, STR, TOT, 0>(x);
  }
}

// Unscaled transform of x[0..N): X[k] = sum_j x[j] exp(SIGN 2 pi i j k / N),
// result at positions out_pos(N, k).
template <typename T, int SIGN, int N>
QX_HD void fft(typename C2<T>::t (&x)[N]) {
  rfft<T, SIGN, N, 0, 1, N>(x);
}

}  // namespace rf
}  // namespace qx
