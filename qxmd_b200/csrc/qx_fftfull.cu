// Full-grid FP64 transforms of the density side (rfft3/fft3 drop-in, the
// passes of launch_full_fft) for lines of at most 32 points: one grid line
// per thread with the whole line in registers (compile-time-length FFTs of
// qx_regfft.cuh, twiddles exact to double rounding).  In the z and y passes
// thread t takes the line at i1 = t mod k1, so consecutive threads read and
// write consecutive 16-byte elements of every plane they cross; in the x
// pass each thread walks its own contiguous line.
#include "qx_internal.h"
#include "qx_regfft.cuh"

namespace qx {

constexpr int FL_T = 128;

// AXIS 2: lines along z (i3), one per (i1, i2); AXIS 1: along y (i2), one per
// (i1, i3); AXIS 0: along x (i1), one per (i2, i3), each thread reading its
// own contiguous line, and the result times scale (the last pass).
// g[(i3 k2 + i2) k1 + i1], in place.
template <int N, int SIGN, int AXIS>
__global__ void __launch_bounds__(FL_T) k_full_lines(double2 *__restrict__ g, int k1, int k2, int k3, double scale) {
  using rf::out_pos;
  const long t = blockIdx.x * (long)FL_T + threadIdx.x;
  const long nlines = AXIS == 0 ? (long)k2 * k3 : (long)k1 * (AXIS == 2 ? k2 : k3);
  if (t >= nlines) return;
  long stride;
  double2 *base;
  if (AXIS == 0) {
    stride = 1;
    base = g + t * k1;
  } else {
    const int i1 = (int)(t % k1), o = (int)(t / k1);
    stride = AXIS == 2 ? (long)k1 * k2 : (long)k1;
    base = g + (AXIS == 2 ? (long)o * k1 + i1 : (long)o * k2 * k1 + i1);
  }
  double2 x[N];
#pragma unroll
  for (int i = 0; i < N; ++i) x[i] = base[i * stride];
  rf::fft<double, SIGN, N>(x);
  rf::static_for<0, N>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    double2 z = x[out_pos(N, i)];
    if (AXIS == 0) {
      z.x *= scale;
      z.y *= scale;
    }
    base[i * stride] = z;
  });
}

template <int N>
static void full_lines_go(double2 *g, int k1, int k2, int k3, int axis, int sign, double scale, cudaStream_t st) {
  const long nl = axis == 0 ? (long)k2 * k3 : (long)k1 * (axis == 2 ? k2 : k3);
  const int blocks = (int)((nl + FL_T - 1) / FL_T);
  if (axis == 2) {
    if (sign > 0) k_full_lines<N, +1, 2><<<blocks, FL_T, 0, st>>>(g, k1, k2, k3, 1.0);
    else k_full_lines<N, -1, 2><<<blocks, FL_T, 0, st>>>(g, k1, k2, k3, 1.0);
  } else if (axis == 1) {
    if (sign > 0) k_full_lines<N, +1, 1><<<blocks, FL_T, 0, st>>>(g, k1, k2, k3, 1.0);
    else k_full_lines<N, -1, 1><<<blocks, FL_T, 0, st>>>(g, k1, k2, k3, 1.0);
  } else {
    if (sign > 0) k_full_lines<N, +1, 0><<<blocks, FL_T, 0, st>>>(g, k1, k2, k3, scale);
    else k_full_lines<N, -1, 0><<<blocks, FL_T, 0, st>>>(g, k1, k2, k3, scale);
  }
  note_launch();
}

// QX_FULL_LINES=0 keeps every pass on the shared-memory kernels (read at
// every call).
static bool full_lines_enabled() {
  const char *e = getenv("QX_FULL_LINES");
  return !(e && e[0] == '0');
}

int launch_full_lines_f64(double2 *g, int k1, int k2, int k3, int axis, int sign, double scale, cudaStream_t st) {
  if (!full_lines_enabled() || axis < 0 || axis > 2) return -1;
  switch (axis == 2 ? k3 : axis == 1 ? k2 : k1) {
    case 20: full_lines_go<20>(g, k1, k2, k3, axis, sign, scale, st); return 0;
    case 21: full_lines_go<21>(g, k1, k2, k3, axis, sign, scale, st); return 0;
    case 24: full_lines_go<24>(g, k1, k2, k3, axis, sign, scale, st); return 0;
    case 25: full_lines_go<25>(g, k1, k2, k3, axis, sign, scale, st); return 0;
    case 27: full_lines_go<27>(g, k1, k2, k3, axis, sign, scale, st); return 0;
    case 30: full_lines_go<30>(g, k1, k2, k3, axis, sign, scale, st); return 0;
    case 32: full_lines_go<32>(g, k1, k2, k3, axis, sign, scale, st); return 0;
    default: return -1;
  }
}

}  // namespace qx
