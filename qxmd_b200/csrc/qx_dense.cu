// FP64 dense kernels on the nb x nb band matrices: Cholesky + triangular
// inverse (rsdecmp/rsinvcd, schmidt.f90:428-544) and the symmetric
// eigen-decomposition of the subspace Hamiltonian (the role of RsEIGQR,
// funcs.f90:380, called from untryt2, eigen.f90:1237) by parallel cyclic
// Jacobi.  Each runs as one CTA; matrices live in shared memory when they fit
// and in global memory (L2) otherwise.  No wait in these kernels depends on
// another block.
#include <algorithm>

#include "qx_internal.h"

namespace qx {

constexpr int DT = 1024;
constexpr size_t JSMEM_MAX_CH = 220 * 1024;

// Column-major n x n.  info: 0 ok, 1+i if pivot i <= 1e-30.
// rsdecmp order (left-looking: column i from columns < i) and rsinvcd order
// (in place, columns from the right); each row's dot product is a warp
// reduction, rows spread over the warps.
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(DT) k_cholinv(double *__restrict__ Sg, int n, int *__restrict__ info, int use_smem) {
  extern __shared__ double sm[];
  __shared__ double dsh;
  __shared__ int bad;
  // shared copy with an odd leading dimension: row and column walks are
  // both free of bank conflicts
  const int ld = use_smem ? (n | 1) : n;
  double *S = use_smem ? sm : Sg;
  double *w = sm + (use_smem ? (long)ld * n : 0);   // n doubles of row results
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (use_smem)
    for (long e = threadIdx.x; e < (long)n * n; e += blockDim.x) {
      const int j = (int)(e / n), i = (int)(e - (long)j * n);
      S[(long)j * ld + i] = Sg[e];
    }
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
#define S_(i, j) S[(long)(j) * ld + (i)]
  for (int i = 0; i < n; ++i) {
    if (warp == 0) {
      double p = 0.0;
      for (int k = lane; k < i; k += 32) p += S_(i, k) * S_(i, k);
      p = warp_sum(p);
      if (lane == 0) {
        const double d = S_(i, i) - p;
        if (d > 1.0e-30) dsh = sqrt(d);
        else { dsh = 0.0; if (!bad) bad = 1 + i; }
      }
    }
    __syncthreads();
    const double d = dsh;
    if (d == 0.0) break;
    const double r = 1.0 / d;
    for (int j = i + 1 + warp; j < n; j += nw) {
      double p = 0.0;
      for (int k = lane; k < i; k += 32) p += S_(j, k) * S_(i, k);
      p = warp_sum(p);
      if (lane == 0) S_(j, i) = (S_(j, i) - p) * r;
    }
    if (threadIdx.x == 0) S_(i, i) = d;
    __syncthreads();
  }
  if (bad) {
    if (threadIdx.x == 0) *info = bad;
    return;
  }
  for (long e = threadIdx.x; e < (long)n * n; e += blockDim.x) {
    const int j = (int)(e / n), i = (int)(e - (long)j * n);
    if (i > j) S_(i, j) = S_(i, j) * (1.0 / S_(j, j));
    else if (i < j) S_(i, j) = 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) S_(i, i) = 1.0 / S_(i, i);
  __syncthreads();
  // column j of L^-1 from the finished columns k > j:
  // S(i,j) = -sum_{k=j+1..i} X(i,k) M(k,j); all reads of column j finish
  // before it is overwritten.
  for (int j = n - 2; j >= 0; --j) {
    for (int i = j + 1 + warp; i < n; i += nw) {
      double p = 0.0;
      for (int k = j + 1 + lane; k <= i; k += 32) p += S_(i, k) * S_(k, j);
      p = warp_sum(p);
      if (lane == 0) w[i] = p;
    }
    __syncthreads();
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) S_(i, j) = -w[i];
    __syncthreads();
  }
#undef S_
  if (use_smem)
    for (long e = threadIdx.x; e < (long)n * n; e += blockDim.x) {
      const int j = (int)(e / n), i = (int)(e - (long)j * n);
      Sg[e] = S[(long)j * ld + i];
    }
  if (threadIdx.x == 0) *info = 0;
}

int cholinv(double *S, int n, int *d_info, cudaStream_t st) {
  if (n > 8192) { set_error("cholinv: n=%d too large", n); return 1; }
  const size_t bytes = sizeof(double) * ((size_t)(n | 1) * n + n);
  const int use = bytes <= JSMEM_MAX_CH;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_cholinv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)JSMEM_MAX_CH);
    attr = true;
  }
  k_cholinv<<<1, DT, use ? bytes : sizeof(double) * n, st>>>(S, n, d_info, use); note_launch();
  return 0;
}

// --------------------------------------------------------------------------
// Symmetric eigen-decomposition of the subspace Hamiltonian (the role of
// RsEIGQR, funcs.f90:380-764, which also reduces to tridiagonal form by
// Householder reflections): (1) Householder tridiagonalisation T = Q^T A Q
// in one CTA, A in shared memory with an odd leading dimension when it fits;
// (2) eigenvalues of T by Sturm-count bisection, one thread per eigenvalue;
// (3) eigenvectors of T by inverse iteration with a pivoted tridiagonal LU,
// one thread per cluster of close eigenvalues, members re-orthogonalised
// against each other (modified Gram-Schmidt); (4) V = Q Z by applying the
// reflectors, columns spread over CTAs.  Eigenpairs are ascending; each
// eigenvector's largest-magnitude component is made positive (first index on
// ties).  Every loop is bounded.

constexpr int TRD_T = 1024;

// Householder reflector of x (GVL house): P = I - tau v v^T, v(0) = 1,
// P x = |x| e1.  Returns tau, writes beta (v = x / beta for i >= 1) and |x|.
__device__ __forceinline__ void house(double x0, double sigma, double &tau, double &beta, double &alpha) {
  if (sigma == 0.0) {
    tau = (x0 < 0.0) ? 2.0 : 0.0;
    beta = 1.0;
    alpha = fabs(x0);
    return;
  }
  const double mu = sqrt(x0 * x0 + sigma);
  const double v1 = (x0 <= 0.0) ? x0 - mu : -sigma / (x0 + mu);
  tau = 2.0 * v1 * v1 / (sigma + v1 * v1);
  beta = v1;
  alpha = mu;
}

__global__ void __launch_bounds__(TRD_T) k_sytrd(double *__restrict__ Ag, int n, double *__restrict__ d,
                                                 double *__restrict__ e, double *__restrict__ HV,
                                                 double *__restrict__ tau, int use_smem) {
  extern __shared__ double sm[];
  __shared__ double sc[4];
  const int ld = use_smem ? (n | 1) : n;
  double *A = use_smem ? sm : Ag;
  double *v = sm + (use_smem ? (long)ld * n : 0);
  double *p = v + n;
  double *part = p + n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (use_smem)
    for (long q = threadIdx.x; q < (long)n * n; q += blockDim.x) {
      const int j = (int)(q / n), i = (int)(q - (long)j * n);
      A[(long)j * ld + i] = Ag[q];
    }
  __syncthreads();
#define A_(i, j) A[(long)(j) * ld + (i)]
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;
    if (warp == 0) {
      double sg = 0.0;
      for (int i = 1 + lane; i < m; i += 32) { const double x = A_(k + 1 + i, k); sg += x * x; }
      for (int o = 16; o > 0; o >>= 1) sg += __shfl_xor_sync(0xffffffffu, sg, o);
      if (lane == 0) {
        double t, be, al;
        house(A_(k + 1, k), sg, t, be, al);
        sc[0] = t; sc[1] = be; sc[2] = al;
      }
    }
    __syncthreads();
    const double tk = sc[0], be = sc[1];
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      const double vi = (i == 0) ? 1.0 : ((tk != 0.0) ? A_(k + 1 + i, k) / be : 0.0);
      v[i] = vi;
      HV[(long)k * n + k + 1 + i] = vi;
    }
    if (threadIdx.x == 0) {
      tau[k] = tk;
      d[k] = A_(k, k);
      e[k] = sc[2];
    }
    __syncthreads();
    if (tk != 0.0) {
      // p = tau * B v, B = A(k+1:, k+1:); rows split over G groups of columns
      const int G = max(1, (int)blockDim.x / m);
      {
        const int i = threadIdx.x % m, g = threadIdx.x / m;
        if (g < G) {
          double s2 = 0.0;
          for (int j = g; j < m; j += G) s2 += A_(k + 1 + i, k + 1 + j) * v[j];
          part[g * m + i] = s2;
        }
      }
      __syncthreads();
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        double s2 = 0.0;
        for (int g = 0; g < G; ++g) s2 += part[g * m + i];
        p[i] = tk * s2;
      }
      __syncthreads();
      if (warp == 0) {
        double kk = 0.0;
        for (int i = lane; i < m; i += 32) kk += v[i] * p[i];
        for (int o = 16; o > 0; o >>= 1) kk += __shfl_xor_sync(0xffffffffu, kk, o);
        if (lane == 0) sc[3] = 0.5 * tk * kk;
      }
      __syncthreads();
      const double K = sc[3];
      for (int i = threadIdx.x; i < m; i += blockDim.x) p[i] -= K * v[i];
      __syncthreads();
      for (long q = threadIdx.x; q < (long)m * m; q += blockDim.x) {
        const int j = (int)(q / m), i = (int)(q - (long)j * m);
        A_(k + 1 + i, k + 1 + j) -= v[i] * p[j] + p[i] * v[j];
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (n >= 2) {
      d[n - 2] = A_(n - 2, n - 2);
      e[n - 2] = A_(n - 1, n - 2);
    }
    d[n - 1] = A_(n - 1, n - 1);
  }
#undef A_
}

// Number of eigenvalues of T below x (Sturm count, pivots guarded by pmin).
__device__ __forceinline__ int sturm(const double *d, const double *e2, int n, double x, double pmin) {
  int c = 0;
  double q = d[0] - x;
  if (fabs(q) < pmin) q = -pmin;
  if (q < 0.0) ++c;
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (fabs(q) < pmin) q = -pmin;
    if (q < 0.0) ++c;
  }
  return c;
}

// k-th smallest eigenvalue of T by bisection to 2 eps |T| (at most 200 halvings).
__global__ void k_bisect(const double *__restrict__ d, const double *__restrict__ e, int n, double *__restrict__ w,
                         double *__restrict__ e2buf) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  for (int i = threadIdx.x; i < n - 1; i += blockDim.x) e2buf[i] = e[i] * e[i];
  __syncthreads();   // every block writes the same e^2 values; its own threads read them
  if (t >= n) return;
  double lo = d[0], hi = d[0], tn = 0.0;
  for (int i = 0; i < n; ++i) {
    const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
    tn = fmax(tn, fabs(d[i]) + r);
  }
  const double eps = 2.220446049250313e-16;
  const double pmin = 1e-300 + eps * eps * tn * tn * 1e-10;
  lo -= 2.0 * eps * tn + 1e-300;
  hi += 2.0 * eps * tn + 1e-300;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (hi - lo <= 2.0 * eps * tn + 4.0 * pmin || mid == lo || mid == hi) break;
    if (sturm(d, e2buf, n, mid, pmin) > t) hi = mid;
    else lo = mid;
  }
  w[t] = 0.5 * (lo + hi);
}

// Inverse iteration on T for the eigenvalues of one cluster (consecutive
// eigenvalues closer than 1e-6 |T|), members orthogonalised against the
// earlier ones.  Thread t is active if eigenvalue t starts a cluster.
// ws: per thread 5*n doubles (LU factors).  Z(:, t) = eigenvector t of T.
__global__ void k_invit(const double *__restrict__ d, const double *__restrict__ e, const double *__restrict__ w,
                        int n, double *__restrict__ Z, double *__restrict__ ws, int *__restrict__ nclus) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double tn = 0.0;
  for (int i = 0; i < n; ++i)
    tn = fmax(tn, fabs(d[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0));
  const double eps = 2.220446049250313e-16;
  const double gaptol = 1e-6 * tn;
  if (t > 0 && w[t] - w[t - 1] < gaptol) return;   // not a cluster head
  atomicAdd(nclus, 1);
  int tend = t + 1;
  while (tend < n && w[tend] - w[tend - 1] < gaptol) ++tend;
  double *u0 = ws + (long)t * 5 * n, *u1 = u0 + n, *u2 = u1 + n, *lm = u2 + n, *pv = lm + n;
  const double tiny = eps * tn + 1e-300;
  for (int c = t; c < tend; ++c) {
    // perturb members apart so their LU factors differ
    const double lam = w[c] + (double)(c - t) * 4.0 * eps * tn;
    // LU with partial pivoting of T - lam I (rows i, i+1 may swap)
    // u0: diagonal of U, u1: first superdiagonal, u2: second, lm: multipliers, pv: swapped flag
    double a = d[0] - lam, b = (n > 1) ? e[0] : 0.0;
    for (int i = 0; i < n - 1; ++i) {
      const double cdn = e[i];                 // subdiagonal below a
      const double dn = d[i + 1] - lam;        // next diagonal
      const double en = (i + 1 < n - 1) ? e[i + 1] : 0.0;
      if (fabs(a) >= fabs(cdn)) {
        const double aa = (fabs(a) < tiny) ? tiny : a;
        const double l = cdn / aa;
        u0[i] = aa; u1[i] = b; u2[i] = 0.0; lm[i] = l; pv[i] = 0.0;
        a = dn - l * b;
        b = en;
      } else {
        const double l = a / cdn;
        u0[i] = cdn; u1[i] = dn; u2[i] = en; lm[i] = l; pv[i] = 1.0;
        a = b - l * dn;
        b = -l * en;
      }
    }
    u0[n - 1] = (fabs(a) < tiny) ? tiny : a;
    // start vector: ones with a member-dependent sign pattern
    double *z = Z + (long)c * n;
    for (int i = 0; i < n; ++i) z[i] = 1.0 + 0.01 * (double)((i * (c + 3)) % 7);
    for (int it = 0; it < 4; ++it) {
      // forward: apply the row interchanges and multipliers
      for (int i = 0; i < n - 1; ++i) {
        if (pv[i] != 0.0) { const double tmp = z[i]; z[i] = z[i + 1]; z[i + 1] = tmp - lm[i] * z[i]; }
        else z[i + 1] -= lm[i] * z[i];
      }
      // back substitution with U (two superdiagonals)
      z[n - 1] /= u0[n - 1];
      if (n > 1) z[n - 2] = (z[n - 2] - u1[n - 2] * z[n - 1]) / u0[n - 2];
      for (int i = n - 3; i >= 0; --i) z[i] = (z[i] - u1[i] * z[i + 1] - u2[i] * z[i + 2]) / u0[i];
      // orthogonalise against the earlier members of the cluster
      for (int q = t; q < c; ++q) {
        const double *zq = Z + (long)q * n;
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += zq[i] * z[i];
        for (int i = 0; i < n; ++i) z[i] -= s * zq[i];
      }
      double nr = 0.0;
      for (int i = 0; i < n; ++i) nr += z[i] * z[i];
      nr = 1.0 / sqrt(nr);
      for (int i = 0; i < n; ++i) z[i] *= nr;
    }
  }
}

// V(:, cols) = Q Z(:, cols): reflectors k = n-3 .. 0 applied to a block of
// columns held in shared memory; then the sign convention.
__global__ void __launch_bounds__(256) k_backtrans(const double *__restrict__ Z, const double *__restrict__ HV,
                                                   const double *__restrict__ tau, int n, int cols,
                                                   double *__restrict__ V) {
  extern __shared__ double zb[];   // n x cols, column-major
  __shared__ double wsum[32];
  const int c0 = blockIdx.x * cols;
  const int nc = min(cols, n - c0);
  for (int q = threadIdx.x; q < n * nc; q += blockDim.x) zb[q] = Z[(long)c0 * n + q];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = n - 3; k >= 0; --k) {
    const double tk = tau[k];
    if (tk == 0.0) continue;   // uniform across the block
    const double *v = HV + (long)k * n;   // v at rows k+1 .. n-1
    // w_c = v^T z_c, one warp per column
    for (int c = warp; c < nc; c += nw) {
      double s = 0.0;
      for (int i = k + 1 + lane; i < n; i += 32) s += v[i] * zb[c * n + i];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) wsum[c] = tk * s;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n * nc; q += blockDim.x) {
      const int c = q / n, i = q - c * n;
      if (i > k) zb[q] -= v[i] * wsum[c];
    }
    __syncthreads();
  }
  // largest-magnitude component positive, write out
  for (int c = warp; c < nc; c += nw) {
    double mx = -1.0;
    int km = 0;
    for (int i = lane; i < n; i += 32) {
      const double a = fabs(zb[c * n + i]);
      if (a > mx) { mx = a; km = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double m2 = __shfl_xor_sync(0xffffffffu, mx, o);
      const int k2 = __shfl_xor_sync(0xffffffffu, km, o);
      if (m2 > mx || (m2 == mx && k2 < km)) { mx = m2; km = k2; }
    }
    const double sg = zb[c * n + km] < 0.0 ? -1.0 : 1.0;
    for (int i = lane; i < n; i += 32) V[(long)(c0 + c) * n + i] = sg * zb[c * n + i];
  }
}

constexpr size_t TRD_SMEM_MAX = 222 * 1024;

// A (n x n, destroyed), w (n) eigenvalues ascending, V (n x n) eigenvectors.
// work: at least 8*n*n + 16*n doubles.  info: number of eigenvalue clusters.
int syev(double *A, int n, double *w, double *V, double *work, int *d_info, cudaStream_t st) {
  if (n < 1) { set_error("syev: n=%d", n); return 1; }
  double *d = work, *e = d + n, *tau = e + n, *e2 = tau + n, *HV = e2 + n, *Z = HV + (long)n * n,
         *lu = Z + (long)n * n;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_sytrd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRD_SMEM_MAX);
    cudaFuncSetAttribute(k_backtrans, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    attr = true;
  }
  const size_t vec = sizeof(double) * (2 * (size_t)n + TRD_T);
  const size_t mat = sizeof(double) * (size_t)(n | 1) * n;
  const int use = mat + vec <= TRD_SMEM_MAX;
  cudaMemsetAsync(HV, 0, sizeof(double) * (size_t)n * n, st);
  cudaMemsetAsync(d_info, 0, sizeof(int), st);
  k_sytrd<<<1, TRD_T, use ? mat + vec : vec, st>>>(A, n, d, e, HV, tau, use); note_launch();
  if (n == 1) {
    cudaMemcpyAsync(w, d, sizeof(double), cudaMemcpyDeviceToDevice, st);
    const double one = 1.0;
    cudaMemcpyAsync(V, &one, sizeof(double), cudaMemcpyHostToDevice, st);
    return 0;
  }
  const int tb = 128, nbk = (n + tb - 1) / tb;
  k_bisect<<<nbk, tb, 0, st>>>(d, e, n, w, e2); note_launch();
  k_invit<<<nbk, tb, 0, st>>>(d, e, w, n, Z, lu, d_info); note_launch();
  const int cols = std::max(1, std::min(32, (int)(48 * 1024 / (sizeof(double) * n))));
  k_backtrans<<<(n + cols - 1) / cols, 256, sizeof(double) * (size_t)n * cols, st>>>(Z, HV, tau, n, cols, V);
  note_launch();
  return 0;
}

// --------------------------------------------------------------------------
template <typename Tin, typename Tout>
__global__ void k_convert(const Tin *__restrict__ in, Tout *__restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = (Tout)in[i];
}

template <typename Tin, typename Tout>
void convert(const Tin *in, Tout *out, long n, cudaStream_t st) {
  if (n <= 0) return;
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_convert<Tin, Tout><<<blocks, 256, 0, st>>>(in, out, n); note_launch();
}
template void convert<float, double>(const float *, double *, long, cudaStream_t);
template void convert<double, float>(const double *, float *, long, cudaStream_t);
template void convert<double, double>(const double *, double *, long, cudaStream_t);
template void convert<float, float>(const float *, float *, long, cudaStream_t);

// out(j,i) = out(i,j) = in(j,i) for j <= i (the lower triangle of the
// column-major product in, as hmatrix2 fills it, engrad.f90:869-895).
template <typename T>
__global__ void k_symmetrize(const T *__restrict__ in, double *__restrict__ out, double *__restrict__ diag, int n) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= (long)n * n) return;
  const int i = (int)(e / n), j = (int)(e - (long)i * n);   // column i, row j
  const int lo = j < i ? j : i, hi = j < i ? i : j;
  const double v = (double)in[(long)hi * n + lo];             // row lo, column hi: <c_lo|hc_hi>
  out[e] = v;
  if (i == j && diag) diag[i] = v;
}

template <typename T>
void symmetrize_lower(const T *in, double *out, double *diag, int n, cudaStream_t st) {
  const long nn = (long)n * n;
  k_symmetrize<T><<<(int)((nn + 255) / 256), 256, 0, st>>>(in, out, diag, n); note_launch();
}
template void symmetrize_lower<float>(const float *, double *, double *, int, cudaStream_t);
template void symmetrize_lower<double>(const double *, double *, double *, int, cudaStream_t);

}  // namespace qx
