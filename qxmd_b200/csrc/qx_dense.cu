// FP64 dense kernels on the nb x nb band matrices: Cholesky + triangular
// inverse (rsdecmp/rsinvcd, schmidt.f90:428-544) and the symmetric
// eigen-decomposition of the subspace Hamiltonian (the role of RsEIGQR,
// funcs.f90:380, called from untryt2, eigen.f90:1237).
//
// At nb of a few hundred these are latency problems, not flop problems, so
// every kernel is shaped to shorten the chain of dependent steps: 32-wide
// blocks factored inside one warp, panel and trailing updates spread over
// the CTA, one warp per eigenvalue for multisection, one warp per column for
// the back-transformation.  Matrices live in shared memory (odd leading
// dimension) when they fit and in global memory (L2) otherwise.  No wait in
// these kernels depends on another block.
#include <algorithm>

#include "qx_internal.h"

namespace qx {

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// --------------------------------------------------------------------------
// Cholesky S = L L^T and L^-1, blocked by CB = 32.  Column-major n x n; on
// return the lower triangle holds L^-1 and the upper triangle zeros.
// info: 0, or 1+i for the first row i whose pivot (the Schur-complement
// diagonal S(i,i) - sum_k L(i,k)^2 that rsdecmp tests) is not > 1e-30
// (schmidt.f90:256-267).
constexpr int CB = 32;
constexpr int CHT = 512;            // threads of k_cholinv (16 warps)
constexpr int DLD = CB + 1;         // leading dimension of the 32 x 32 temporary
constexpr size_t CH_SMEM_MAX = 220 * 1024;

// X = L^-1 of the lower-triangular bs x bs block at B (leading dimension ld),
// in place, columns right to left (X(i,j) = -sum_{k=j+1..i} X(i,k) L(k,j) /
// L(j,j)), lane = row.  Only the lower triangle is read or written.  Called
// by one whole warp.
__device__ __forceinline__ void warp_trinv(double *B, int ld, int bs, int lane) {
  for (int j = bs - 1; j >= 0; --j) {
    const double xjj = 1.0 / B[(long)j * ld + j];
    double s = 0.0;
    if (lane > j && lane < bs)
      for (int k = j + 1; k <= lane; ++k) s += B[(long)k * ld + lane] * B[(long)j * ld + k];
    __syncwarp();
    if (lane == j) B[(long)j * ld + j] = xjj;
    if (lane > j && lane < bs) B[(long)j * ld + lane] = -s * xjj;
    __syncwarp();
  }
}

__global__ void __launch_bounds__(CHT) k_cholinv(double *__restrict__ Sg, int n, double *__restrict__ work,
                                                  int *__restrict__ info, int use_smem) {
  extern __shared__ double sm[];
  __shared__ int bad;
  const int ld = use_smem ? (n | 1) : n;
  double *A = use_smem ? sm : Sg;
  double *T = use_smem ? sm + (long)ld * n : work;   // CB x DLD temporary
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = CHT / 32;
#define A_(i, j) A[(long)(j) * ld + (i)]
  if (use_smem)
    for (long q = tid; q < (long)n * n; q += CHT) {
      const int j = (int)(q / n), i = (int)(q - (long)j * n);
      A_(i, j) = Sg[q];
    }
  if (tid == 0) bad = 0;
  __syncthreads();
  const int nblk = (n + CB - 1) / CB;
  // ---- right-looking blocked Cholesky ----
  for (int J = 0; J < nblk; ++J) {
    const int j0 = J * CB, bs = min(CB, n - j0);
    if (warp == 0) {
      // diagonal block, lane = row
      for (int k = 0; k < bs; ++k) {
        const double piv = A_(j0 + k, j0 + k);
        if (!(piv > 1.0e-30)) {            // also catches NaN
          if (lane == 0) bad = 1 + j0 + k;
          break;
        }
        const double s = sqrt(piv), r = 1.0 / s;
        __syncwarp();
        if (lane > k && lane < bs) A_(j0 + lane, j0 + k) *= r;
        if (lane == k) A_(j0 + k, j0 + k) = s;
        __syncwarp();
        if (lane > k && lane < bs) {
          const double lik = A_(j0 + lane, j0 + k);
          for (int j = k + 1; j <= lane; ++j) A_(j0 + lane, j0 + j) -= lik * A_(j0 + j, j0 + k);
        }
        __syncwarp();
      }
    }
    __syncthreads();
    if (bad) break;
    const int r0 = j0 + bs, mr = n - r0;
    if (mr <= 0) break;
    // panel: L(r, j0+c) = sum_{k <= c} A(r, j0+k) Linv_JJ(c, k), Linv_JJ
    // formed in the temporary T
    if (warp == 0) {
      for (int q = lane; q < CB * CB; q += 32) {
        const int jj = q >> 5, ii = q & 31;
        T[jj * DLD + ii] = (ii >= jj && ii < bs && jj < bs) ? A_(j0 + ii, j0 + jj) : 0.0;
      }
      __syncwarp();
      warp_trinv(T, DLD, bs, lane);
    }
    __syncthreads();
    for (int r = r0 + warp; r < n; r += nw) {
      const double a = (lane < bs) ? A_(r, j0 + lane) : 0.0;
      double s = 0.0;
      for (int k = 0; k < bs; ++k) {
        const double ak = __shfl_sync(0xffffffffu, a, k);
        s += ak * ((k <= lane) ? T[k * DLD + lane] : 0.0);
      }
      __syncwarp();
      if (lane < bs) A_(r, j0 + lane) = s;
    }
    __syncthreads();
    // trailing update of the lower triangle: A(r, c) -= sum_k L(r, j0+k) L(c, j0+k)
    for (long q = tid; q < (long)mr * mr; q += CHT) {
      const int c = (int)(q / mr), r = (int)(q - (long)c * mr);
      if (r < c) continue;
      double s = 0.0;
      for (int k = 0; k < bs; ++k) s += A_(r0 + r, j0 + k) * A_(r0 + c, j0 + k);
      A_(r0 + r, r0 + c) -= s;
    }
    __syncthreads();
  }
  if (bad) {
    if (tid == 0) *info = bad;
    return;
  }
  // ---- L^-1, blocked ----
  // zero the strict upper triangle (it still holds S)
  for (long q = tid; q < (long)n * n; q += CHT) {
    const int j = (int)(q / n), i = (int)(q - (long)j * n);
    if (i < j) A_(i, j) = 0.0;
  }
  __syncthreads();
  // diagonal blocks in place, one warp each
  for (int J = warp; J < nblk; J += nw) {
    const int j0 = J * CB;
    warp_trinv(&A_(j0, j0), ld, min(CB, n - j0), lane);
  }
  __syncthreads();
  // row blocks top-down, column blocks left to right, in place:
  // X_IJ = -X_II * sum_{K=J}^{I-1} L_IK X_KJ  (L_IK, K >= J, not yet overwritten)
  for (int I = 1; I < nblk; ++I) {
    const int i0 = I * CB, bi = min(CB, n - i0);
    for (int J = 0; J < I; ++J) {
      const int j0 = J * CB;
      for (int q = tid; q < CB * CB; q += CHT) {
        const int jj = q >> 5, ii = q & 31;
        double s = 0.0;
        if (ii < bi)
          for (int k = j0; k < i0; ++k) s += A_(i0 + ii, k) * A_(k, j0 + jj);
        T[jj * DLD + ii] = s;
      }
      __syncthreads();
      for (int q = tid; q < CB * CB; q += CHT) {
        const int jj = q >> 5, ii = q & 31;
        if (ii < bi) {
          double s = 0.0;
          for (int k = 0; k <= ii; ++k) s += A_(i0 + ii, i0 + k) * T[jj * DLD + k];
          A_(i0 + ii, j0 + jj) = -s;
        }
      }
      __syncthreads();
    }
  }
  if (use_smem)
    for (long q = tid; q < (long)n * n; q += CHT) {
      const int j = (int)(q / n), i = (int)(q - (long)j * n);
      Sg[q] = A_(i, j);
    }
#undef A_
  if (tid == 0) *info = 0;
}

// S: n x n column-major.  When S does not fit shared memory the kernel works
// in S itself (L2-resident) and uses work (>= CB*DLD doubles) as temporary.
int cholinv(double *S, int n, double *work, int *d_info, cudaStream_t st) {
  if (n > 8192) { set_error("cholinv: n=%d too large", n); return 1; }
  const size_t bytes = sizeof(double) * ((size_t)(n | 1) * n + CB * DLD);
  const int use = bytes <= CH_SMEM_MAX;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_cholinv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CH_SMEM_MAX);
    attr = true;
  }
  if (!use && !work) { set_error("cholinv: n=%d needs a work buffer", n); return 1; }
  k_cholinv<<<1, CHT, use ? bytes : 0, st>>>(S, n, work, d_info, use); note_launch();
  return 0;
}

// --------------------------------------------------------------------------
// Symmetric eigen-decomposition of the subspace Hamiltonian (the role of
// RsEIGQR, funcs.f90:380-764, which also reduces to tridiagonal form by
// Householder reflections):
//  (1) k_sytrd: Householder tridiagonalisation T = Q^T A Q in one CTA, three
//      barriers per column (reflector, matrix-vector product, rank-2 update);
//  (2) k_bisect: eigenvalues of T by Sturm-count multisection, one warp per
//      eigenvalue, 33 subintervals per round;
//  (3) k_invit: eigenvectors of T by inverse iteration with a pivoted
//      tridiagonal LU, one thread per cluster of close eigenvalues, members
//      re-orthogonalised against each other; per-thread work arrays are
//      interleaved across threads so every access is coalesced;
//  (4) k_backtrans: V = Q Z, one warp per column.
// Eigenpairs are ascending; each eigenvector's largest-magnitude component is
// made positive (first index on ties).  Every loop is bounded.

constexpr int TRD_T = 1024;
constexpr size_t TRD_SMEM_MAX = 222 * 1024;

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

// gvec: 2n doubles of global memory for v and p when A is not in shared memory.
__global__ void __launch_bounds__(TRD_T) k_sytrd(double *__restrict__ Ag, int n, double *__restrict__ d,
                                                 double *__restrict__ e, double *__restrict__ HV,
                                                 double *__restrict__ tau, int use_smem, double *__restrict__ gvec) {
  extern __shared__ double sm[];
  __shared__ double sc[2];
  const int ld = use_smem ? (n | 1) : n;
  double *A = use_smem ? sm : Ag;
  double *v = use_smem ? sm + (long)ld * n : gvec;
  double *p = v + n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#define A_(i, j) A[(long)(j) * ld + (i)]
  if (use_smem)
    for (long q = tid; q < (long)n * n; q += TRD_T) {
      const int j = (int)(q / n), i = (int)(q - (long)j * n);
      A_(i, j) = Ag[q];
    }
  __syncthreads();
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;
    if (warp == 0) {
      double sg = 0.0;
      for (int i = 1 + lane; i < m; i += 32) { const double x = A_(k + 1 + i, k); sg += x * x; }
      sg = warp_sum(sg);
      double t = 0.0, be = 1.0, al = 0.0;
      if (lane == 0) house(A_(k + 1, k), sg, t, be, al);
      t = __shfl_sync(0xffffffffu, t, 0);
      be = __shfl_sync(0xffffffffu, be, 0);
      for (int i = lane; i < m; i += 32) {
        const double vi = (i == 0) ? 1.0 : ((t != 0.0) ? A_(k + 1 + i, k) / be : 0.0);
        v[i] = vi;
        HV[(long)k * n + k + 1 + i] = vi;
      }
      if (lane == 0) {
        tau[k] = t;
        d[k] = A_(k, k);
        e[k] = al;
        sc[k & 1] = t;
      }
    }
    __syncthreads();
    // uniform: written before the barrier; alternating slots keep a thread
    // that reads late from seeing the next column's value
    const double t = sc[k & 1];
    if (t == 0.0) continue;
    // p = t * B v, B = A(k+1:, k+1:); G lanes per row (G | 32)
    int G = 1;
    while (G < 32 && 2 * G * m <= TRD_T) G *= 2;
    const int R = TRD_T / G, g = tid % G, r = tid / G;
    for (int i0 = 0; i0 < m; i0 += R) {
      const int i = i0 + r;
      double s = 0.0;
      if (i < m)
        for (int j = g; j < m; j += G) s += A_(k + 1 + i, k + 1 + j) * v[j];
      for (int o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (g == 0 && i < m) p[i] = t * s;
    }
    __syncthreads();
    // K = t/2 v^T p (every warp computes it), w = p - K v, B -= v w^T + w v^T
    double kk = 0.0;
    for (int i = lane; i < m; i += 32) kk += v[i] * p[i];
    const double K = 0.5 * t * warp_sum(kk);
    for (long q = tid; q < (long)m * m; q += TRD_T) {
      const int j = (int)(q / m), i = (int)(q - (long)j * m);
      const double vi = v[i], vj = v[j];
      const double wi = p[i] - K * vi, wj = p[j] - K * vj;
      A_(k + 1 + i, k + 1 + j) -= vi * wj + wi * vj;
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (n >= 2) {
      d[n - 2] = A_(n - 2, n - 2);
      e[n - 2] = A_(n - 1, n - 2);
    }
    d[n - 1] = A_(n - 1, n - 1);
  }
#undef A_
}

// Number of eigenvalues of T below x (Sturm count, pivots guarded by pmin).
__device__ __forceinline__ int sturm(const double *__restrict__ d, const double *__restrict__ e, int n, double x,
                                     double pmin) {
  int c = 0;
  double q = d[0] - x;
  if (fabs(q) < pmin) q = -pmin;
  if (q < 0.0) ++c;
  for (int i = 1; i < n; ++i) {
    const double ei = e[i - 1];
    q = d[i] - x - ei * ei / q;
    if (fabs(q) < pmin) q = -pmin;
    if (q < 0.0) ++c;
  }
  return c;
}

// Eigenvalue t of T (ascending) by multisection: each round the 32 lanes of
// warp t count the eigenvalues below 32 interior points of [lo, hi] and the
// interval shrinks to the one of 33 parts that holds eigenvalue t, until it
// is 2 eps |T| wide (at most 24 rounds).
__global__ void k_bisect(const double *__restrict__ d, const double *__restrict__ e, int n, double *__restrict__ w) {
  const int t = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (t >= n) return;   // whole warp
  double lo = 1e300, hi = -1e300, tn = 0.0;
  for (int i = lane; i < n; i += 32) {
    const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
    tn = fmax(tn, fabs(d[i]) + r);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    tn = fmax(tn, __shfl_xor_sync(0xffffffffu, tn, o));
  }
  const double eps = 2.220446049250313e-16;
  const double pmin = 1e-300 + eps * eps * tn * tn * 1e-10;
  lo -= 2.0 * eps * tn + 1e-300;
  hi += 2.0 * eps * tn + 1e-300;
  for (int it = 0; it < 24; ++it) {
    if (hi - lo <= 2.0 * eps * tn + 4.0 * pmin) break;
    const double h = (hi - lo) * (1.0 / 33.0);
    const double x = lo + (double)(lane + 1) * h;
    const int c = sturm(d, e, n, x, pmin);
    const unsigned bal = __ballot_sync(0xffffffffu, c > t);
    const int l = bal ? __ffs(bal) - 1 : 32;   // eigenvalue t lies in [x_{l-1}, x_l)
    const double nlo = (l == 0) ? lo : lo + (double)l * h;
    const double nhi = (l == 32) ? hi : lo + (double)(l + 1) * h;
    if (!(nhi > nlo)) break;                    // no representable progress
    lo = nlo;
    hi = nhi;
  }
  if (lane == 0) w[t] = 0.5 * (lo + hi);
}

// Inverse iteration on T for the eigenvalues of one cluster (consecutive
// eigenvalues closer than 1e-6 |T|), members orthogonalised against the
// earlier ones.  Thread t is active if eigenvalue t starts a cluster.
// ws: 6 arrays of n x NT doubles, element (a, i) of thread t at
// ws[(a*n + i)*NT + t] (coalesced across threads).  Z(:, t) = eigenvector t.
__global__ void k_invit(const double *__restrict__ d, const double *__restrict__ e, const double *__restrict__ w,
                        int n, double *__restrict__ Z, double *__restrict__ ws, int NT, int *__restrict__ nclus) {
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
#define WS(a, i) ws[((long)(a) * n + (i)) * NT + t]
  // 0: 1/U(i,i), 1: U(i,i+1), 2: U(i,i+2), 3: multiplier, 4: row swap flag, 5: z
  const double tiny = eps * tn + 1e-300;
  for (int c = t; c < tend; ++c) {
    // perturb members apart so their LU factors differ
    const double lam = w[c] + (double)(c - t) * 4.0 * eps * tn;
    double a = d[0] - lam, b = (n > 1) ? e[0] : 0.0;
    for (int i = 0; i < n - 1; ++i) {
      const double cdn = e[i];                 // subdiagonal below a
      const double dn = d[i + 1] - lam;        // next diagonal
      const double en = (i + 1 < n - 1) ? e[i + 1] : 0.0;
      if (fabs(a) >= fabs(cdn)) {
        const double aa = (fabs(a) < tiny) ? tiny : a;
        const double l = cdn / aa;
        WS(0, i) = 1.0 / aa; WS(1, i) = b; WS(2, i) = 0.0; WS(3, i) = l; WS(4, i) = 0.0;
        a = dn - l * b;
        b = en;
      } else {
        const double l = a / cdn;
        WS(0, i) = 1.0 / cdn; WS(1, i) = dn; WS(2, i) = en; WS(3, i) = l; WS(4, i) = 1.0;
        a = b - l * dn;
        b = -l * en;
      }
    }
    WS(0, n - 1) = 1.0 / ((fabs(a) < tiny) ? tiny : a);
    // start vector: ones with a member-dependent pattern
    for (int i = 0; i < n; ++i) WS(5, i) = 1.0 + 0.01 * (double)((i * (c + 3)) % 7);
    for (int it = 0; it < 3; ++it) {
      // forward: row interchanges and multipliers
      double zi = WS(5, 0);
      for (int i = 0; i < n - 1; ++i) {
        const double zn = WS(5, i + 1);
        if (WS(4, i) != 0.0) { WS(5, i) = zn; zi = zi - WS(3, i) * zn; }   // rows i, i+1 swapped
        else { WS(5, i) = zi; zi = zn - WS(3, i) * zi; }
      }
      WS(5, n - 1) = zi;
      // back substitution with U (two superdiagonals)
      double z2 = 0.0, z1 = WS(5, n - 1) * WS(0, n - 1);
      WS(5, n - 1) = z1;
      if (n > 1) {
        const double z0 = (WS(5, n - 2) - WS(1, n - 2) * z1) * WS(0, n - 2);
        WS(5, n - 2) = z0;
        z2 = z1;
        z1 = z0;
      }
      for (int i = n - 3; i >= 0; --i) {
        const double z0 = (WS(5, i) - WS(1, i) * z1 - WS(2, i) * z2) * WS(0, i);
        WS(5, i) = z0;
        z2 = z1;
        z1 = z0;
      }
      // orthogonalise against the earlier members of the cluster
      for (int q = t; q < c; ++q) {
        const double *zq = Z + (long)q * n;
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += zq[i] * WS(5, i);
        for (int i = 0; i < n; ++i) WS(5, i) -= s * zq[i];
      }
      double nr = 0.0;
      for (int i = 0; i < n; ++i) { const double x = WS(5, i); nr += x * x; }
      nr = 1.0 / sqrt(nr);
      for (int i = 0; i < n; ++i) WS(5, i) *= nr;
    }
    double *z = Z + (long)c * n;
    for (int i = 0; i < n; ++i) z[i] = WS(5, i);
  }
#undef WS
}

// V(:, c) = Q Z(:, c), one warp per column c: reflectors k = n-3 .. 0; then
// the sign convention.  zs: (blockDim/32) * n doubles of shared memory.
__global__ void __launch_bounds__(256) k_backtrans(const double *__restrict__ Z, const double *__restrict__ HV,
                                                   const double *__restrict__ tau, int n, double *__restrict__ V) {
  extern __shared__ double zs[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * (blockDim.x >> 5) + warp;
  if (c >= n) return;   // whole warp
  double *z = zs + (long)warp * n;
  for (int i = lane; i < n; i += 32) z[i] = Z[(long)c * n + i];
  // each lane reads and writes only its own entries i = lane mod 32
  for (int k = n - 3; k >= 0; --k) {
    const double tk = tau[k];
    if (tk == 0.0) continue;
    const double *v = HV + (long)k * n;
    double s = 0.0;
    for (int i = k + 1 + lane; i < n; i += 32) s += v[i] * z[i];
    s = tk * warp_sum(s);
    for (int i = k + 1 + lane; i < n; i += 32) z[i] -= v[i] * s;
  }
  double mx = -1.0;
  int km = 0;
  for (int i = lane; i < n; i += 32) {
    const double a = fabs(z[i]);
    if (a > mx) { mx = a; km = i; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double m2 = __shfl_xor_sync(0xffffffffu, mx, o);
    const int k2 = __shfl_xor_sync(0xffffffffu, km, o);
    if (m2 > mx || (m2 == mx && k2 < km)) { mx = m2; km = k2; }
  }
  const double sg = z[km] < 0.0 ? -1.0 : 1.0;
  for (int i = lane; i < n; i += 32) V[(long)c * n + i] = sg * z[i];
}

// A (n x n, destroyed), w (n) eigenvalues ascending, V (n x n) eigenvectors.
// work: at least 8*n*n + 1024*n doubles.  info: number of eigenvalue clusters.
int syev(double *A, int n, double *w, double *V, double *work, int *d_info, cudaStream_t st) {
  if (n < 1) { set_error("syev: n=%d", n); return 1; }
  const int NT = ((n + 127) / 128) * 128;
  double *d = work, *e = d + n, *tau = e + n, *vp = tau + n, *HV = vp + 2 * (long)n, *Z = HV + (long)n * n,
         *ws = Z + (long)n * n;   // 6 * n * NT <= 6n^2 + 762n: total <= 8n^2 + 767n
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_sytrd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRD_SMEM_MAX);
    cudaFuncSetAttribute(k_backtrans, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  const size_t smem = sizeof(double) * ((size_t)(n | 1) * n + 2 * (size_t)n);
  const int use = smem <= TRD_SMEM_MAX;
  cudaMemsetAsync(d_info, 0, sizeof(int), st);
  k_sytrd<<<1, TRD_T, use ? smem : 0, st>>>(A, n, d, e, HV, tau, use, vp); note_launch();
  if (n == 1) {
    cudaMemcpyAsync(w, d, sizeof(double), cudaMemcpyDeviceToDevice, st);
    static const double one = 1.0;
    cudaMemcpyAsync(V, &one, sizeof(double), cudaMemcpyHostToDevice, st);
    return 0;
  }
  k_bisect<<<(n * 32 + 255) / 256, 256, 0, st>>>(d, e, n, w); note_launch();
  k_invit<<<NT / 128, 128, 0, st>>>(d, e, w, n, Z, ws, NT, d_info); note_launch();
  const size_t bt = sizeof(double) * 8 * (size_t)n;
  if (bt > 200 * 1024) { set_error("syev: n=%d too large for the back-transformation", n); return 1; }
  k_backtrans<<<(n + 7) / 8, 256, bt, st>>>(Z, HV, tau, n, V); note_launch();
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
