// FP64 dense kernels on the nb x nb band matrices: Cholesky + triangular
// inverse (rsdecmp/rsinvcd, schmidt.f90:428-544) and the symmetric
// eigen-decomposition of the subspace Hamiltonian (the role of RsEIGQR,
// funcs.f90:380, called from untryt2, eigen.f90:1237) by parallel cyclic
// Jacobi.  Each runs as one CTA; matrices live in shared memory when they fit
// and in global memory (L2) otherwise.  No wait in these kernels depends on
// another block.
#include "qx_internal.h"

namespace qx {

constexpr int DT = 1024;
constexpr size_t SMEM_MAX = 200 * 1024;

// Column-major n x n.  info: 0 ok, 1+i if pivot i <= 1e-30.
__global__ void __launch_bounds__(DT) k_cholinv(double *__restrict__ Sg, int n, int *__restrict__ info, int use_smem) {
  extern __shared__ double sm[];
  __shared__ double red[DT / 32];
  __shared__ int bad;
  double *S = use_smem ? sm : Sg;
  if (use_smem)
    for (long i = threadIdx.x; i < (long)n * n; i += blockDim.x) S[i] = Sg[i];
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
#define S_(i, j) S[(long)(j) * n + (i)]
  // rsdecmp: left-looking, row i of L from rows < i.
  for (int i = 0; i < n; ++i) {
    double part = 0.0;
    for (int k = threadIdx.x; k < i; k += blockDim.x) part += S_(i, k) * S_(i, k);
    const double ss = block_sum(part, red);
    double d = S_(i, i) - ss;
    if (d > 1.0e-30) {
      d = sqrt(d);
      for (int j = i + 1 + threadIdx.x; j < n; j += blockDim.x) {
        double s = S_(j, i);
        for (int k = 0; k < i; ++k) s -= S_(j, k) * S_(i, k);
        S_(j, i) = s / d;
      }
    } else {
      for (int j = i + 1 + threadIdx.x; j < n; j += blockDim.x) S_(j, i) = 0.0;
      if (threadIdx.x == 0 && !bad) bad = 1 + i;
      d = 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) S_(i, i) = d;
    __syncthreads();
  }
  if (bad) {
    if (threadIdx.x == 0) *info = bad;
    return;
  }
  // rsinvcd: scale the strict lower part by 1/diag, diag <- 1/diag, then
  // back-substitute columns from the right.
  for (long e = threadIdx.x; e < (long)n * n; e += blockDim.x) {
    const int j = (int)(e / n), i = (int)(e - (long)j * n);
    if (i > j) S_(i, j) = S_(i, j) / S_(j, j);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) S_(i, i) = 1.0 / S_(i, i);
  for (long e = threadIdx.x; e < (long)n * n; e += blockDim.x) {
    const int j = (int)(e / n), i = (int)(e - (long)j * n);
    if (i < j) S_(i, j) = 0.0;
  }
  __syncthreads();
  for (int j = n - 2; j >= 0; --j) {
    double acc[8];
    int cnt = 0;
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      double s = 0.0;
      for (int k = j + 1; k <= i; ++k) s += S_(i, k) * S_(k, j);
      if (cnt < 8) acc[cnt] = s;
      ++cnt;
    }
    __syncthreads();
    cnt = 0;
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      if (cnt < 8) S_(i, j) = -acc[cnt];
      ++cnt;
    }
    __syncthreads();
  }
#undef S_
  if (use_smem)
    for (long i = threadIdx.x; i < (long)n * n; i += blockDim.x) Sg[i] = S[i];
  if (threadIdx.x == 0) *info = 0;
}

int cholinv(double *S, int n, int *d_info, cudaStream_t st) {
  if (n > 8 * DT) { set_error("cholinv: n=%d too large", n); return 1; }
  const size_t bytes = sizeof(double) * (size_t)n * n;
  const int use = bytes <= SMEM_MAX;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_cholinv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX);
    attr = true;
  }
  k_cholinv<<<1, DT, use ? bytes : 0, st>>>(S, n, d_info, use);
  return 0;
}

// --------------------------------------------------------------------------
// Parallel cyclic Jacobi, round-robin (Brent-Luk) pair order: every round
// rotates m/2 disjoint pairs at once, which gives the same result as
// applying them one after another.  After convergence the eigenpairs are
// sorted ascending and each eigenvector's largest-magnitude component is made
// positive (first index on ties).  info: number of sweeps, or -1.
__global__ void __launch_bounds__(DT) k_jacobi(double *__restrict__ Ag, int n, double *__restrict__ wout,
                                               double *__restrict__ Vout, double *__restrict__ Vw, int maxsweep,
                                               int *__restrict__ info, int use_smem) {
  extern __shared__ double sm[];
  __shared__ double red[DT / 32];
  __shared__ int top[2 * DT + 2];
  __shared__ double cs[DT + 1], sn[DT + 1];
  __shared__ int pp[DT + 1], qq[DT + 1];
  __shared__ int any;
  double *A = use_smem ? sm : Ag;
  if (use_smem)
    for (long i = threadIdx.x; i < (long)n * n; i += blockDim.x) A[i] = Ag[i];
  double *V = Vw;
#define A_(i, j) A[(long)(j) * n + (i)]
#define V_(i, j) V[(long)(j) * n + (i)]
  for (long e = threadIdx.x; e < (long)n * n; e += blockDim.x) {
    const int j = (int)(e / n), i = (int)(e - (long)j * n);
    V_(i, j) = (i == j) ? 1.0 : 0.0;
  }
  const int m = n + (n & 1), half = m / 2;
  for (int i = threadIdx.x; i < m; i += blockDim.x) top[i] = i;
  __syncthreads();
  int sweeps = -1;
  for (int sw = 0; sw < maxsweep; ++sw) {
    double off = 0.0, tot = 0.0;
    for (long e = threadIdx.x; e < (long)n * n; e += blockDim.x) {
      const int j = (int)(e / n), i = (int)(e - (long)j * n);
      const double x = A_(i, j) * A_(i, j);
      tot += x;
      if (i != j) off += x;
    }
    off = block_sum(off, red);
    tot = block_sum(tot, red);
    if (off <= 1e-30 * tot || off == 0.0) { sweeps = sw; break; }
    for (int r = 0; r < m - 1; ++r) {
      if (threadIdx.x == 0) any = 0;
      __syncthreads();
      for (int k = threadIdx.x; k < half; k += blockDim.x) {
        int p = top[k], q = top[m - 1 - k];
        double c = 1.0, s = 0.0;
        if (p < n && q < n) {
          if (p > q) { const int t = p; p = q; q = t; }
          const double apq = A_(p, q);
          if (apq != 0.0) {
            const double theta = (A_(q, q) - A_(p, p)) / (2.0 * apq);
            const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(t * t + 1.0);
            s = t * c;
            any = 1;
          }
        } else {
          p = -1; q = -1;
        }
        pp[k] = p; qq[k] = q; cs[k] = c; sn[k] = s;
      }
      __syncthreads();
      if (any) {
        // columns p, q of A and V
        for (long e = threadIdx.x; e < (long)half * n; e += blockDim.x) {
          const int k = (int)(e / n), i = (int)(e - (long)k * n);
          const int p = pp[k], q = qq[k];
          if (p < 0 || sn[k] == 0.0) continue;
          const double c = cs[k], s = sn[k];
          const double aip = A_(i, p), aiq = A_(i, q);
          A_(i, p) = c * aip - s * aiq;
          A_(i, q) = s * aip + c * aiq;
          const double vip = V_(i, p), viq = V_(i, q);
          V_(i, p) = c * vip - s * viq;
          V_(i, q) = s * vip + c * viq;
        }
        __syncthreads();
        // rows p, q of A
        for (long e = threadIdx.x; e < (long)half * n; e += blockDim.x) {
          const int k = (int)(e / n), i = (int)(e - (long)k * n);
          const int p = pp[k], q = qq[k];
          if (p < 0 || sn[k] == 0.0) continue;
          const double c = cs[k], s = sn[k];
          const double api = A_(p, i), aqi = A_(q, i);
          A_(p, i) = c * api - s * aqi;
          A_(q, i) = s * api + c * aqi;
        }
      }
      __syncthreads();
      // rotate positions 1..m-1 of the tournament
      int nv[4];
      int cnt = 0;
      for (int i = 1 + threadIdx.x; i < m; i += blockDim.x) {
        const int src = (i == 1) ? m - 1 : i - 1;
        if (cnt < 4) nv[cnt] = top[src];
        ++cnt;
      }
      __syncthreads();
      cnt = 0;
      for (int i = 1 + threadIdx.x; i < m; i += blockDim.x) {
        if (cnt < 4) top[i] = nv[cnt];
        ++cnt;
      }
      __syncthreads();
    }
  }
  // eigenvalues, rank sort (ties by index), sign normalisation
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double wi = A_(i, i);
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double wj = A_(j, j);
      if (wj < wi || (wj == wi && j < i)) ++rank;
    }
    wout[rank] = wi;
    // find the largest-magnitude component of column i
    int kmax = 0;
    double mx = -1.0;
    for (int r = 0; r < n; ++r) {
      const double a = fabs(V_(r, i));
      if (a > mx) { mx = a; kmax = r; }
    }
    const double sgn = V_(kmax, i) < 0.0 ? -1.0 : 1.0;
    for (int r = 0; r < n; ++r) Vout[(long)rank * n + r] = sgn * V_(r, i);
  }
#undef A_
#undef V_
  if (threadIdx.x == 0) *info = sweeps;
}

// k_jacobi holds about 33 KB of static shared memory, so its dynamic part
// (the matrix) is limited to 190 KB: n <= 157 runs in shared memory.
constexpr size_t JSMEM_MAX = 190 * 1024;

int jacobi(double *A, int n, double *w, double *V, int maxsweep, int *d_info, cudaStream_t st) {
  if (n > 2 * DT) { set_error("jacobi: n=%d too large", n); return 1; }
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)JSMEM_MAX);
    attr = true;
  }
  const size_t bytes = sizeof(double) * (size_t)n * n;
  const int use = bytes <= JSMEM_MAX;
  // V work array: the second half of A's buffer is not available, so the
  // caller passes V with room for 2*n*n doubles (work + sorted output).
  k_jacobi<<<1, DT, use ? bytes : 0, st>>>(A, n, w, V, V + (long)n * n, maxsweep, d_info, use);
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
  k_convert<Tin, Tout><<<blocks, 256, 0, st>>>(in, out, n);
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
  k_symmetrize<T><<<(int)((nn + 255) / 256), 256, 0, st>>>(in, out, diag, n);
}
template void symmetrize_lower<float>(const float *, double *, double *, int, cudaStream_t);
template void symmetrize_lower<double>(const double *, double *, double *, int, cudaStream_t);

}  // namespace qx
