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
// dimension) when they fit and in global memory (L2) otherwise.  For large
// n the Cholesky and the tridiagonalisation spread the columns over one CTA
// per SM in a cooperative launch, with bounded grid barriers; no other wait
// in these kernels depends on another block.
#include <algorithm>

#include "qx_internal.h"

namespace qx {

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// f(DenseIC<I>{}) for I = B .. E-1: a compile-time index for register arrays,
// used to branch on a uniform runtime slot instead of selecting over slots.
template <int I> struct DenseIC { static constexpr int value = I; };
template <int B, int E, typename F> __device__ __forceinline__ void dense_static_for(F &&f) {
  if constexpr (B < E) {
    f(DenseIC<B>{});
    dense_static_for<B + 1, E>(f);
  }
}

// ---------------------------------------------------------------------------
// Grid barrier for the cooperative kernels of this file (all CTAs co-resident by the
// cooperative launch).  bar[0]: arrival count, bar[1]: generation, both zero
// before the launch.  The last CTA to arrive resets the count and advances
// the generation; the others poll the generation (L2 loads) for at most
// GB_WAIT_NS, after which the barrier reports failure (every later barrier of
// that CTA fails as well, so all CTAs leave their loops).  Writes before the
// barrier are published by the block barrier plus thread 0's fence; reads of
// data written by other CTAs use __ldcg (L2), never a possibly stale L1 line.
constexpr unsigned long long GB_WAIT_NS = 2000000000ull;
__device__ __forceinline__ unsigned long long gb_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned nblk, int *okflag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    if (*okflag) {
      const unsigned g0 = __ldcg(bar + 1);
      __threadfence();
      if (atomicAdd(bar, 1u) == nblk - 1) {
        atomicExch(bar, 0u);
        __threadfence();
        atomicAdd(bar + 1, 1u);
      } else {
        const unsigned long long t0 = gb_now();
        while (__ldcg(bar + 1) == g0) {
          if (gb_now() - t0 > GB_WAIT_NS) {
            *okflag = 0;
            break;
          }
          __nanosleep(64);
        }
      }
      __threadfence();
    }
  }
  __syncthreads();
  return *okflag != 0;
}

// --------------------------------------------------------------------------
// Cholesky S = L L^T and L^-1, blocked by CB = 32.  Column-major n x n; on
// return the lower triangle holds L^-1 and the upper triangle zeros.
// info: 0, or 1+i for the first row i whose pivot (the Schur-complement
// diagonal S(i,i) - sum_k L(i,k)^2 that rsdecmp tests) is not > 1e-30
// (schmidt.f90:256-267).
constexpr int CB = 32;
constexpr int CHT = 256;            // threads of k_cholinv (8 warps)
constexpr int DLD = CB + 1;         // leading dimension of the 32 x 32 temporary
constexpr size_t CH_SMEM_MAX = 220 * 1024;

// 1/sqrt(x): the hardware's approximate reciprocal square root refined by
// two Newton-Raphson steps y <- y (3 - x y^2) / 2, each doubling the number
// of correct bits, to full double precision.
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  y = y * (1.5 - 0.5 * x * y * y);
  y = y * (1.5 - 0.5 * x * y * y);
  return y;
}

// Cholesky of the bs x bs diagonal block at B (leading dimension ld) in
// registers: lane i holds row i; column k of L is broadcast through the
// 32-double shared buffer cb (cheaper than 31 shuffles of doubles per step).
// Writes L (lower triangle, diagonal included) and 1/L(k,k) to rd[k].
// Returns the first row whose pivot is not > 1e-30, or -1.  One whole warp.
__device__ __forceinline__ int warp_chol(double *B, int ld, int bs, int lane, double *rd, double *cb) {
  double r[CB];
#pragma unroll
  for (int j = 0; j < CB; ++j) r[j] = (lane < bs && j < bs && j <= lane) ? B[(long)j * ld + lane] : 0.0;
  // no early exit: a break would keep the loop from unrolling and r[] from
  // staying in registers; after a failed pivot the remaining steps are skipped
  int bad = -1;
#pragma unroll
  for (int k = 0; k < CB; ++k) {
    if (k < bs && bad < 0) {
      const double piv = __shfl_sync(0xffffffffu, r[k], k);
      if (!(piv > 1.0e-30)) {   // uniform; also catches NaN
        bad = k;
        continue;
      }
      const double rs = rsqrt_nr(piv);
      const double lik = (lane == k) ? piv * rs : r[k] * rs;   // L(k,k) on lane k, l_ik below
      r[k] = lik;
      if (lane == k) rd[k] = rs;
      cb[lane] = lik;
      __syncwarp();
#pragma unroll
      for (int j = k + 1; j < CB; ++j)
        if (lane >= j) r[j] -= lik * cb[j];
      __syncwarp();
    }
  }
  if (bad < 0 && lane < bs) {
#pragma unroll
    for (int j = 0; j < CB; ++j)
      if (j <= lane) B[(long)j * ld + lane] = r[j];
  }
  __syncwarp();
  return bad;
}

// X = L^-1 of the lower-triangular bs x bs block at L (leading dimension ldl)
// into X (leading dimension ldx; may equal L), lane j producing column j by
// forward substitution with L's rows read as broadcasts and the diagonal
// reciprocals rd[].  Zeros above the diagonal.  One whole warp.
__device__ __forceinline__ void warp_trinv(const double *L, int ldl, const double *rd, double *X, int ldx, int bs,
                                           int lane) {
  double x[CB];
#pragma unroll
  for (int i = 0; i < CB; ++i) {
    double s = (i == lane) ? 1.0 : 0.0;
    if (i < bs) {
#pragma unroll
      for (int k = 0; k < i; ++k) s -= L[(long)k * ldl + i] * x[k];
      x[i] = s * rd[i];
    } else {
      x[i] = 0.0;
    }
  }
  __syncwarp();
  if (lane < bs) {
#pragma unroll
    for (int i = 0; i < CB; ++i)
      if (i < bs) X[(long)lane * ldx + i] = (i >= lane) ? x[i] : 0.0;
  }
  __syncwarp();
}

// USE_SMEM: the matrix lives in shared memory, and the compiler sees that
// every access to it is a shared-memory access (no generic addressing).
template <bool USE_SMEM>
__global__ void __launch_bounds__(CHT) k_cholinv(double *__restrict__ Sg, int n, double *__restrict__ work,
                                                  int *__restrict__ info) {
  constexpr bool use_smem = USE_SMEM;
  extern __shared__ double sm[];
  __shared__ int bad;
  const int ld = use_smem ? (n | 1) : n;
  double *A = use_smem ? sm : Sg;
  double *T = use_smem ? sm + (long)ld * n : work;   // CB x DLD temporary
  double *rd = T + CB * DLD;                         // n reciprocal pivots
  __shared__ double cb[CB];                          // column broadcast of warp_chol
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = CHT / 32;
#define A_(i, j) A[(long)(j) * ld + (i)]
  if (use_smem)
    for (int j = warp; j < n; j += nw)
      for (int i = lane; i < n; i += 32) A_(i, j) = Sg[(long)j * n + i];
  if (tid == 0) bad = 0;
  __syncthreads();
  const int nblk = (n + CB - 1) / CB;
  // ---- right-looking blocked Cholesky ----
  for (int J = 0; J < nblk; ++J) {
    const int j0 = J * CB, bs = min(CB, n - j0);
    if (warp == 0) {
      const int b = warp_chol(&A_(j0, j0), ld, bs, lane, rd + j0, cb);
      if (b >= 0) {
        if (lane == 0) bad = 1 + j0 + b;
      } else if (j0 + bs < n) {
        warp_trinv(&A_(j0, j0), ld, rd + j0, T, DLD, bs, lane);   // Linv_JJ for the panel
      }
    }
    __syncthreads();
    if (bad) break;
    const int r0 = j0 + bs, mr = n - r0;
    if (mr <= 0) break;
    // panel: L(r, j0+c) = sum_{k <= c} A(r, j0+k) Linv_JJ(c, k), lane = row
    for (int rc = r0 + warp * 32; rc < n; rc += nw * 32) {
      const int r = rc + lane;
      if (r < n) {
        double a[CB];
#pragma unroll
        for (int k = 0; k < CB; ++k) a[k] = (k < bs) ? A_(r, j0 + k) : 0.0;
#pragma unroll
        for (int c = 0; c < CB; ++c) {
          if (c < bs) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k <= c; ++k) s += a[k] * T[k * DLD + c];
            A_(r, j0 + c) = s;
          }
        }
      }
    }
    __syncthreads();
    // trailing update of the lower triangle, 32 x 32 tiles (row chunk qi,
    // column chunk qj <= qi): A(r, c) -= sum_k L(r, j0+k) L(c, j0+k), lane = row
    const int nq = (mr + 31) / 32;
    for (int tile = warp; tile < nq * (nq + 1) / 2; tile += nw) {
      int qi = 0;
      while ((qi + 1) * (qi + 2) / 2 <= tile) ++qi;
      const int qj = tile - qi * (qi + 1) / 2;
      const int r = qi * 32 + lane;
      double a[CB];
#pragma unroll
      for (int k = 0; k < CB; ++k) a[k] = (r < mr && k < bs) ? A_(r0 + r, j0 + k) : 0.0;
      const int cend = min(qj * 32 + 32, mr);
      for (int c = qj * 32; c < cend; ++c) {
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int k = 0; k < CB; k += 2) {
          s0 += a[k] * A_(r0 + c, j0 + k);
          s1 += a[k + 1] * A_(r0 + c, j0 + k + 1);
        }
        if (r < mr && r >= c) A_(r0 + r, r0 + c) -= s0 + s1;
      }
    }
    __syncthreads();
  }
  if (bad) {
    if (tid == 0) *info = bad;
    return;
  }
  // ---- L^-1, blocked ----
  // zero the strict upper triangle (it still holds S)
  for (int j = warp; j < n; j += nw)
    for (int i = lane; i < j; i += 32) A_(i, j) = 0.0;
  __syncthreads();
  // diagonal blocks in place, one warp each
  for (int J = warp; J < nblk; J += nw) {
    const int j0 = J * CB;
    warp_trinv(&A_(j0, j0), ld, rd + j0, &A_(j0, j0), ld, min(CB, n - j0), lane);
  }
  __syncthreads();
  // row blocks top-down, column blocks left to right, in place:
  // X_IJ = -X_II * sum_{K=J}^{I-1} L_IK X_KJ  (L_IK, K >= J, not yet overwritten)
  // lane = row ii, warp = columns jj = warp + 8 u (u < 4)
  for (int I = 1; I < nblk; ++I) {
    const int i0 = I * CB, bi = min(CB, n - i0);
    for (int J = 0; J < I; ++J) {
      const int j0 = J * CB;
      {
        double acc[CB / (CHT / 32)] = {};
        if (lane < bi)
          for (int k = j0; k < i0; ++k) {
            const double a = A_(i0 + lane, k);
#pragma unroll
            for (int u = 0; u < CB / (CHT / 32); ++u) acc[u] += a * A_(k, j0 + warp + u * nw);
          }
#pragma unroll
        for (int u = 0; u < CB / (CHT / 32); ++u) T[(warp + u * nw) * DLD + lane] = acc[u];
      }
      __syncthreads();
      if (lane < bi) {
        double acc[CB / (CHT / 32)] = {};
        for (int k = 0; k <= lane; ++k) {
          const double a = A_(i0 + lane, i0 + k);
#pragma unroll
          for (int u = 0; u < CB / (CHT / 32); ++u) acc[u] += a * T[(warp + u * nw) * DLD + k];
        }
#pragma unroll
        for (int u = 0; u < CB / (CHT / 32); ++u) A_(i0 + lane, j0 + warp + u * nw) = -acc[u];
      }
      __syncthreads();
    }
  }
  if (use_smem)
    for (int j = warp; j < n; j += nw)
      for (int i = lane; i < n; i += 32) Sg[(long)j * n + i] = A_(i, j);
#undef A_
  if (tid == 0) *info = 0;
}

// --------------------------------------------------------------------------
// The same result for n <= CP_MAXN (and within shared memory), 12 warps, one
// n x n shared-memory matrix (odd leading dimension) holding L in the lower
// triangle and X^T = (L^-1)^T strictly above it (X's diagonal apart):
//  * Cholesky right-looking in panels of PB = 8 columns: warp 0 factors the
//    panel in registers (rows lane + 32 q, column values by shuffle, no CTA
//    barrier inside the panel) and copies it row-major to Pr; all warps then
//    apply the rank-8 update to the trailing lower triangle;
//  * inverse in 32 x 32 blocks: the diagonal blocks inverted side by side
//    (one warp each); M_IK = -X_II L_IK in place of L_IK (all blocks at
//    once); X_IJ = sum_{K=J}^{I-1} M_IK X_KJ by block diagonals d = I - J
//    (the blocks of one diagonal at once, two warps a block).  Every inner
//    loop runs over compile-time indices into registers.
constexpr int CPT = 384, CPW = CPT / 32, PB = 8, CP_MQ = 6;
constexpr int CP_MAXN = 32 * CP_MQ;   // also bounded by shared memory

__global__ void __launch_bounds__(CPT) k_cholinv_sm(double *__restrict__ Sg, int n, int *__restrict__ info) {
  extern __shared__ double smf[];
  __shared__ int bad;
  const int ld = n | 1;
  double *A = smf, *xd = A + (long)ld * n, *rd = xd + n, *Pr = rd + n;   // Pr: PB * n
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#define AA(i, j) A[(j) * ld + (i)]
  if (tid == 0) bad = 0;
  for (int j = warp; j < n; j += CPW)
    for (int i = j + lane; i < n; i += 32) AA(i, j) = Sg[(long)j * n + i];
  __syncthreads();
  // ---------------- Cholesky ----------------
  for (int j0 = 0; j0 < n; j0 += PB) {
    const int pb = min(PB, n - j0);
    if (warp == 0) {
      double a[CP_MQ][PB];
#pragma unroll
      for (int q = 0; q < CP_MQ; ++q) {
        const int r = j0 + lane + 32 * q, rr = min(r, n - 1);
#pragma unroll
        for (int c = 0; c < PB; ++c) {
          const double v = AA(rr, min(j0 + c, n - 1));   // clamped address, then selection
          a[q][c] = (c < pb && r < n && r >= j0 + c) ? v : 0.0;
        }
      }
      int b = 0;
#pragma unroll
      for (int c = 0; c < PB; ++c) {
        if (c < pb && b == 0) {   // uniform
          const double piv = __shfl_sync(0xffffffffu, a[0][c], c);   // row j0 + c: lane c, q 0
          if (!(piv > 1.0e-30)) {   // uniform; also catches NaN
            b = 1 + j0 + c;
          } else {
            const double rs = rsqrt_nr(piv);
#pragma unroll
            for (int q = 0; q < CP_MQ; ++q) {
              const int r = j0 + lane + 32 * q;
              a[q][c] = (r == j0 + c) ? piv * rs : a[q][c] * rs;
            }
            if (lane == 0) rd[j0 + c] = rs;
            // columns c2 > c; rows above row j0 + c2 pick up values that are
            // never read (only rows >= j0 + c2 of column c2 are stored)
#pragma unroll
            for (int c2 = c + 1; c2 < PB; ++c2) {
              const double l = __shfl_sync(0xffffffffu, a[0][c], c2);   // L(j0 + c2, j0 + c)
#pragma unroll
              for (int q = 0; q < CP_MQ; ++q) a[q][c2] -= a[q][c] * l;
            }
          }
        }
      }
      if (b) {
        if (lane == 0) bad = b;
      } else {
#pragma unroll
        for (int q = 0; q < CP_MQ; ++q) {
          const int r = j0 + lane + 32 * q;
          if (r < n) {
#pragma unroll
            for (int c = 0; c < PB; ++c) {
              if (c < pb && r >= j0 + c) AA(r, j0 + c) = a[q][c];
              Pr[r * PB + c] = (c < pb) ? a[q][c] : 0.0;   // zero above the diagonal
            }
          }
        }
      }
    }
    __syncthreads();
    if (bad) break;   // uniform
    // trailing update: A(i, j) -= sum_c L(i, j0+c) L(j, j0+c), j0+pb <= j <= i;
    // rows by lane in 32-row chunks, columns by warp, four columns at a time
    const int t0 = j0 + pb;
    if (t0 < n) {
      const int nch = (n - t0 + 31) / 32;
#pragma unroll 1
      for (int ch = 0; ch < nch; ++ch) {
        const int i = t0 + ch * 32 + lane;
        const bool rowok = i < n;
        double li[PB];
#pragma unroll
        for (int c = 0; c < PB; ++c) {
          const double v = Pr[min(i, n - 1) * PB + c];
          li[c] = rowok ? v : 0.0;
        }
        const int jend = min(n, t0 + ch * 32 + 32);   // columns up to this chunk's last row
#pragma unroll 1
        for (int jb = t0 + 4 * warp; jb < jend; jb += 4 * CPW) {
          double acc[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int j = min(jb + u, n - 1);
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int c = 0; c < PB; c += 2) {
              s0 += li[c] * Pr[j * PB + c];
              s1 += li[c + 1] * Pr[j * PB + c + 1];
            }
            acc[u] = s0 + s1;
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int j = jb + u;
            if (rowok && j < jend && i >= j) AA(i, j) -= acc[u];
          }
        }
      }
    }
    __syncthreads();
  }
  if (bad) {
    if (tid == 0) *info = bad;
    return;
  }
  // ---------------- inverse ----------------
  const int nblk = (n + 31) / 32;
  // diagonal blocks: lane = column c of X_JJ, forward substitution down the
  // rows; X(r, c), r > c, goes to A(c, r), the diagonal to xd
  for (int J = warp; J < nblk; J += CPW) {
    const int j0 = J * 32, bs = min(32, n - j0);
    // rows past the matrix (last block) read row n - 1 and are zeroed
    double x[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) {
      const int rr = min(j0 + r, n - 1);
      double sum = (r == lane) ? 1.0 : 0.0;
#pragma unroll
      for (int k = 0; k < r; ++k) sum -= AA(rr, min(j0 + k, n - 1)) * x[k];
      x[r] = (r < bs) ? sum * rd[rr] : 0.0;
    }
    if (lane < bs) {
#pragma unroll
      for (int r = 0; r < 32; ++r) {
        if (r < bs && r > lane) AA(j0 + lane, j0 + r) = x[r];
        if (r == lane) xd[j0 + lane] = x[r];
      }
    }
  }
  __syncthreads();
  // M_IK = -X_II L_IK in place of L_IK, one warp per block; lane = row i,
  // which holds row i of X_II in registers
  for (int pair = warp; pair < nblk * (nblk - 1) / 2; pair += CPW) {
    int I = 1;
    while (I * (I + 1) / 2 <= pair) ++I;
    const int K = pair - I * (I - 1) / 2;
    const int i0 = I * 32, k0 = K * 32, bi = min(32, n - i0);
    const bool rowok = lane < bi;
    // row i of X_II (zero past the diagonal and for rows past the matrix);
    // loads from clamped addresses, selection after the load
    const int ir = min(i0 + lane, n - 1);
    double xr[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      const int kr = min(i0 + k, n - 1);
      const double v = AA(kr, ir), dv = xd[kr];
      xr[k] = (!rowok || k > lane || k >= bi) ? 0.0 : (k == lane ? dv : v);
    }
#pragma unroll 1
    for (int c = 0; c < 32; ++c) {   // the columns of block K are full (K < I)
      const double *col = &AA(0, k0 + c);
      double s0 = 0.0, s1 = 0.0;
#pragma unroll
      for (int k = 0; k < 32; k += 2) {
        s0 += xr[k] * col[min(i0 + k, n - 1)];
        s1 += xr[k + 1] * col[min(i0 + k + 1, n - 1)];
      }
      __syncwarp();
      if (rowok) AA(i0 + lane, k0 + c) = -(s0 + s1);
      __syncwarp();
    }
  }
  __syncthreads();
  // X_IJ = sum_{K=J}^{I-1} M_IK X_KJ by block diagonals; two warps a block
  // (16 columns each), lane = row i; X(k, c) for k > c read from A(c, k)
  for (int d = 1; d < nblk; ++d) {
    const int nb_d = nblk - d;
    for (int task = warp; task < nb_d * 2; task += CPW) {
      const int J = task >> 1, half = task & 1, I = J + d;
      const int i0 = I * 32, j0 = J * 32, bi = min(32, n - i0);
      const int cb = j0 + 16 * half;
      const int i = i0 + lane;
      const bool rowok = lane < bi;
      const int ir = min(i, n - 1);
      double acc[16], xdv[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        acc[u] = 0.0;
        xdv[u] = xd[cb + u];
      }
#pragma unroll 1
      for (int K = J; K < I; ++K) {
        const int k0 = K * 32;
#pragma unroll 1
        for (int kk = 0; kk < 32; ++kk) {
          const int k = k0 + kk;
          const double mv = AA(ir, k);
          const double m = rowok ? mv : 0.0;
          const double *xrow = &AA(cb, k);   // X(k, cb + u) = A(cb + u, k) for k > cb + u
#pragma unroll
          for (int u = 0; u < 16; ++u) {
            const int c = cb + u;
            const double xu = xrow[u];
            const double xv = (k > c) ? xu : ((k == c) ? xdv[u] : 0.0);
            acc[u] += m * xv;
          }
        }
      }
      if (rowok) {
#pragma unroll
        for (int u = 0; u < 16; ++u) AA(cb + u, i) = acc[u];   // X(i, c) to A(c, i)
      }
    }
    __syncthreads();
  }
  // out: X in the lower triangle, zeros above
  for (int j = warp; j < n; j += CPW)
    for (int i = lane; i < n; i += 32) Sg[(long)j * n + i] = (i > j) ? AA(j, i) : ((i == j) ? xd[j] : 0.0);
#undef AA
  if (tid == 0) *info = 0;
}

// Cholesky and L^-1 together with the matrix in registers (n <= W NR and
// n <= 32 NC; one CTA of W warps; thread (w, l) keeps rows NR w .. NR w + NR - 1
// of the columns l + 32 c).  X = L^-1 is found by rows (X L = I top down)
// with running right-hand sides R (R(i,:) = e_i at the start), stored where L
// was consumed.  Columns go two at a time (k, k + 1; NR even, so rows k and
// k + 1 sit in one warp): columns k and k + 1 (the Schur complement) are
// published and replaced by e_k, e_(k+1), which start R's columns; rows k
// and k + 1 (R(k, :), R(k+1, :)) are published; one barrier.  Then
// L(k,k) = sqrt(piv0), l = L(k+1,k), L(k+1,k+1) = sqrt(piv1 - l^2),
// m0_i = L(i,k), m1_i = L(i,k+1) and y0, y1 (the rows of X for the columns
// <= k + 1, the L columns beyond) give every row below k one rank-2 update
// a(i,:) -= m0_i y0 + m1_i y1: the Cholesky update of the columns > k + 1 and
// the forward-substitution update of the columns <= k + 1 (y0 is 0 at k + 1:
// that part of the Schur update is folded into piv1).  Rows k and k + 1 are
// final from then on and are scaled by their 1 / L(i,i) when written out.
// The gathered columns and rows alternate by parity, so one barrier a step
// suffices.  The matrix is staged through shared memory on the way in (the
// lower triangle, as rsdecmp reads it) and out (coalesced column-major
// stores).  info as k_cholinv_sm; S is left as it was on failure.
template <int W, int NR, int NC>
__global__ void __launch_bounds__(W * 32, 1) k_cholinv_rg(double *__restrict__ Sg, int n, int *__restrict__ info) {
  constexpr int NROW = W * NR, NCOL = 32 * NC;
  constexpr int NX = NROW > NCOL ? NROW : NCOL;
  static_assert(NR <= 32 && NR % 2 == 0, "lane r of a warp keeps m of row r; row pairs stay in one warp");
  extern __shared__ double stg[];   // n x (n | 1) staging
  __shared__ __align__(16) double xcol[2][2][NX];
  __shared__ __align__(16) double xrow[2][2][NX];
  __shared__ double rsv[NX];
  __shared__ double2 mw[W][NR];     // m0, m1 of each warp's rows (read back as broadcasts)
  const int ld = n | 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = warp * NR;
  // global to shared by cp.async: every copy of a thread in flight at once,
  // none through registers; element q = j n + i, stepped by the block size
  // without a division
  {
    int j = tid / n, i = tid - j * n;
    for (long q = tid; q < (long)n * n; q += W * 32) {
      const unsigned sa = (unsigned)__cvta_generic_to_shared(stg + (long)j * ld + i);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(Sg + q) : "memory");
      i += W * 32;
      while (i >= n) {
        i -= n;
        ++j;
      }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  }
  __syncthreads();
  double a[NR][NC];
#pragma unroll
  for (int r = 0; r < NR; ++r)
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const int row = r0 + r, col = lane + 32 * c;
      const int hi = row > col ? row : col, lo = row > col ? col : row;
      const double v = stg[(long)min(lo, n - 1) * ld + min(hi, n - 1)];   // S(hi, lo), clamped address
      a[r][c] = (row < n && col < n) ? v : 0.0;
    }
  for (int k = 0; k < n; k += 2) {
    const int b = (k >> 1) & 1, kc = k >> 5, kl = k & 31;   // k even: k and k + 1 share slot kc
    const bool two = k + 1 < n;
    if (lane == kl || (two && lane == kl + 1)) {   // columns k, k + 1 out, e_k, e_(k+1) in
      const int h = lane - kl, col = k + h;
      dense_static_for<0, NC>([&](auto cc) {
        constexpr int C = decltype(cc)::value;
        if (C == kc) {
#pragma unroll
          for (int r = 0; r < NR; r += 2) {
            *reinterpret_cast<double2 *>(&xcol[b][h][r0 + r]) = make_double2(a[r][C], a[r + 1][C]);
            a[r][C] = (r0 + r == col) ? 1.0 : 0.0;
            a[r + 1][C] = (r0 + r + 1 == col) ? 1.0 : 0.0;
          }
        }
      });
    }
    if (warp == k / NR) {     // rows k, k + 1 out
      const int kr = k - r0;
      dense_static_for<0, NR / 2>([&](auto rr) {
        constexpr int R = 2 * decltype(rr)::value;
        if (R == kr) {
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            xrow[b][0][lane + 32 * c] = a[R][c];
            xrow[b][1][lane + 32 * c] = a[R + 1][c];
          }
        }
      });
    }
    __syncthreads();
    const double *x0 = xcol[b][0], *x1 = xcol[b][1], *w0 = xrow[b][0], *w1 = xrow[b][1];
    const double piv0 = x0[k];
    if (!(piv0 > 1.0e-30)) {   // the same in every thread; also catches NaN
      if (tid == 0) *info = 1 + k;
      return;
    }
    const double rs0 = rsqrt_nr(piv0);   // 1 / L(k,k)
    const double l10 = two ? x0[k + 1] * rs0 : 0.0;
    double rs1 = 0.0;
    if (two) {
      const double piv1 = x1[k + 1] - l10 * l10;
      if (!(piv1 > 1.0e-30)) {
        if (tid == 0) *info = 2 + k;
        return;
      }
      rs1 = rsqrt_nr(piv1);
    }
    if (tid == 0) {
      rsv[k] = rs0;
      if (two) rsv[k + 1] = rs1;
    }
    // lane r < NR: m0, m1 of row r0 + r (0 where the row takes no update)
    const int ri = r0 + lane, rc = min(ri, NX - 1);
    const double m0row = (lane < NR && ri > k && ri < n) ? x0[rc] * rs0 : 0.0;
    const double m1row = (two && lane < NR && ri > k + 1 && ri < n) ? (x1[rc] - m0row * l10) * rs1 : 0.0;
    if (lane < NR) mw[warp][lane] = make_double2(m0row, m1row);
    __syncwarp();
    if (r0 + NR > k + 1) {    // rows below k in this warp
      double y0[NC], y1[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const int col = lane + 32 * c, cc = min(col, NX - 1);
        const double s0 = (col <= k) ? w0[cc] : x0[cc];
        const double s1 = (col <= k + 1) ? w1[cc] : x1[cc];
        y0[c] = (col == k + 1 || col >= n) ? 0.0 : s0 * rs0;
        y1[c] = (two && col < n) ? (s1 - l10 * y0[c]) * rs1 : 0.0;
      }
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const double2 mi = mw[warp][r];
#pragma unroll
        for (int c = 0; c < NC; ++c) a[r][c] = fma(-mi.y, y1[c], fma(-mi.x, y0[c], a[r][c]));
      }
    }
    __syncwarp();   // mw is rewritten in the next step
  }
  __syncthreads();
  // X to the staging area (lower triangle, zeros above), then out column-major
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const int row = r0 + r;
    const double sc = rsv[min(row, NX - 1)];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const int col = lane + 32 * c;
      if (row < n && col < n) stg[(long)col * ld + row] = (row >= col) ? a[r][c] * sc : 0.0;
    }
  }
  __syncthreads();
  {
    int j = tid / n, i = tid - j * n;
    for (long q = tid; q < (long)n * n; q += W * 32) {
      Sg[q] = stg[(long)j * ld + i];
      i += W * 32;
      while (i >= n) {
        i -= n;
        ++j;
      }
    }
  }
  if (tid == 0) *info = 0;
}

// Cholesky and L^-1 over the whole GPU for large n (one cooperative launch of
// G CTAs; the algorithm of k_cholinv_rg, one rank-1 update a column): CTA c
// keeps the columns j = c + G q in shared memory.  Step k: the owner of column
// k publishes it (the Schur complement) and replaces it by e_k; every CTA
// publishes its entries of row k (R(k, .) left of k); one grid barrier; then
// with rs = 1 / L(k,k), m_i = S(i,k) rs and y_j = R(k,j) rs (j <= k) or m_j
// (j > k), every CTA applies a(i,j) -= m_i y_j to the rows i > k of its
// columns.  Row k is final from then on and is scaled by rs when written out.
// The published column and row alternate by parity.  gs: 5n doubles of
// global scratch (column, row, 1/L(k,k)); bar: two zeroed unsigned ints.
// info as k_cholinv_sm (S left as it was on a bad pivot); -1 on a barrier
// time-out.
constexpr int CHG_T = 256;

__global__ void __launch_bounds__(CHG_T) k_cholinv_grid(double *__restrict__ Sg, int n, double *gs, unsigned *bar,
                                                        int *__restrict__ info) {
  const int G = gridDim.x, c = blockIdx.x;
  const int nq = (n + G - 1) / G;
  extern __shared__ double sm[];
  double *A = sm;                     // [nq][n]: column j = c + G q at A + q n
  double *mc = A + (long)nq * n;      // the published column of this step
  double *xcol = gs, *xrow = gs + 2 * (long)n, *rsv = gs + 4 * (long)n;
  __shared__ int ok;
  const int tid = threadIdx.x;
  if (tid == 0) ok = 1;
  // the lower triangle, as rsdecmp reads it
  for (long q = tid; q < (long)nq * n; q += CHG_T) {
    const int qq = (int)(q / n), i = (int)(q - (long)qq * n), j = c + G * qq;
    double v = 0.0;
    if (j < n) v = (i >= j) ? Sg[(long)j * n + i] : Sg[(long)i * n + j];
    A[q] = v;
  }
  __syncthreads();
  bool bad = false;
  for (int k = 0; k < n; ++k) {
    const int par = k & 1;
    double *xc = xcol + (long)par * n, *xr = xrow + (long)par * n;
    if (c == k % G) {
      double *col = A + (long)(k / G) * n;
      for (int i = tid; i < n; i += CHG_T) {
        xc[i] = col[i];
        col[i] = (i == k) ? 1.0 : 0.0;
      }
    }
    __syncthreads();
    for (int q = tid; q < nq; q += CHG_T) {
      const int j = c + G * q;
      if (j < n) xr[j] = A[(long)q * n + k];
    }
    if (!grid_barrier(bar, G, &ok)) break;
    const double piv = __ldcg(xc + k);
    if (!(piv > 1.0e-30)) {   // the same in every CTA; also catches NaN
      if (c == 0 && tid == 0) *info = 1 + k;
      bad = true;
      break;
    }
    const double rs = rsqrt_nr(piv);
    if (c == 0 && tid == 0) rsv[k] = rs;
    for (int i = k + 1 + tid; i < n; i += CHG_T) mc[i] = __ldcg(xc + i) * rs;
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31;
    for (int q = warp; q < nq; q += CHG_T / 32) {
      const int j = c + G * q;
      if (j >= n) break;   // uniform in the warp
      const double y = ((j <= k) ? __ldcg(xr + j) : __ldcg(xc + j)) * rs;
      double *col = A + (long)q * n;
      for (int i = k + 1 + lane; i < n; i += 32) col[i] = fma(-mc[i], y, col[i]);
    }
    __syncthreads();
  }
  if (bad) return;
  if (!grid_barrier(bar, G, &ok) || !ok) {
    if (tid == 0) atomicExch(info, -1);
    return;
  }
  // X: row i scaled by 1 / L(i,i), zeros above the diagonal
  for (long q = tid; q < (long)nq * n; q += CHG_T) {
    const int qq = (int)(q / n), i = (int)(q - (long)qq * n), j = c + G * qq;
    if (j < n) Sg[(long)j * n + i] = (i >= j) ? A[q] * __ldcg(rsv + i) : 0.0;
  }
  if (c == 0 && tid == 0 && *info >= 0) *info = 0;
}

// The cooperative Cholesky + inverse when the columns fit one CTA per SM and
// cooperative launch is available; false if it was not launched.  work:
// at least 5n doubles + 2 unsigned ints.  QX_CHOLINV_GRID=0 turns it off
// (read at every call).
static bool cholinv_grid(double *S, int n, double *work, int *d_info, cudaStream_t st) {
  const char *env = getenv("QX_CHOLINV_GRID");
  if ((env && env[0] == '0') || !work) return false;
  int dev = 0, nsm = 0, coop = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) return false;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return false;
  const int G = std::min(nsm, n);
  const int nq = (n + G - 1) / G;
  const size_t sm = sizeof(double) * ((size_t)nq * n + (size_t)n);
  if (sm > 200 * 1024) return false;
  static size_t sm_set = 0;   // per process: set at the first call, then only ever raised
  if (sm > sm_set) {
    if (cudaFuncSetAttribute(k_cholinv_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
      return false;
    sm_set = 200 * 1024;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cholinv_grid, CHG_T, sm) != cudaSuccess ||
      per_sm < 1)
    return false;
  double *gs = work;
  unsigned *bar = reinterpret_cast<unsigned *>(work + 5L * n);
  if (cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), st) != cudaSuccess ||
      cudaMemsetAsync(d_info, 0, sizeof(int), st) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  void *args[] = {(void *)&S, (void *)&n, (void *)&gs, (void *)&bar, (void *)&d_info};
  if (cudaLaunchCooperativeKernel((const void *)k_cholinv_grid, dim3(G), dim3(CHG_T), args, sm, st) !=
      cudaSuccess) {
    cudaGetLastError();   // not launched: the one-CTA kernels run instead
    return false;
  }
  note_launch();
  return true;
}

// QX_CHOLINV_REG=0 keeps the shared-memory kernels at every size (read at
// every call).
static bool cholinv_registers_enabled() {
  const char *v = getenv("QX_CHOLINV_REG");
  return !(v && v[0] == '0');
}

// S: n x n column-major.  When S does not fit shared memory the kernel works
// in S itself (L2-resident) and uses work (>= CB*DLD + n doubles) as temporary.
int cholinv(double *S, int n, double *work, int *d_info, cudaStream_t st) {
  if (n > 8192) { set_error("cholinv: n=%d too large", n); return 1; }
  const size_t bytes = sizeof(double) * ((size_t)(n | 1) * n + CB * DLD + n);
  const int use = bytes <= CH_SMEM_MAX;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_cholinv<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CH_SMEM_MAX);
    attr = true;
  }
  if (!use && !work) { set_error("cholinv: n=%d needs a work buffer", n); return 1; }
  const size_t pbytes = sizeof(double) * ((size_t)(n | 1) * n + 2 * (size_t)n + (size_t)PB * n);
  const size_t rbytes = sizeof(double) * (size_t)(n | 1) * n;
  if (n <= 160 && cholinv_registers_enabled()) {
    // per process, only ever raised; the first call always sets it (the
    // kernels' static shared buffers count against the 48 KB default, so a
    // dynamic size below 48 KB can still need the opt-in)
    static size_t rset = 0;
    if (rbytes > rset) {
      // exactly what this size needs: with the kernels' static buffers the
      // opt-in ceiling is below the 227 KB of a CTA
      const cudaError_t e1 = cudaFuncSetAttribute(k_cholinv_rg<8, 10, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)rbytes);
      const cudaError_t e2 = cudaFuncSetAttribute(k_cholinv_rg<8, 20, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)rbytes);
      if (e1 != cudaSuccess || e2 != cudaSuccess) {
        set_error("cholinv: n=%d: shared-memory opt-in failed: %s", n, cudaGetErrorString(e1 ? e1 : e2));
        return 1;
      }
      rset = rbytes;
    }
    if (n <= 80) k_cholinv_rg<8, 10, 3><<<1, 8 * 32, rbytes, st>>>(S, n, d_info);
    else k_cholinv_rg<8, 20, 5><<<1, 8 * 32, rbytes, st>>>(S, n, d_info);
    note_launch();
    return 0;
  }
  if (n > 192 && cholinv_grid(S, n, work, d_info, st)) return 0;
  if (n <= CP_MAXN && pbytes <= CH_SMEM_MAX) {
    static bool pattr = false;
    if (!pattr) {
      cudaFuncSetAttribute(k_cholinv_sm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CH_SMEM_MAX);
      pattr = true;
    }
    k_cholinv_sm<<<1, CPT, pbytes, st>>>(S, n, d_info);
    note_launch();
    return 0;
  }
  if (use) k_cholinv<true><<<1, CHT, bytes, st>>>(S, n, work, d_info);
  else k_cholinv<false><<<1, CHT, 0, st>>>(S, n, work, d_info);
  note_launch();
  return 0;
}

// --------------------------------------------------------------------------
// Symmetric eigen-decomposition of the subspace Hamiltonian (the role of
// RsEIGQR, funcs.f90:380-764, which also reduces to tridiagonal form by
// Householder reflections):
//  (1) k_sytrd: Householder tridiagonalisation T = Q^T A Q in one CTA, three
//      barriers per column (reflector, matrix-vector product, rank-2 update);
//  (2) k_bisect: eigenvalues of T by Sturm-count multisection, one warp per
//      eigenvalue, 33 subintervals per round, division-free counts;
//  (3) k_invit: eigenvectors of T by inverse iteration with a pivoted
//      tridiagonal LU, one thread per cluster of close eigenvalues, members
//      re-orthogonalised against each other; per-thread work arrays are
//      interleaved across threads so every access is coalesced;
//  (4) k_wy_t + k_backtrans_wy: V = Q Z, one warp per column, the reflectors
//      in compact-WY blocks of 8; for n > 256 k_backtrans_tile, one CTA per 8
//      columns held in shared memory, the same blocks (QX_BACKTRANS_TILE=0:
//      k_backtrans, one warp per column and one reflector at a time).
// Eigenpairs are ascending; each eigenvector's largest-magnitude component is
// made positive (first index on ties).  Every loop is bounded.

constexpr int TRD_T = 1024;
constexpr size_t TRD_SMEM_MAX = 222 * 1024;

// 1/x to full double precision: approximate reciprocal and two Newton-Raphson
// steps r <- r (2 - x r).
__device__ __forceinline__ double recip2_nr(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  r = r * fma(-x, r, 2.0);
  return r * fma(-x, r, 2.0);
}

// Householder reflector of x (GVL house): P = I - tau v v^T, v(0) = 1,
// P x = |x| e1.  Returns tau, writes 1/beta (v = x / beta for i >= 1) and
// |x|.  Square root and divisions by Newton-refined hardware approximations
// (rsqrt_nr, recip2_nr): this is on the critical path of every column.
__device__ __forceinline__ void house(double x0, double sigma, double &tau, double &rbeta, double &alpha) {
  if (sigma == 0.0) {
    tau = (x0 < 0.0) ? 2.0 : 0.0;
    rbeta = 1.0;
    alpha = fabs(x0);
    return;
  }
  const double s2 = x0 * x0 + sigma;
  const double mu = s2 * rsqrt_nr(s2);
  const double v1 = (x0 <= 0.0) ? x0 - mu : -sigma * recip2_nr(x0 + mu);
  const double v1s = v1 * v1;
  tau = 2.0 * v1s * recip2_nr(sigma + v1s);
  rbeta = recip2_nr(v1);
  alpha = mu;
}

// Per column k (m = n-k-1 trailing rows): warp 0 forms the reflector from
// column k (which it updated itself in step k-1), then three barriers:
// (1) reflector published; (2) matrix-vector product B v in 4 column groups
// of 32-row strips, partial sums to `part`; (3) p = t * sum of the groups.
// The rank-2 update B -= v w^T + w v^T (w = p - K v) is spread by columns
// over the warps and needs no barrier of its own: v, and the scalars, are
// double-buffered by column parity, so warp 0 can form the next reflector
// while other warps finish this update, and the next matrix-vector product
// starts only after barrier (1) of the next column.
// gvec: 7n doubles of global memory for v (two buffers), p and part when A
// is not in shared memory.
template <bool USE_SMEM>
__global__ void __launch_bounds__(TRD_T) k_sytrd(double *__restrict__ Ag, int n, double *__restrict__ d,
                                                 double *__restrict__ e, double *__restrict__ HV,
                                                 double *__restrict__ tau, double *__restrict__ gvec) {
  constexpr bool use_smem = USE_SMEM;
  extern __shared__ double sm[];
  __shared__ double sc[2];
  const int ld = use_smem ? (n | 1) : n;
  double *A = use_smem ? sm : Ag;
  double *vb = use_smem ? sm + (long)ld * n : gvec;   // 2 x n
  double *p = vb + 2 * (long)n;                       // n
  double *part = p + n;                               // 4 x n
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = TRD_T / 32, NG = 4;
#define A_(i, j) A[(long)(j) * ld + (i)]
  if (use_smem)
    for (long q = tid; q < (long)n * n; q += TRD_T) {
      const int j = (int)(q / n), i = (int)(q - (long)j * n);
      A_(i, j) = Ag[q];
    }
  __syncthreads();
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;
    double *v = vb + (k & 1) * (long)n;
    if (warp == 0) {
      double sg = 0.0;
      for (int i = 1 + lane; i < m; i += 32) { const double x = A_(k + 1 + i, k); sg += x * x; }
      sg = warp_sum(sg);
      double t = 0.0, rb = 1.0, al = 0.0;
      if (lane == 0) house(A_(k + 1, k), sg, t, rb, al);
      t = __shfl_sync(0xffffffffu, t, 0);
      const double rbe = __shfl_sync(0xffffffffu, rb, 0);
      for (int i = lane; i < m; i += 32) {
        const double vi = (i == 0) ? 1.0 : ((t != 0.0) ? A_(k + 1 + i, k) * rbe : 0.0);
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
    __syncthreads();                                   // (1)
    const double t = sc[k & 1];
    if (t == 0.0) continue;                            // uniform
    const int nrb = (m + 31) >> 5;
    for (int task = warp; task < nrb * NG; task += NW) {
      const int rb = task / NG, g = task - rb * NG, i = rb * 32 + lane;
      if (i < m) {
        const double *__restrict__ col = &A_(k + 1 + i, k + 1);
        const double *__restrict__ vv = v;
        double s0 = 0.0, s1 = 0.0;
        int j = g;
        for (; j + NG < m; j += 2 * NG) {
          s0 += col[(long)j * ld] * vv[j];
          s1 += col[(long)(j + NG) * ld] * vv[j + NG];
        }
        if (j < m) s0 += col[(long)j * ld] * vv[j];
        part[g * n + i] = s0 + s1;
      }
    }
    __syncthreads();                                   // (2)
    for (int i = tid; i < m; i += TRD_T) p[i] = t * (part[i] + part[n + i] + part[2 * n + i] + part[3 * n + i]);
    __syncthreads();                                   // (3)
    double kk = 0.0;
    for (int i = lane; i < m; i += 32) kk += v[i] * p[i];
    const double K = 0.5 * t * warp_sum(kk);
    // rows of this lane: i = lane + 32 q; their v and w in registers when
    // m <= 32 * RQ, otherwise reloaded per column
    constexpr int RQ = 6;
    double vi[RQ], wi[RQ];
#pragma unroll
    for (int q = 0; q < RQ; ++q) {
      const int i = lane + 32 * q;
      vi[q] = (i < m) ? v[i] : 0.0;
      wi[q] = (i < m) ? p[i] - K * vi[q] : 0.0;
    }
    // warp 0 updates only column 0 of B (the next reflector's column) and then
    // goes on to form the next reflector while warps 1..31 update the rest
    for (int j = (warp == 0) ? 0 : warp; j < m; j += (warp == 0) ? m : NW - 1) {
      const double vj = v[j], wj = p[j] - K * vj;
      double *__restrict__ col = &A_(k + 1, k + 1 + j);
      if (m <= 32 * RQ) {
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
          const int i = lane + 32 * q;
          if (i < m) col[i] -= vi[q] * wj + wi[q] * vj;
        }
      } else {
        for (int i = lane; i < m; i += 32) {
          const double a = v[i], b = p[i] - K * a;
          col[i] -= a * wj + b * vj;
        }
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    if (n >= 2) {
      d[n - 2] = A_(n - 2, n - 2);
      e[n - 2] = A_(n - 1, n - 2);
    }
    d[n - 1] = A_(n - 1, n - 1);
  }
#undef A_
}

// The same tridiagonalisation with the whole matrix in registers (n <= W NR
// and n <= 32 NC; one CTA of W warps): warp w holds rows NR w .. NR w + NR - 1,
// lane l the columns l + 32 c, so thread (w, l) keeps an NR x NC block and no
// element of A passes through shared memory after the load.  Per column k,
// three barriers:
//   (1) lane k mod 32 of every warp has put its piece of column k (and the
//       partial sum of squares below the subdiagonal) in shared memory; every
//       thread then forms the same reflector (house) and its own v entries;
//   (2) column partial sums of A v over each warp's rows are in shared memory
//       (A is symmetric, so (A v)_j is a column sum);
//   (3) p = tau A v is summed, zero for rows <= k; every warp forms
//       K = tau v^T p / 2, w = p - K v, and updates its block in registers:
//       A_ij -= v_i w_j + w_i v_j (rows and columns <= k have v = w = 0).
// The column buffer and the sums of squares alternate by column parity, so a
// warp that gathers column k + 1 never overwrites what a slower warp still
// reads for column k.  A must be symmetric; it is read by rows (coalesced).
template <int TRR_W, int NR, int NC>
__global__ void __launch_bounds__(TRR_W * 32, 1)
    k_sytrd_rg(const double *__restrict__ Ag, int n, double *__restrict__ d, double *__restrict__ e,
               double *__restrict__ HV, double *__restrict__ tau) {
  constexpr int NROW = TRR_W * NR, NCOL = 32 * NC;
  static_assert(NROW <= NCOL, "p is indexed by rows and by columns");
  static_assert(NR <= 32, "lane r of a warp keeps v and w of the warp's row r");
  __shared__ __align__(16) double xs[2][NROW];
  __shared__ double sigp[2][TRR_W];
  __shared__ double part[TRR_W][NCOL];
  __shared__ double ps[NCOL];
  __shared__ double vsm[TRR_W][NR], wsm[TRR_W][NR];   // v, w of each warp's rows (read back as broadcasts)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = warp * NR;
  double a[NR][NC];
#pragma unroll
  for (int r = 0; r < NR; ++r)
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const int row = r0 + r, col = lane + 32 * c;
      a[r][c] = (row < n && col < n) ? Ag[(long)row * n + col] : 0.0;
    }
  // column kk of A into xs[b] (all rows); sum of squares of rows > kk + 1 into sigp[b]
  auto gather = [&](int kk, int b) {
    if (lane == (kk & 31)) {
      const int kc = kk >> 5;
      dense_static_for<0, NC>([&](auto cc) {
        constexpr int C = decltype(cc)::value;
        if (C == kc) {
          double sg[2] = {0.0, 0.0};
#pragma unroll
          for (int r = 0; r < NR; r += 2) {
            const double x0 = a[r][C], x1 = a[r + 1][C];
            *reinterpret_cast<double2 *>(&xs[b][r0 + r]) = make_double2(x0, x1);
            sg[0] += (r0 + r > kk + 1) ? x0 * x0 : 0.0;
            sg[1] += (r0 + r + 1 > kk + 1) ? x1 * x1 : 0.0;
          }
          sigp[b][warp] = sg[0] + sg[1];
        }
      });
    }
  };
  for (int k = 0; k + 2 < n; ++k) {
    const int b = k & 1;
    gather(k, b);
    __syncthreads();                                                   // (1)
    double sigma = 0.0;
#pragma unroll
    for (int w = 0; w < TRR_W; ++w) sigma += sigp[b][w];
    double t = 0.0, rb = 1.0, al = 0.0;
    house(xs[b][k + 1], sigma, t, rb, al);
    const double *x = xs[b];
    // v(i) = 1 at k + 1, x_i / beta below, 0 elsewhere (all of v is e1 when
    // tau = 0); the load is unconditional (clamped index) and the selection
    // follows, so unrolled uses do not serialise on it
    auto vof = [&](int i) {
      const double xv = x[min(i, NROW - 1)] * rb;
      return (i == k + 1) ? 1.0 : ((i > k + 1 && i < n && t != 0.0) ? xv : 0.0);
    };
    if (tid == 0) {
      tau[k] = t;
      d[k] = x[k];
      e[k] = al;
    }
    for (int i = k + 1 + tid; i < n; i += TRR_W * 32) HV[(long)k * n + i] = vof(i);
    if (t == 0.0) continue;                                            // same in every thread
    const bool rows_active = r0 + NR > k + 1;                          // uniform in the warp
    // lane r < NR keeps v of row r0 + r; the warp reads it by shuffles
    const double vrow = (lane < NR) ? vof(r0 + lane) : 0.0;
    if (lane < NR) vsm[warp][lane] = vrow;
    __syncwarp();
    // The product and the update for column k, compiled once for each first
    // live column slot P = k / 32: the columns j <= k of slots below P are
    // never read again (the product's entries j <= k are masked, the next
    // columns gathered are > k), so their FMAs are left out.  P is a
    // compile-time constant in each copy, so no branch sits inside the
    // unrolled loops; the result is the same bit for bit.
    auto product_update = [&](auto pc) {
      constexpr int P = decltype(pc)::value;
      {
        double sc[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) sc[c] = 0.0;
        if (rows_active) {
#pragma unroll
          for (int r = 0; r < NR; ++r) {
            const double vr = vsm[warp][r];
#pragma unroll
            for (int c = P; c < NC; ++c) sc[c] = fma(a[r][c], vr, sc[c]);
          }
        }
#pragma unroll
        for (int c = P; c < NC; ++c) part[warp][lane + 32 * c] = sc[c];
      }
      __syncthreads();                                                 // (2)
      for (int j = 32 * P + tid; j < NCOL; j += TRR_W * 32) {
        double acc = 0.0;
#pragma unroll
        for (int w = 0; w < TRR_W; ++w) acc += part[w][j];
        ps[j] = (j > k && j < n) ? t * acc : 0.0;
      }
      __syncthreads();                                                 // (3)
      double kk = 0.0;
#pragma unroll
      for (int c = P; c < NC; ++c) kk = fma(vof(lane + 32 * c), ps[lane + 32 * c], kk);
      const double K = 0.5 * t * warp_sum(kk);
      // p of rows <= k is zero (ps below slot P is not rewritten in this copy)
      const double prow = (r0 + lane > k) ? ps[min(r0 + lane, NCOL - 1)] : 0.0;
      const double wrow = (lane < NR) ? fma(-K, vrow, prow) : 0.0;
      if (lane < NR) wsm[warp][lane] = wrow;
      __syncwarp();
      // A -= v w^T, then A -= w v^T: each pass keeps one vector of the
      // lane's columns live beside the block
      if (rows_active) {
        double wc[NC];
#pragma unroll
        for (int c = P; c < NC; ++c) wc[c] = fma(-K, vof(lane + 32 * c), ps[lane + 32 * c]);
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const double vi = vsm[warp][r];
#pragma unroll
          for (int c = P; c < NC; ++c) a[r][c] = fma(-vi, wc[c], a[r][c]);
        }
        double vc[NC];
#pragma unroll
        for (int c = P; c < NC; ++c) vc[c] = vof(lane + 32 * c);
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const double wi = wsm[warp][r];
#pragma unroll
          for (int c = P; c < NC; ++c) a[r][c] = fma(-wi, vc[c], a[r][c]);
        }
      }
    };
    const int pk = k >> 5;   // uniform: every thread takes the same copy
    dense_static_for<0, NC>([&](auto pc) {
      if (decltype(pc)::value == pk) product_update(pc);
    });
    __syncwarp();   // vsm, wsm are rewritten in the next step
  }
  // the last 2 x 2 block
  if (n >= 2) {
    gather(n - 2, 0);
    __syncthreads();
    if (tid == 0) {
      d[n - 2] = xs[0][n - 2];
      e[n - 2] = xs[0][n - 1];
    }
  }
  gather(n - 1, 1);
  __syncthreads();
  if (tid == 0) d[n - 1] = xs[1][n - 1];
}

// Householder tridiagonalisation over the whole GPU for large n (one
// cooperative launch of G CTAs, the role of k_sytrd when the matrix does not
// fit one SM): CTA c keeps the columns j = c + G q of A in shared memory.
// Per column k (m = n - k - 1 trailing rows), two grid barriers:
//   (1) the owner of column k has formed the reflector (house) and written v
//       (and tau) to global memory;
//   (2) every CTA has written p_j = tau (A v)_j for its columns (column dot
//       products: A is symmetric) and its part of v^T p;
// then every CTA forms K = tau v^T p / 2 (the G parts in a fixed order),
// w = p - K v, and updates its own columns, A_ij -= v_i w_j + w_i v_j.  v
// alternates between two buffers by column parity; p and the parts are
// rewritten only after the next barrier (1), which every CTA reaches after
// its reads.  gs: 3n + G + 2 doubles of global scratch; bar: two zeroed
// unsigned ints.  On a barrier time-out *info is made negative.
constexpr int TRG_T = 256;

__global__ void __launch_bounds__(TRG_T) k_sytrd_grid(const double *__restrict__ Ag, int n, double *__restrict__ d,
                                                      double *__restrict__ e, double *__restrict__ HV,
                                                      double *__restrict__ tau, double *gs, unsigned *bar,
                                                      int *info) {
  const int G = gridDim.x, c = blockIdx.x;
  const int nq = (n + G - 1) / G;
  extern __shared__ double sm[];
  double *A = sm;                     // [nq][n]: column j = c + G q at A + q n
  double *vs = A + (long)nq * n;      // v by row
  double *pw = vs + n;                // p by row
  double *vbuf = gs, *pbuf = gs + 2 * (long)n, *kpart = gs + 3 * (long)n, *tbuf = kpart + G;
  __shared__ double red[TRG_T / 32];
  __shared__ double tK[2];
  __shared__ int ok;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = TRG_T / 32;
  if (tid == 0) ok = 1;
  for (long q = tid; q < (long)nq * n; q += TRG_T) {
    const int qq = (int)(q / n), i = (int)(q - (long)qq * n), j = c + G * qq;
    A[q] = (j < n) ? Ag[(long)j * n + i] : 0.0;
  }
  __syncthreads();
  for (int k = 0; k + 2 < n; ++k) {
    const int own = k % G, par = k & 1;
    double *vb = vbuf + (long)par * n;
    if (c == own && warp == 0) {
      const double *col = A + (long)(k / G) * n;
      double sg = 0.0;
      for (int i = k + 2 + lane; i < n; i += 32) {
        const double x = col[i];
        sg += x * x;
      }
      sg = warp_sum(sg);
      double t = 0.0, rb = 1.0, al = 0.0;
      if (lane == 0) house(col[k + 1], sg, t, rb, al);
      t = __shfl_sync(0xffffffffu, t, 0);
      const double rbe = __shfl_sync(0xffffffffu, rb, 0);
      for (int i = k + 1 + lane; i < n; i += 32) {
        const double vi = (i == k + 1) ? 1.0 : ((t != 0.0) ? col[i] * rbe : 0.0);
        vb[i] = vi;
        HV[(long)k * n + i] = vi;
      }
      if (lane == 0) {
        tau[k] = t;
        d[k] = col[k];
        e[k] = al;
        tbuf[par] = t;
      }
    }
    if (!grid_barrier(bar, G, &ok)) break;                        // (1)
    const double t = __ldcg(tbuf + par);
    if (t == 0.0) continue;                                        // the same in every CTA
    for (int i = k + 1 + tid; i < n; i += TRG_T) vs[i] = __ldcg(vb + i);
    __syncthreads();
    const int q_lo = (k + 1 > c) ? (k + 1 - c + G - 1) / G : 0;
    double kk = 0.0;
    for (int q = q_lo + warp; q < nq; q += NW) {
      const int j = c + G * q;
      if (j >= n) break;                                           // uniform in the warp
      const double *col = A + (long)q * n;
      double s0 = 0.0, s1 = 0.0;
      int i = k + 1 + lane;
      for (; i + 32 < n; i += 64) {
        s0 += col[i] * vs[i];
        s1 += col[i + 32] * vs[i + 32];
      }
      if (i < n) s0 += col[i] * vs[i];
      const double pj = t * warp_sum(s0 + s1);
      if (lane == 0) {
        pbuf[j] = pj;
        kk += vs[j] * pj;
      }
    }
    if (lane == 0) red[warp] = kk;
    __syncthreads();
    if (tid == 0) {
      double x = 0.0;
      for (int w = 0; w < NW; ++w) x += red[w];
      kpart[c] = x;
    }
    if (!grid_barrier(bar, G, &ok)) break;                        // (2)
    if (warp == 0) {
      double x = 0.0;
      for (int r = lane; r < G; r += 32) x += __ldcg(kpart + r);
      x = warp_sum(x);
      if (lane == 0) tK[1] = 0.5 * t * x;
    }
    for (int i = k + 1 + tid; i < n; i += TRG_T) pw[i] = __ldcg(pbuf + i);
    __syncthreads();
    const double K = tK[1];
    for (int q = q_lo + warp; q < nq; q += NW) {
      const int j = c + G * q;
      if (j >= n) break;
      const double vj = vs[j], wj = pw[j] - K * vj;
      double *col = A + (long)q * n;
      for (int i = k + 1 + lane; i < n; i += 32) {
        const double vi = vs[i], wi = pw[i] - K * vi;
        col[i] -= vi * wj + wi * vj;
      }
    }
    __syncthreads();
  }
  __syncthreads();
  if (!ok) {
    if (tid == 0) atomicExch(info, -(1 << 30));
    return;
  }
  if (tid == 0) {
    if (n >= 2 && c == (n - 2) % G) {
      const double *col = A + (long)((n - 2) / G) * n;
      d[n - 2] = col[n - 2];
      e[n - 2] = col[n - 1];
    }
    if (c == (n - 1) % G) d[n - 1] = A[(long)((n - 1) / G) * n + n - 1];
  }
}

// Number of eigenvalues of T below x: sign changes of the Sturm sequence
// p_0 = 1, p_1 = d_0 - x, p_i = (d_{i-1} - x) p_{i-1} - e_{i-2}^2 p_{i-2}
// (zeros dropped).  No division on the dependent chain (one FMA a step; the
// ratio form q_i = p_i / p_{i-1} needs a reciprocal a step); every 8 steps
// both terms are rescaled by a power of two, which changes no sign.  d and
// e2 = e^2 are read from shared memory (broadcasts), eight steps at a time.
__device__ __forceinline__ void sturm_step(double di, double e2, double x, double &p1, double &p2, bool &neg,
                                           int &c) {
  const double p = fma(di - x, p1, -e2 * p2);
  if (p != 0.0) {
    const bool ng = p < 0.0;
    c += (ng != neg) ? 1 : 0;
    neg = ng;
  }
  p2 = p1;
  p1 = p;
}
__device__ __forceinline__ void sturm_rescale(double &p1, double &p2) {
  const double m = fmax(fabs(p1), fabs(p2));
  if (m > 0.0 && m < 1e300) {
    const int ex = (int)((__double_as_longlong(m) >> 52) & 0x7ff);
    const double sc = __longlong_as_double((long long)(2046 - ex) << 52);   // 2^(1023 - ex)
    p1 *= sc;
    p2 *= sc;
  }
}
__device__ __forceinline__ int sturm_count(const double *__restrict__ d, const double *__restrict__ e2, int n,
                                           double x) {
  double p2 = 1.0, p1 = d[0] - x;
  int c = p1 < 0.0 ? 1 : 0;
  bool neg = p1 < 0.0;   // sign of the last nonzero term
  int i = 1;
  for (; i + 8 <= n; i += 8) {
    double dd[8], ee[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) { dd[u] = d[i + u]; ee[u] = e2[i + u - 1]; }
#pragma unroll
    for (int u = 0; u < 8; ++u) sturm_step(dd[u], ee[u], x, p1, p2, neg, c);
    sturm_rescale(p1, p2);
  }
  for (; i < n; ++i) sturm_step(d[i], e2[i - 1], x, p1, p2, neg, c);
  return c;
}

// Eigenvalue t of T (ascending) by multisection: each round the 32 lanes of
// warp t count the eigenvalues below 32 interior points of [lo, hi] and the
// interval shrinks to the one of 33 parts that holds eigenvalue t, until it
// is 2 eps |T| wide (at most 24 rounds).
__global__ void k_bisect(const double *__restrict__ d, const double *__restrict__ e, int n, double *__restrict__ w) {
  const int t = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  extern __shared__ double bs_de[];   // d (n), then e^2 (n - 1)
  if (t >= n) return;   // whole warp (one warp per block)
  double *sd = bs_de, *se2 = bs_de + n;
  double lo = 1e300, hi = -1e300, tn = 0.0;
  for (int i = lane; i < n; i += 32) {
    const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
    tn = fmax(tn, fabs(d[i]) + r);
    sd[i] = d[i];
    if (i < n - 1) se2[i] = e[i] * e[i];
  }
  __syncwarp();
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    tn = fmax(tn, __shfl_xor_sync(0xffffffffu, tn, o));
  }
  const double eps = 2.220446049250313e-16;
  lo -= 2.0 * eps * tn + 1e-300;
  hi += 2.0 * eps * tn + 1e-300;
  for (int it = 0; it < 24; ++it) {
    if (hi - lo <= 2.0 * eps * tn + 1e-290) break;
    const double h = (hi - lo) * (1.0 / 33.0);
    const double x = lo + (double)(lane + 1) * h;
    const int c = sturm_count(sd, se2, n, x);
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
// With SMT > 0 the six arrays live in shared memory instead, interleaved
// across the block's threads (6 * n * blockDim doubles).  d and e are staged
// in shared memory behind them (2n doubles) so that no global load sits on
// the dependent chains of the factorisation and the solves.
template <int SMT>
__global__ void k_invit(const double *__restrict__ dg, const double *__restrict__ eg, const double *__restrict__ w,
                        int n, double *__restrict__ Z, double *__restrict__ wsg, int NTg, int *__restrict__ nclus) {
  // SMT > 0: the work arrays in shared memory for blocks of SMT threads
  // (compile-time stride, shared-memory addressing); SMT == 0: global memory
  extern __shared__ double wss[];
  double *d = wss + (SMT ? 6 * n * SMT : 0), *e = d + n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[i] = dg[i];
    e[i] = (i < n - 1) ? eg[i] : 0.0;
  }
  __syncthreads();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double *ws = SMT ? wss : wsg;
  const int NT = SMT ? SMT : NTg;
  const int tt = SMT ? (int)threadIdx.x : t;
  double tn = 0.0;
#pragma unroll 4
  for (int i = 0; i < n; ++i)
    tn = fmax(tn, fabs(d[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0) + fabs(e[i]));
  const double eps = 2.220446049250313e-16;
  const double gaptol = 1e-6 * tn;
  if (t > 0 && w[t] - w[t - 1] < gaptol) return;   // not a cluster head
  atomicAdd(nclus, 1);
  int tend = t + 1;
  while (tend < n && w[tend] - w[tend - 1] < gaptol) ++tend;
#define WS(a, i) ws[((a) * n + (i)) * NT + tt]
  // 0: 1/U(i,i), 1: U(i,i+1), 2: U(i,i+2), 3: multiplier, 4: row swap flag, 5: z
  const double tiny = eps * tn + 1e-300;
  for (int c = t; c < tend; ++c) {
    // perturb members apart so their LU factors differ
    const double lam = w[c] + (double)(c - t) * 4.0 * eps * tn;
    double a = d[0] - lam, b = (n > 1) ? e[0] : 0.0;
    // branch-free: both pivot choices are formed and one is selected, so no
    // load or store of a step waits on the comparison of the previous one
#pragma unroll 2
    for (int i = 0; i < n - 1; ++i) {
      const double cdn = e[i];                 // subdiagonal below a
      const double dn = d[i + 1] - lam;        // next diagonal
      const double en = e[i + 1];              // e[n - 1] is staged as 0
      // reciprocals by Newton-refined hardware approximations (recip2_nr,
      // full double precision up to the last bit or two): inverse iteration
      // needs an accurate factorisation of a nearby matrix, not correctly
      // rounded quotients
      const bool keep = fabs(a) >= fabs(cdn);  // no row interchange
      const double aa = (fabs(a) < tiny) ? tiny : a;
      const double r = recip2_nr(keep ? aa : cdn);
      const double l = (keep ? cdn : a) * r;
      WS(0, i) = r;
      WS(1, i) = keep ? b : dn;
      WS(2, i) = keep ? 0.0 : en;
      WS(3, i) = l;
      WS(4, i) = keep ? 0.0 : 1.0;
      const double an = keep ? dn - l * b : b - l * dn;
      b = keep ? en : -l * en;
      a = an;
    }
    WS(0, n - 1) = recip2_nr((fabs(a) < tiny) ? tiny : a);
    // start vector: ones with a member-dependent pattern
    for (int i = 0; i < n; ++i) WS(5, i) = 1.0 + 0.01 * (double)((i * (c + 3)) % 7);
    // an isolated eigenvalue (bisected to 2 eps |T|) needs two solves; the
    // members of a cluster, re-orthogonalised each round, get three
    const int nit = (tend - t == 1) ? 2 : 3;
    for (int it = 0; it < nit; ++it) {
      // forward: row interchanges and multipliers
      double zi = WS(5, 0);
#pragma unroll 4
      for (int i = 0; i < n - 1; ++i) {
        const double zn = WS(5, i + 1), l = WS(3, i);
        const bool sw = WS(4, i) != 0.0;      // rows i, i+1 swapped
        WS(5, i) = sw ? zn : zi;
        zi = sw ? zi - l * zn : zn - l * zi;
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
#pragma unroll 4
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
      double nr4[4] = {0.0, 0.0, 0.0, 0.0};
      int i4 = 0;
      for (; i4 + 4 <= n; i4 += 4)
#pragma unroll
        for (int u = 0; u < 4; ++u) { const double x = WS(5, i4 + u); nr4[u] += x * x; }
      for (; i4 < n; ++i4) { const double x = WS(5, i4); nr4[0] += x * x; }
      const double nr = rsqrt_nr((nr4[0] + nr4[1]) + (nr4[2] + nr4[3]));
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

// --------------------------------------------------------------------------
// Back-transformation with the reflectors in blocks of WYB (compact WY form,
// as in LAPACK's dlarft/dlarfb): H_k0 H_k0+1 ... H_k0+b-1 = I - Y T Y^T, Y the
// block's reflectors (v_k(k+1) = 1, zero above), T upper triangular.  A block
// costs one batched warp reduction of WYB dot products instead of WYB
// dependent ones.
constexpr int WYB = 8;

// T of every block, one warp per block: G = Y^T Y above the diagonal, then
// T(i,j) = -tau_j sum_{l=i}^{j-1} T(i,l) G(l,j), T(j,j) = tau_j.
__global__ void k_wy_t(const double *__restrict__ HV, const double *__restrict__ tau, int n, double *__restrict__ Tm) {
  __shared__ double G[WYB][WYB];
  const int blk = blockIdx.x, lane = threadIdx.x;
  const int nref = n - 2, k0 = blk * WYB, b = min(WYB, nref - k0);
  for (int p = 0; p < WYB * WYB; ++p) {
    const int i = p / WYB, j = p - i * WYB;
    if (i >= j || j >= b) continue;   // uniform
    const double *vi = HV + (long)(k0 + i) * n, *vj = HV + (long)(k0 + j) * n;
    double sum = 0.0;
    for (int r = k0 + j + 1 + lane; r < n; r += 32) sum += vi[r] * vj[r];
    sum = warp_sum(sum);
    if (lane == 0) G[i][j] = sum;
  }
  __syncwarp();
  if (lane == 0) {
    double T[WYB][WYB];
    for (int i = 0; i < WYB; ++i)
      for (int j = 0; j < WYB; ++j) T[i][j] = 0.0;
    for (int j = 0; j < b; ++j) {
      const double tj = tau[k0 + j];
      T[j][j] = tj;
      for (int i = 0; i < j; ++i) {
        double acc = 0.0;
        for (int l = i; l < j; ++l) acc += T[i][l] * G[l][j];
        T[i][j] = -tj * acc;
      }
    }
    for (int i = 0; i < WYB; ++i)
      for (int j = 0; j < WYB; ++j) Tm[(long)blk * WYB * WYB + i * WYB + j] = T[i][j];
  }
}

// V(:, c) = Q Z(:, c), one warp per column, blocks applied last to first; lane
// holds rows lane + 32 q (q < MC).  Then the sign convention of k_backtrans.
template <int MC>
__global__ void __launch_bounds__(128) k_backtrans_wy(const double *__restrict__ Z, const double *__restrict__ HV,
                                                      const double *__restrict__ Tm, int n, double *__restrict__ V) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * (blockDim.x >> 5) + warp;
  if (c >= n) return;   // whole warp
  double z[MC];
#pragma unroll
  for (int q = 0; q < MC; ++q) {
    const int i = lane + 32 * q;
    z[q] = (i < n) ? Z[(long)c * n + i] : 0.0;
  }
  const int nref = n - 2, nblk = (nref + WYB - 1) / WYB;
  for (int blk = nblk - 1; blk >= 0; --blk) {
    const int k0 = blk * WYB;
    double y[WYB][MC];
    double sv[WYB];
#pragma unroll
    for (int j = 0; j < WYB; ++j) {
      const int k = k0 + j;
      sv[j] = 0.0;
#pragma unroll
      for (int q = 0; q < MC; ++q) {
        const int i = lane + 32 * q;
        y[j][q] = (k < nref && i > k && i < n) ? HV[(long)k * n + i] : 0.0;
        sv[j] += y[j][q] * z[q];
      }
    }
    // the WYB reductions side by side
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int j = 0; j < WYB; ++j) sv[j] += __shfl_xor_sync(0xffffffffu, sv[j], o);
    const double *T = Tm + (long)blk * WYB * WYB;
    double u[WYB];
#pragma unroll
    for (int i = 0; i < WYB; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int j = i; j < WYB; ++j) acc += T[i * WYB + j] * sv[j];
      u[i] = acc;
    }
#pragma unroll
    for (int q = 0; q < MC; ++q) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < WYB; ++j) acc += y[j][q] * u[j];
      z[q] -= acc;
    }
  }
  double mx = -1.0;
  int km = 0;
  double zk = 0.0;
#pragma unroll
  for (int q = 0; q < MC; ++q) {
    const int i = lane + 32 * q;
    if (i < n && fabs(z[q]) > mx) { mx = fabs(z[q]); km = i; zk = z[q]; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double m2 = __shfl_xor_sync(0xffffffffu, mx, o);
    const int k2 = __shfl_xor_sync(0xffffffffu, km, o);
    const double z2 = __shfl_xor_sync(0xffffffffu, zk, o);
    if (m2 > mx || (m2 == mx && k2 < km)) { mx = m2; km = k2; zk = z2; }
  }
  const double sg = zk < 0.0 ? -1.0 : 1.0;
#pragma unroll
  for (int q = 0; q < MC; ++q) {
    const int i = lane + 32 * q;
    if (i < n) V[(long)c * n + i] = sg * z[q];
  }
}

// V(:, c) = Q Z(:, c) for n > 256: one CTA per BTC columns, the columns in
// shared memory (row i's BTC entries side by side), thread t owning rows
// i = t mod 256 for the whole run.  Per compact-WY block of WYB reflectors
// (last to first): S = Y^T Z (WYB x BTC sums: per-thread partials, warp
// shuffles, then across warps), U = T S, Z -= Y U; two barriers per block.
// Then the sign convention of k_backtrans, one warp per column.
constexpr int BTC = 8;
__global__ void __launch_bounds__(256) k_backtrans_tile(const double *__restrict__ Z, const double *__restrict__ HV,
                                                        const double *__restrict__ Tm, int n,
                                                        double *__restrict__ V) {
  extern __shared__ double zt[];   // n * BTC
  __shared__ double red[8][WYB * BTC];
  __shared__ double Us[WYB * BTC];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int c0 = blockIdx.x * BTC, nc = min(BTC, n - c0);
  for (long q = t; q < (long)n * BTC; q += blockDim.x) {
    const int i = (int)(q / BTC), cc = (int)(q - (long)i * BTC);
    zt[q] = cc < nc ? Z[(long)(c0 + cc) * n + i] : 0.0;
  }
  __syncthreads();
  const int nref = n - 2, nblk = (nref + WYB - 1) / WYB;
  for (int blk = nblk - 1; blk >= 0; --blk) {
    const int k0 = blk * WYB;
    double acc[WYB][BTC];
#pragma unroll
    for (int j = 0; j < WYB; ++j)
#pragma unroll
      for (int cc = 0; cc < BTC; ++cc) acc[j][cc] = 0.0;
    for (int i = t; i < n; i += 256) {
      if (i <= k0) continue;
      double z[BTC];
#pragma unroll
      for (int cc = 0; cc < BTC; ++cc) z[cc] = zt[(long)i * BTC + cc];
#pragma unroll
      for (int j = 0; j < WYB; ++j) {
        const int k = k0 + j;
        const double y = (k < nref && i > k) ? HV[(long)k * n + i] : 0.0;
#pragma unroll
        for (int cc = 0; cc < BTC; ++cc) acc[j][cc] += y * z[cc];
      }
    }
#pragma unroll
    for (int j = 0; j < WYB; ++j)
#pragma unroll
      for (int cc = 0; cc < BTC; ++cc) {
        double v = acc[j][cc];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][j * BTC + cc] = v;
      }
    __syncthreads();
    if (t < WYB * BTC) {
      // S(j, cc) summed over the warps, then U = T S (T upper triangular)
      const int i = t / BTC, cc = t - (t / BTC) * BTC;
      const double *T = Tm + (long)blk * WYB * WYB;
      double u = 0.0;
      for (int j = i; j < WYB; ++j) {
        double sj = 0.0;
        for (int w = 0; w < 8; ++w) sj += red[w][j * BTC + cc];
        u += T[i * WYB + j] * sj;
      }
      Us[i * BTC + cc] = u;
    }
    __syncthreads();
    for (int i = t; i < n; i += 256) {
      if (i <= k0) continue;
      double d[BTC];
#pragma unroll
      for (int cc = 0; cc < BTC; ++cc) d[cc] = 0.0;
#pragma unroll
      for (int j = 0; j < WYB; ++j) {
        const int k = k0 + j;
        const double y = (k < nref && i > k) ? HV[(long)k * n + i] : 0.0;
#pragma unroll
        for (int cc = 0; cc < BTC; ++cc) d[cc] += y * Us[j * BTC + cc];
      }
#pragma unroll
      for (int cc = 0; cc < BTC; ++cc) zt[(long)i * BTC + cc] -= d[cc];
    }
  }
  __syncthreads();
  if (warp < nc) {
    const int cc = warp;
    double mx = -1.0, zk = 0.0;
    int km = 0;
    for (int i = lane; i < n; i += 32) {
      const double v = zt[(long)i * BTC + cc];
      if (fabs(v) > mx) { mx = fabs(v); km = i; zk = v; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double m2 = __shfl_xor_sync(0xffffffffu, mx, o);
      const int k2 = __shfl_xor_sync(0xffffffffu, km, o);
      const double z2 = __shfl_xor_sync(0xffffffffu, zk, o);
      if (m2 > mx || (m2 == mx && k2 < km)) { mx = m2; km = k2; zk = z2; }
    }
    const double sg = zk < 0.0 ? -1.0 : 1.0;
    for (int i = lane; i < n; i += 32) V[(long)(c0 + cc) * n + i] = sg * zt[(long)i * BTC + cc];
  }
}

// The cooperative tridiagonalisation when the matrix fits the shared memory
// of the GPU's CTAs (one per SM) and cooperative launch is available; false
// if it was not launched.  Scratch in vp (7n doubles): v (2n), p (n), the
// per-CTA parts (G), tau (2), then the barrier words.  QX_SYTRD_GRID=0
// turns it off (read at every call).
static bool sytrd_grid(double *A, int n, double *d, double *e, double *HV, double *tau, double *vp, int *d_info,
                       cudaStream_t st) {
  const char *env = getenv("QX_SYTRD_GRID");
  if (env && env[0] == '0') return false;
  int dev = 0, nsm = 0, coop = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) return false;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return false;
  const int G = std::min(nsm, n);
  const int nq = (n + G - 1) / G;
  const size_t sm = sizeof(double) * ((size_t)nq * n + 2 * (size_t)n);
  if (sm > 200 * 1024 || 3L * n + G + 2 + 1 > 7L * n) return false;
  static size_t sm_set = 0;   // per process: set at the first call, then only ever raised
  if (sm > sm_set) {
    if (cudaFuncSetAttribute(k_sytrd_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
      return false;
    sm_set = 200 * 1024;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sytrd_grid, TRG_T, sm) != cudaSuccess || per_sm < 1)
    return false;
  double *gs = vp;
  unsigned *bar = reinterpret_cast<unsigned *>(vp + 3L * n + G + 2);
  if (cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), st) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const double *Ac = A;
  void *args[] = {(void *)&Ac, (void *)&n, (void *)&d, (void *)&e, (void *)&HV, (void *)&tau, (void *)&gs,
                  (void *)&bar, (void *)&d_info};
  if (cudaLaunchCooperativeKernel((const void *)k_sytrd_grid, dim3(G), dim3(TRG_T), args, sm, st) != cudaSuccess) {
    cudaGetLastError();   // not launched: the one-CTA kernel runs instead
    return false;
  }
  return true;
}

// QX_SYTRD_REG=0 keeps the shared-memory tridiagonalisation at every size
// (read at every call).
static bool sytrd_registers_enabled() {
  const char *v = getenv("QX_SYTRD_REG");
  return !(v && v[0] == '0');
}

// A (n x n, destroyed), w (n) eigenvalues ascending, V (n x n) eigenvectors.
// work: at least 8*n*n + 1024*n doubles.  info: number of eigenvalue clusters.
// side, evf, evj (optional): a second stream and two events; the T matrices
// of the compact-WY blocks (which need only the reflectors) are then formed
// there while the eigenvalues and the tridiagonal eigenvectors are found.
int syev(double *A, int n, double *w, double *V, double *work, int *d_info, cudaStream_t st, cudaStream_t side,
         cudaEvent_t evf, cudaEvent_t evj) {
  if (n < 1) { set_error("syev: n=%d", n); return 1; }
  const int NT = ((n + 127) / 128) * 128;
  double *d = work, *e = d + n, *tau = e + n, *vp = tau + n, *HV = vp + 7 * (long)n, *Z = HV + (long)n * n,
         *ws = Z + (long)n * n;   // 6 * n * NT <= 6n^2 + 762n: total <= 8n^2 + 772n
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_sytrd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRD_SMEM_MAX);
    cudaFuncSetAttribute(k_backtrans, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_backtrans_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_invit<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  const size_t smem = sizeof(double) * ((size_t)(n | 1) * n + 7 * (size_t)n);
  const int use = smem <= TRD_SMEM_MAX;
  cudaMemsetAsync(d_info, 0, sizeof(int), st);
  const bool rg = sytrd_registers_enabled();
  if (rg && n <= 80) {
    k_sytrd_rg<8, 10, 3><<<1, 8 * 32, 0, st>>>(A, n, d, e, HV, tau);
  } else if (rg && n <= 160) {
    k_sytrd_rg<8, 20, 5><<<1, 8 * 32, 0, st>>>(A, n, d, e, HV, tau);
  } else if (use) {
    k_sytrd<true><<<1, TRD_T, smem, st>>>(A, n, d, e, HV, tau, vp);
  } else if (!sytrd_grid(A, n, d, e, HV, tau, vp, d_info, st)) {
    k_sytrd<false><<<1, TRD_T, 0, st>>>(A, n, d, e, HV, tau, vp);
  }
  note_launch();
  // T of the WY blocks: on the side stream when one is given
  double *Tm = ws + 6 * (long)n * NT;   // (n/WYB + 1) WYB^2 doubles, inside the work size
  static const bool tile_bt = !getenv("QX_BACKTRANS_TILE") || atoi(getenv("QX_BACKTRANS_TILE")) != 0;
  const bool need_t = n >= 2 && (n <= 256 || tile_bt);
  const bool fork = need_t && side && evf && evj;
  if (need_t) {
    const int nblk = (n - 2 + WYB - 1) / WYB;
    cudaStream_t ts = st;
    if (fork) {
      cudaEventRecord(evf, st);
      cudaStreamWaitEvent(side, evf, 0);
      ts = side;
    }
    if (nblk > 0) { k_wy_t<<<nblk, 32, 0, ts>>>(HV, tau, n, Tm); note_launch(); }
    if (fork) cudaEventRecord(evj, side);
  }
  if (n == 1) {
    cudaMemcpyAsync(w, d, sizeof(double), cudaMemcpyDeviceToDevice, st);
    static const double one = 1.0;
    cudaMemcpyAsync(V, &one, sizeof(double), cudaMemcpyHostToDevice, st);
    return 0;
  }
  // one warp per eigenvalue, one warp per block: spread over the SMs
  const size_t bsm = sizeof(double) * 2 * (size_t)n;
  static size_t bsm_set = 0;   // per process: set at the first call, then only ever raised (contexts of several sizes coexist)
  if (bsm > bsm_set) {
    cudaFuncSetAttribute(k_bisect, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm);
    bsm_set = bsm;
  }
  k_bisect<<<n, 32, bsm, st>>>(d, e, n, w); note_launch();
  const size_t wsm = sizeof(double) * 6 * (size_t)n * 16, dem = sizeof(double) * 2 * (size_t)n;
  if (wsm + dem <= 200 * 1024) {
    k_invit<16><<<(n + 15) / 16, 16, wsm + dem, st>>>(d, e, w, n, Z, ws, NT, d_info); note_launch();
  } else {
    k_invit<0><<<NT / 128, 128, dem, st>>>(d, e, w, n, Z, ws, NT, d_info); note_launch();
  }
  if (n <= 256) {
    if (fork) cudaStreamWaitEvent(st, evj, 0);
    k_backtrans_wy<8><<<(n + 3) / 4, 128, 0, st>>>(Z, HV, Tm, n, V); note_launch();
  } else {
    const size_t bt = sizeof(double) * 8 * (size_t)n;
    if (bt > 200 * 1024) { set_error("syev: n=%d too large for the back-transformation", n); return 1; }
    if (tile_bt) {
      if (fork) cudaStreamWaitEvent(st, evj, 0);
      k_backtrans_tile<<<(n + BTC - 1) / BTC, 256, sizeof(double) * BTC * (size_t)n, st>>>(Z, HV, Tm, n, V);
    } else {
      k_backtrans<<<(n + 7) / 8, 256, bt, st>>>(Z, HV, tau, n, V);
    }
    note_launch();
  }
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
