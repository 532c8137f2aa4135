// GEMMs of the band and projector contractions (CUDA-core kernels for the
// small FP32 shapes and those with a column map, FP64 tensor-core kernel for
// FP64):
// S = C^T C (schmidt.f90:190-237), H_sub = C^T HC (engrad.f90:869-895),
// <beta|psi> and its back-application (nlkbpp.f90:1678-1713), subgs3
// (engrad.f90:1122-1142), C*U (eigen.f90:1482-1510) and C*L^-T
// (schmidt.f90:284-313).  The Gamma-point half-sphere metric
// 2*sum - x(1)*y(1) is applied in the epilogue.
#include <algorithm>
#include <atomic>

#include "qx_internal.h"
#include "qx_cg.h"

namespace qx {

constexpr int BM = 64, BN = 64, BK = 16;

// SPLIT: block z sums k in [z*kchunk, (z+1)*kchunk) and stores its raw
// partial tile to W[z][n][m] (n = logical column); k_gemm_reduce finishes.
template <typename T, bool TA, bool TB, bool SPLIT>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, T alpha, const T *__restrict__ A, long lda,
                                              const T *__restrict__ B, long ldb, T beta, T *__restrict__ Cm, long ldc,
                                              int gamma, const int *__restrict__ colmap, const int *__restrict__ ncol_dev,
                                              int kchunk, T *__restrict__ W) {
  __shared__ T As[BK][BM + 1];
  __shared__ T Bs[BK][BN + 1];
  const int Nact = ncol_dev ? min(N, *ncol_dev) : N;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  if (n0 >= Nact) return;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0;
  const int kb = SPLIT ? blockIdx.z * kchunk : 0;
  const int ke = SPLIT ? min(K, kb + kchunk) : K;
  for (int k0 = kb; k0 < ke; k0 += BK) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int e = tid + 256 * r;
      int m, k;
      if (TA) { k = e & 15; m = e >> 4; } else { m = e & 63; k = e >> 6; }
      const int gm = m0 + m, gk = k0 + k;
      T v = 0;
      if (gm < M && gk < ke) v = TA ? A[(long)gm * lda + gk] : A[(long)gk * lda + gm];
      As[k][m] = v;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int e = tid + 256 * r;
      int n, k;
      if (!TB) { k = e & 15; n = e >> 4; } else { n = e & 63; k = e >> 6; }
      const int gn = n0 + n, gk = k0 + k;
      T v = 0;
      if (gn < Nact && gk < ke) {
        const long cn = colmap ? colmap[gn] : gn;
        v = TB ? B[(long)gk * ldb + cn] : B[cn * ldb + gk];
      }
      Bs[k][n] = v;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      T a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[k][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[k][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + tx + 16 * j;
      if (gn >= Nact) continue;
      if (SPLIT) {
        W[((long)blockIdx.z * N + gn) * M + gm] = acc[i][j];
        continue;
      }
      const long cn = colmap ? colmap[gn] : gn;
      T v = acc[i][j];
      if (gamma) {
        const T a0 = TA ? A[(long)gm * lda] : A[gm];
        const T b0 = TB ? B[cn] : B[cn * ldb];
        v = (T)2 * v - a0 * b0;
        if (gamma == 2) {
          const T a1 = TA ? A[(long)gm * lda + 1] : A[lda + gm];
          const T b1 = TB ? B[ldb + cn] : B[cn * ldb + 1];
          v -= (T)2 * a1 * b1;
        }
      }
      T *c = Cm + cn * ldc + gm;
      *c = (beta == (T)0) ? alpha * v : alpha * v + beta * *c;
    }
  }
}

// Sum the split-K partials in a fixed order, apply the Gamma-metric
// epilogue and alpha/beta, scatter through colmap.  A block of RD_T threads
// finishes 32 consecutive outputs: warp w sums the partials z = w, w + 8,
// w + 16, ... (all loads of a lane independent, 128-byte rows across the
// warp), then lane l of warp 0 adds the eight warp sums in order w = 0..7.
constexpr int RD_T = 256;
template <typename T, bool TA, bool TB>
__global__ void __launch_bounds__(RD_T) k_gemm_reduce(int M, int N, int nsplit, T alpha, const T *__restrict__ A,
                                                      long lda, const T *__restrict__ B, long ldb, T beta,
                                                      T *__restrict__ Cm, long ldc, int gamma,
                                                      const int *__restrict__ colmap, const int *__restrict__ ncol_dev,
                                                      const T *__restrict__ W, const T *__restrict__ rowscale) {
  __shared__ T ws[RD_T / 32][32];
  const int Nact = ncol_dev ? min(N, *ncol_dev) : N;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long e = blockIdx.x * 32L + lane;
  const bool live = e < (long)M * Nact;
  const long zs = (long)N * M;
  T v = 0;
  if (live) {
    const T *w = W + e;   // element (n, m) of partial z at W[z][n][m], e = n * M + m
    int z = warp;
    for (; z + 3 * (RD_T / 32) < nsplit; z += 4 * (RD_T / 32)) {
      const T t0 = w[(long)z * zs], t1 = w[(long)(z + 8) * zs], t2 = w[(long)(z + 16) * zs],
              t3 = w[(long)(z + 24) * zs];
      v += t0;
      v += t1;
      v += t2;
      v += t3;
    }
    for (; z < nsplit; z += RD_T / 32) v += w[(long)z * zs];
  }
  ws[warp][lane] = v;
  __syncthreads();
  if (warp != 0 || !live) return;
  v = ws[0][lane];
#pragma unroll
  for (int q = 1; q < RD_T / 32; ++q) v += ws[q][lane];
  const int gn = (int)(e / M), gm = (int)(e - (long)gn * M);
  const long cn = colmap ? colmap[gn] : gn;
  if (gamma) {
    const T a0 = TA ? A[(long)gm * lda] : A[gm];
    const T b0 = TB ? B[cn] : B[cn * ldb];
    v = (T)2 * v - a0 * b0;
    if (gamma == 2) {
      const T a1 = TA ? A[(long)gm * lda + 1] : A[lda + gm];
      const T b1 = TB ? B[ldb + cn] : B[cn * ldb + 1];
      v -= (T)2 * a1 * b1;
    }
  }
  if (rowscale) v *= rowscale[gm];
  T *c = Cm + cn * ldc + gm;
  *c = (beta == (T)0) ? alpha * v : alpha * v + beta * *c;
}

template <typename T, bool TA, bool TB>
static void launch(dim3 g, int M, int N, int K, T alpha, const T *A, long lda, const T *B, long ldb, T beta, T *C,
                   long ldc, int gamma, const int *colmap, const int *ncol_dev, int nsplit, int kchunk, T *W,
                   cudaStream_t st) {
  if (nsplit <= 1) {
    k_gemm<T, TA, TB, false><<<g, 256, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma, colmap,
                                               ncol_dev, 0, nullptr);
    note_launch();
    return;
  }
  g.z = nsplit;
  k_gemm<T, TA, TB, true><<<g, 256, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma, colmap, ncol_dev,
                                            kchunk, W);
  note_launch();
  const long mn = (long)M * N;
  k_gemm_reduce<T, TA, TB><<<(int)((mn + 31) / 32), RD_T, 0, st>>>(M, N, nsplit, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                    gamma, colmap, ncol_dev, W, nullptr);
  note_launch();
}

// Finish FP32 split-K partials W[z][n][m] (any producer with that layout).
void gemm_reduce_f32(bool ta, bool tb, int M, int N, int nsplit, float alpha, const float *A, long lda, const float *B,
                     long ldb, float beta, float *C, long ldc, int gamma, const float *W, cudaStream_t st,
                     const float *rowscale) {
  const long mn = (long)M * N;
  const int g = (int)((mn + 31) / 32);
  if (ta && tb) k_gemm_reduce<float, true, true><<<g, RD_T, 0, st>>>(M, N, nsplit, alpha, A, lda, B, ldb, beta, C, ldc, gamma, nullptr, nullptr, W, rowscale);
  else if (ta) k_gemm_reduce<float, true, false><<<g, RD_T, 0, st>>>(M, N, nsplit, alpha, A, lda, B, ldb, beta, C, ldc, gamma, nullptr, nullptr, W, rowscale);
  else if (tb) k_gemm_reduce<float, false, true><<<g, RD_T, 0, st>>>(M, N, nsplit, alpha, A, lda, B, ldb, beta, C, ldc, gamma, nullptr, nullptr, W, rowscale);
  else k_gemm_reduce<float, false, false><<<g, RD_T, 0, st>>>(M, N, nsplit, alpha, A, lda, B, ldb, beta, C, ldc, gamma, nullptr, nullptr, W, rowscale);
  note_launch();
}

// Dispatch (gemm<T> below): FP32 without a column map and above the size
// threshold goes to the tensor-core kernel (qx_tcgemm.cu) when the operands
// meet its TMA rules; all FP64 work goes to the DMMA kernel k_dgemm; the
// rest of FP32 (small shapes, a column map, operands outside the TMA rules)
// runs on the CUDA-core kernel k_sgemm below (A and B both transposed, not
// used by the library, on k_gemm above).  Split K when the output has too
// few tiles to fill the GPU and the caller provides a workspace of at least
// nsplit*M*N elements.
// ---------------------------------------------------------------------------
// FP64 contractions on the FP64 tensor cores: mma.sync m8n8k4 (DMMA, 256
// FMAs a warp instruction; the FP64 FMA pipe of a B200 measures about 10 %
// below it, and DFMA kernels are bound by instruction issue long before).
// A CTA owns a TM x TM output tile, warps arranged WGM x WGN, each warp a
// (TM / WGM) x (TM / WGN) block of 8 x 8 DMMA fragments.  k-blocks of DKB
// are staged in shared memory by cp.async, DST deep (DST - 1 blocks in
// flight while one is multiplied; one barrier a k-block).  Each operand
// keeps its global layout in shared memory:
//   k-contiguous (A transposed, B not): [row][DKB + 2]; a lane reads the
//     double2 at k-pair q (its index in its quad) of row g (its quad), one
//     16-byte load serving two DMMAs; the odd pitch in 16-byte units puts
//     the 32 lanes' loads in the fewest shared-memory wavefronts;
//   row-contiguous (A not transposed, B transposed): [k][TM + 2]; a lane
//     reads k = 2q + h of row g, two scalar loads.
// DMMA k-index q of both operands holds k = 2q + h in the h-th DMMA of a
// k-pair, so the products pair up and the sum runs over all k.  TM = 128
// (8 warps of 64 x 32) for large outputs, TM = 64 (4 warps of 32 x 32, more
// CTAs an SM) where 128-wide tiles would mostly be padding, e.g. the
// 160 x 160 band matrices.  colmap / ncol_dev as in k_gemm (output column n
// is stored column colmap[n] of B and C; columns from *ncol_dev on are not
// computed).  Split-K partials W[z][n][m] as k_gemm's.
constexpr int DKB = 16, DST = 3;

__device__ __forceinline__ void cp_async8(double *sdst, const double *gsrc, bool live) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(live ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// doubles of one operand's k-block in shared memory
template <int TM, bool KMAJ>
constexpr int dop_size() {
  return KMAJ ? TM * (DKB + 2) : DKB * (TM + 2);
}
template <int TM, bool TA, bool TB>
constexpr size_t dgemm_smem() {
  return sizeof(double) * DST * (size_t)(dop_size<TM, TA>() + dop_size<TM, !TB>());
}

template <int TM, int WGM, int WGN, bool TA, bool TB, bool SPLIT>
__global__ void __launch_bounds__(32 * WGM *WGN) k_dgemm(int M, int N, int K, double alpha,
                                                          const double *__restrict__ A, long lda,
                                                          const double *__restrict__ B, long ldb, double beta,
                                                          double *__restrict__ Cm, long ldc, int gamma,
                                                          const int *__restrict__ colmap,
                                                          const int *__restrict__ ncol_dev, int kchunk,
                                                          double *__restrict__ W) {
  constexpr int NT = 32 * WGM * WGN, MF = TM / WGM / 8, NF = TM / WGN / 8;
  constexpr int KP = DKB + 2, MP = TM + 2, L = TM * DKB / NT;   // L: elements a thread stages per operand
  constexpr int SA = dop_size<TM, TA>(), SST = SA + dop_size<TM, !TB>();
  extern __shared__ __align__(16) double dsm[];
  const int Nact = ncol_dev ? min(N, *ncol_dev) : N;
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TM;
  if (n0 >= Nact) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % WGM, wn = warp / WGM, g = lane >> 2, q = lane & 3;
  const int kb = SPLIT ? blockIdx.z * kchunk : 0;
  const int ke = SPLIT ? min(K, kb + kchunk) : K;
  const int nk = (ke - kb + DKB - 1) / DKB;
  // the rows a thread stages are the same in every k-block: source row
  // offsets once (B through the column map), then only k moves
  long aoff[L], boff[L];
  unsigned alive = 0, blive = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    const int e = tid + NT * i;
    const int ra = TA ? e / DKB : e % TM, rb = TB ? e % TM : e / DKB;
    const int gm = m0 + ra, gn = n0 + rb;
    if (gm < M) alive |= 1u << i;
    if (gn < Nact) blive |= 1u << i;
    aoff[i] = gm < M ? (TA ? (long)gm * lda : (long)gm) : 0;
    const long cn = gn < Nact ? (colmap ? (long)colmap[gn] : (long)gn) : 0;
    boff[i] = TB ? cn : cn * ldb;
  }
  auto stage = [&](int blk) {
    double *S = dsm + (blk % DST) * SST;
    const int k0 = kb + blk * DKB;
#pragma unroll
    for (int i = 0; i < L; ++i) {
      const int e = tid + NT * i;
      {
        const int r = TA ? e / DKB : e % TM, k = TA ? e % DKB : e / TM;
        const bool live = ((alive >> i) & 1) && k0 + k < ke;
        const double *src = live ? (TA ? A + aoff[i] + k0 + k : A + aoff[i] + (long)(k0 + k) * lda) : A;
        cp_async8(TA ? S + r * KP + k : S + k * MP + r, src, live);
      }
      {
        const int r = TB ? e % TM : e / DKB, k = TB ? e / TM : e % DKB;
        const bool live = ((blive >> i) & 1) && k0 + k < ke;
        const double *src = live ? (TB ? B + boff[i] + (long)(k0 + k) * ldb : B + boff[i] + k0 + k) : B;
        cp_async8(TB ? S + SA + k * MP + r : S + SA + r * KP + k, src, live);
      }
    }
  };
#pragma unroll
  for (int s = 0; s < DST - 1; ++s) {
    if (s < nk) stage(s);
    cp_async_commit();
  }
  double acc[MF][NF][2];
#pragma unroll
  for (int i = 0; i < MF; ++i)
#pragma unroll
    for (int j = 0; j < NF; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  for (int it = 0; it < nk; ++it) {
    cp_async_wait<DST - 2>();   // this thread's copies of block it are in
    __syncthreads();            // everyone's are, and block it - 1 is consumed
    if (it + DST - 1 < nk) stage(it + DST - 1);
    cp_async_commit();
    const double *As = dsm + (it % DST) * SST, *Bs = As + SA;
#pragma unroll
    for (int kp = 0; kp < DKB; kp += 8) {
      double a[MF][2], b[NF][2];
#pragma unroll
      for (int f = 0; f < MF; ++f) {
        const int row = wm * (TM / WGM) + 8 * f + g;
        if (TA) {
          const double2 v = *reinterpret_cast<const double2 *>(As + row * KP + kp + 2 * q);
          a[f][0] = v.x;
          a[f][1] = v.y;
        } else {
          a[f][0] = As[(kp + 2 * q) * MP + row];
          a[f][1] = As[(kp + 2 * q + 1) * MP + row];
        }
      }
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const int col = wn * (TM / WGN) + 8 * f + g;
        if (!TB) {
          const double2 v = *reinterpret_cast<const double2 *>(Bs + col * KP + kp + 2 * q);
          b[f][0] = v.x;
          b[f][1] = v.y;
        } else {
          b[f][0] = Bs[(kp + 2 * q) * MP + col];
          b[f][1] = Bs[(kp + 2 * q + 1) * MP + col];
        }
      }
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int i = 0; i < MF; ++i)
#pragma unroll
          for (int j = 0; j < NF; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i][h], b[j][h]);
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int i = 0; i < MF; ++i) {
    const int gm = m0 + wm * (TM / WGM) + 8 * i + g;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < NF; ++j)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int gn = n0 + wn * (TM / WGN) + 8 * j + 2 * q + c;
        if (gn >= Nact) continue;
        if (SPLIT) {
          W[((long)blockIdx.z * N + gn) * M + gm] = acc[i][j][c];
          continue;
        }
        const long cn = colmap ? colmap[gn] : gn;
        double v = acc[i][j][c];
        if (gamma) {
          const double a0 = TA ? A[(long)gm * lda] : A[gm];
          const double b0 = TB ? B[cn] : B[cn * ldb];
          v = 2.0 * v - a0 * b0;
          if (gamma == 2) {
            const double a1 = TA ? A[(long)gm * lda + 1] : A[lda + gm];
            const double b1 = TB ? B[ldb + cn] : B[cn * ldb + 1];
            v -= 2.0 * a1 * b1;
          }
        }
        double *c_ = Cm + cn * ldc + gm;
        *c_ = (beta == 0.0) ? alpha * v : alpha * v + beta * *c_;
      }
  }
}

// QX_DGEMM=0 keeps every FP64 contraction on k_gemm (read at every call).
static bool dgemm_enabled() {
  const char *e = getenv("QX_DGEMM");
  return !(e && e[0] == '0');
}

// Dynamic shared-memory opt-in of one k_dgemm shape and its resident CTAs an
// SM, once per device.
template <int TM, int WGM, int WGN, bool TA, bool TB>
static int dgemm_prepare() {
  static std::atomic<int> per_sm[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    set_error("k_dgemm: no current device");
    return 0;
  }
  const int known = per_sm[dev].load();
  if (known > 0) return known;
  constexpr int smem = (int)dgemm_smem<TM, TA, TB>();
  const cudaError_t e1 =
      cudaFuncSetAttribute(k_dgemm<TM, WGM, WGN, TA, TB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const cudaError_t e2 =
      cudaFuncSetAttribute(k_dgemm<TM, WGM, WGN, TA, TB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  int n = 0;
  const cudaError_t e3 =
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_dgemm<TM, WGM, WGN, TA, TB, true>, 32 * WGM * WGN, smem);
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || n < 1) {
    set_error("k_dgemm: shared-memory opt-in of %d bytes failed: %s", smem,
              cudaGetErrorString(e1 ? e1 : e2 ? e2 : e3));
    return 0;
  }
  per_sm[dev].store(n);
  return n;
}

template <int TM, int WGM, int WGN, bool TA, bool TB>
static int launch_dgemm_tm(int M, int N, int K, double alpha, const double *A, long lda, const double *B, long ldb,
                           double beta, double *C, long ldc, int gamma, const int *colmap, const int *ncol_dev,
                           void *ws, size_t ws_bytes, cudaStream_t st) {
  constexpr int NT = 32 * WGM * WGN;
  const int per_sm = dgemm_prepare<TM, WGM, WGN, TA, TB>();
  if (per_sm < 1) return 2;
  dim3 g((M + TM - 1) / TM, (N + TM - 1) / TM);
  const long tiles = (long)g.x * g.y, slots = 148L * per_sm;
  // The fewest K-splits (each at least 64 deep, all partials in the
  // workspace, at most four waves) whose CTAs fill 90 % of the waves they
  // take, else the best-filling count.
  auto fill = [&](long ctas) { return (double)ctas / (double)(((ctas + slots - 1) / slots) * slots); };
  int nsplit = 1, kchunk = K;
  if (ws && K >= 128 && fill(tiles) < 0.9) {
    long cap = std::min<long>((4 * slots + tiles - 1) / tiles, (K + 63) / 64);
    cap = std::min<long>(cap, (long)(ws_bytes / ((size_t)M * N * sizeof(double))));
    double best = fill(tiles);
    for (int n = 2; n <= cap; ++n) {
      const int kc = ((K + n - 1) / n + DKB - 1) / DKB * DKB, ns = (K + kc - 1) / kc;
      const double f = fill(tiles * ns);
      if (f > best + 1e-9) {
        best = f;
        nsplit = ns;
        kchunk = kc;
      }
      if (f >= 0.9) break;
    }
  }
  constexpr size_t smem = dgemm_smem<TM, TA, TB>();
  if (nsplit <= 1) {
    k_dgemm<TM, WGM, WGN, TA, TB, false><<<g, NT, smem, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma,
                                                              colmap, ncol_dev, K, nullptr);
    note_launch();
    return 0;
  }
  g.z = nsplit;
  k_dgemm<TM, WGM, WGN, TA, TB, true><<<g, NT, smem, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma,
                                                           colmap, ncol_dev, kchunk, (double *)ws);
  note_launch();
  const long mn = (long)M * N;
  k_gemm_reduce<double, TA, TB><<<(int)((mn + 31) / 32), RD_T, 0, st>>>(M, N, nsplit, alpha, A, lda, B, ldb, beta, C,
                                                                       ldc, gamma, colmap, ncol_dev,
                                                                       (const double *)ws, nullptr);
  note_launch();
  return 0;
}

// 128-wide tiles unless they would cover more than 15 % more padded area
// than 64-wide ones.
static int dgemm_tile(int M, int N) {
  const long a128 = (long)((M + 127) / 128) * ((N + 127) / 128) * 128 * 128;
  const long a64 = (long)((M + 63) / 64) * ((N + 63) / 64) * 64 * 64;
  return a128 * 100 <= a64 * 115 ? 128 : 64;
}

template <bool TA, bool TB>
static int launch_dgemm(int M, int N, int K, double alpha, const double *A, long lda, const double *B, long ldb,
                        double beta, double *C, long ldc, int gamma, const int *colmap, const int *ncol_dev, void *ws,
                        size_t ws_bytes, cudaStream_t st) {
  if (dgemm_tile(M, N) == 128)
    return launch_dgemm_tm<128, 2, 4, TA, TB>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma, colmap, ncol_dev,
                                              ws, ws_bytes, st);
  return launch_dgemm_tm<64, 2, 2, TA, TB>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma, colmap, ncol_dev, ws,
                                           ws_bytes, st);
}

// FP32 contractions below this many flops (2 M N K) run on the CUDA-core
// kernel: the tensor-core kernel's fixed cost per CTA (TMEM allocation,
// barriers, pipeline fill, a TMEM drain per k-block) outweighs their work.
// Measured on the 48-cell batch (all its contractions below 0.2 GFLOP) and
// on Si64 (every contraction 0.48 GFLOP or more).  QX_TC_MIN_FLOPS overrides
// it (read at every call).
constexpr double TC_MIN_FLOPS_DEFAULT = 2.0e8;
static double tc_min_flops() {
  const char *e = getenv("QX_TC_MIN_FLOPS");
  return e ? atof(e) : TC_MIN_FLOPS_DEFAULT;
}

// ---------------------------------------------------------------------------
// FP32 contractions on the CUDA cores (the shapes below the tensor-core size
// threshold, and those with a column map): 256 threads as 16 x 16, each an
// MT x NT block of the (16 MT) x (16 NT) output tile, so that a band count
// of 20-80 is not padded to a multiple of 64 (MT, NT in 2..5 picked per
// shape).  k-blocks of SBK are staged in shared memory by 4-byte cp.async
// (zero-filled outside the operands), SST deep, one barrier a k-block; the
// row offsets of what a thread stages are computed once (B through the
// column map).  Shared layout [k][row] for both operands (pitch rows + 1):
// in a warp the A reads are two broadcasts and the B reads 16 consecutive
// words.  Split-K partials and the epilogue as k_gemm's.
constexpr int SBK = 16, SST = 3;

__device__ __forceinline__ void cp_async4(float *sdst, const float *gsrc, bool live) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gsrc), "r"(live ? 4 : 0) : "memory");
}

template <int MT, int NT>
constexpr size_t sgemm_smem() {
  return sizeof(float) * SST * (size_t)SBK * (16 * MT + 1 + 16 * NT + 1);
}

template <bool TA, bool TB, bool SPLIT, int MT, int NT>
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, float alpha, const float *__restrict__ A, long lda,
                                               const float *__restrict__ B, long ldb, float beta,
                                               float *__restrict__ Cm, long ldc, int gamma,
                                               const int *__restrict__ colmap, const int *__restrict__ ncol_dev,
                                               int kchunk, float *__restrict__ W, int *__restrict__ cnt) {
  constexpr int TMM = 16 * MT, TNN = 16 * NT, PA = TMM + 1, PB = TNN + 1;
  constexpr int SA = SBK * PA, SSZ = SA + SBK * PB;
  extern __shared__ __align__(16) float ssm[];
  const int Nact = ncol_dev ? min(N, *ncol_dev) : N;
  const int m0 = blockIdx.x * TMM, n0 = blockIdx.y * TNN;
  if (n0 >= Nact) return;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int kb = SPLIT ? blockIdx.z * kchunk : 0;
  const int ke = SPLIT ? min(K, kb + kchunk) : K;
  const int nk = (ke - kb + SBK - 1) / SBK;
  // element e = tid + 256 i of a k-block: k-contiguous operands (A
  // transposed, B not) take k = e % 16, row e / 16; the others row e % rows,
  // k = e / rows
  long aoff[MT], boff[NT];
  unsigned alive = 0, blive = 0;
#pragma unroll
  for (int i = 0; i < MT; ++i) {
    const int e = tid + 256 * i, r = TA ? e / SBK : e % TMM, gm = m0 + r;
    if (gm < M) alive |= 1u << i;
    aoff[i] = gm < M ? (TA ? (long)gm * lda : (long)gm) : 0;
  }
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    const int e = tid + 256 * i, r = TB ? e % TNN : e / SBK, gn = n0 + r;
    if (gn < Nact) blive |= 1u << i;
    const long cn = gn < Nact ? (colmap ? (long)colmap[gn] : (long)gn) : 0;
    boff[i] = TB ? cn : cn * ldb;
  }
  auto stage = [&](int blk) {
    float *S = ssm + (blk % SST) * SSZ;
    const int k0 = kb + blk * SBK;
#pragma unroll
    for (int i = 0; i < MT; ++i) {
      const int e = tid + 256 * i;
      const int r = TA ? e / SBK : e % TMM, k = TA ? e % SBK : e / TMM;
      const bool live = ((alive >> i) & 1) && k0 + k < ke;
      const float *src = live ? (TA ? A + aoff[i] + k0 + k : A + aoff[i] + (long)(k0 + k) * lda) : A;
      cp_async4(S + k * PA + r, src, live);
    }
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      const int e = tid + 256 * i;
      const int r = TB ? e % TNN : e / SBK, k = TB ? e / TNN : e % SBK;
      const bool live = ((blive >> i) & 1) && k0 + k < ke;
      const float *src = live ? (TB ? B + boff[i] + (long)(k0 + k) * ldb : B + boff[i] + k0 + k) : B;
      cp_async4(S + SA + k * PB + r, src, live);
    }
  };
#pragma unroll
  for (int s = 0; s < SST - 1; ++s) {
    if (s < nk) stage(s);
    cp_async_commit();
  }
  float acc[MT][NT];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[i][j] = 0.f;
  for (int it = 0; it < nk; ++it) {
    cp_async_wait<SST - 2>();   // this thread's copies of block it are in
    __syncthreads();            // everyone's are, and block it - 1 is consumed
    if (it + SST - 1 < nk) stage(it + SST - 1);
    cp_async_commit();
    const float *As = ssm + (it % SST) * SSZ, *Bs = As + SA;
#pragma unroll
    for (int k = 0; k < SBK; ++k) {
      float a[MT], b[NT];
#pragma unroll
      for (int i = 0; i < MT; ++i) a[i] = As[k * PA + ty + 16 * i];
#pragma unroll
      for (int j = 0; j < NT; ++j) b[j] = Bs[k * PB + tx + 16 * j];
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
  }
  cp_async_wait<0>();
  if (SPLIT) {
    // Split K: every CTA stores its partial tile (element e of thread t at
    // W[((z tiles + tile) MT NT + e) 256 + t], coalesced), counts itself in
    // for the tile, and the last to arrive sums the partials in z order and
    // finishes the tile; it then clears the count for the next launch.  No
    // CTA waits for another.
    const int tile = blockIdx.y * gridDim.x + blockIdx.x;
    const long zs = (long)gridDim.x * gridDim.y * MT * NT * 256;
    float *Wt = W + (long)tile * MT * NT * 256 + tid;
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j) Wt[blockIdx.z * zs + (i * NT + j) * 256] = acc[i][j];
    __threadfence();
    __syncthreads();
    __shared__ int last;
    if (tid == 0) last = atomicAdd(cnt + tile, 1) == (int)gridDim.z - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j) acc[i][j] = 0.f;
    for (int z = 0; z < (int)gridDim.z; ++z)
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) acc[i][j] += __ldcg(Wt + z * zs + (i * NT + j) * 256);
    if (tid == 0) cnt[tile] = 0;
  }
#pragma unroll
  for (int i = 0; i < MT; ++i) {
    const int gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const int gn = n0 + tx + 16 * j;
      if (gn >= Nact) continue;
      const long cn = colmap ? colmap[gn] : gn;
      float v = acc[i][j];
      if (gamma) {
        const float a0 = TA ? A[(long)gm * lda] : A[gm];
        const float b0 = TB ? B[cn] : B[cn * ldb];
        v = 2.f * v - a0 * b0;
        if (gamma == 2) {
          const float a1 = TA ? A[(long)gm * lda + 1] : A[lda + gm];
          const float b1 = TB ? B[ldb + cn] : B[cn * ldb + 1];
          v -= 2.f * a1 * b1;
        }
      }
      float *c = Cm + cn * ldc + gm;
      *c = (beta == 0.f) ? alpha * v : alpha * v + beta * *c;
    }
  }
}

// QX_SGEMM=0 keeps the FP32 CUDA-core contractions on k_gemm (read at every
// call).
static bool sgemm_enabled() {
  const char *e = getenv("QX_SGEMM");
  return !(e && e[0] == '0');
}

// Rows of a tile a thread-row covers for an extent of n: the smallest of
// 2..5 (tiles of 32..80) that holds n, else 4 (64-row tiles).
static int sgemm_rows(int n) {
  for (int t = 2; t <= 5; ++t)
    if (16 * t >= n) return t;
  return 4;
}

template <bool TA, bool TB, bool SPLIT, int MT, int NT>
static void sgemm_go(dim3 g, int M, int N, int K, float alpha, const float *A, long lda, const float *B, long ldb,
                     float beta, float *C, long ldc, int gamma, const int *colmap, const int *ncol_dev, int kchunk,
                     float *W, int *cnt, cudaStream_t st) {
  constexpr size_t sm = sgemm_smem<MT, NT>();
  static_assert(sm <= 48 * 1024, "stages fit the default shared-memory limit");
  k_sgemm<TA, TB, SPLIT, MT, NT><<<g, 256, sm, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma, colmap,
                                                     ncol_dev, kchunk, W, cnt);
  note_launch();
}

// One shape's launch: tile rows MT x NT from the extents (k-contiguous A:
// both from the band-sized extents; otherwise 64-row tiles down M), K split
// as k_gemm's, the partials summed by the last CTA of each tile (cnt: one
// zeroed counter per tile).
template <bool TA, bool TB>
static void sgemm_launch(int M, int N, int K, float alpha, const float *A, long lda, const float *B, long ldb,
                         float beta, float *C, long ldc, int gamma, const int *colmap, const int *ncol_dev, void *ws,
                         size_t ws_bytes, int *cnt, cudaStream_t st) {
  const int mt = TA ? sgemm_rows(M) : 4, nt = sgemm_rows(N);
  dim3 g((M + 16 * mt - 1) / (16 * mt), (N + 16 * nt - 1) / (16 * nt));
  const long tiles = (long)g.x * g.y;
  const size_t part = sizeof(float) * (size_t)tiles * 256 * mt * nt;   // one split's partial tiles
  int nsplit = 1, kchunk = K;
  if (ws && cnt && tiles <= GEMM_TILE_COUNTERS && tiles < 2 * 148 && K >= 4 * 256) {
    nsplit = (int)std::min<long>((2 * 148 + tiles - 1) / tiles, (K + 255) / 256);
    kchunk = ((K + nsplit - 1) / nsplit + SBK - 1) / SBK * SBK;
    nsplit = (K + kchunk - 1) / kchunk;
    if ((size_t)nsplit * part > ws_bytes) {
      nsplit = (int)(ws_bytes / part);
      if (nsplit < 2) nsplit = 1;
      else {
        kchunk = ((K + nsplit - 1) / nsplit + SBK - 1) / SBK * SBK;
        nsplit = (K + kchunk - 1) / kchunk;
      }
    }
  }
  if (nsplit <= 1) kchunk = K;
  g.z = nsplit;
  float *W = (float *)ws;
  const bool split = nsplit > 1;
#define QX_SG(MT_, NT_)                                                                                              \
  if (mt == MT_ && nt == NT_) {                                                                                      \
    if (split) sgemm_go<TA, TB, true, MT_, NT_>(g, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma, colmap,     \
                                                ncol_dev, kchunk, W, cnt, st);                                       \
    else sgemm_go<TA, TB, false, MT_, NT_>(g, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma, colmap, ncol_dev, \
                                           kchunk, W, nullptr, st);                                                  \
  }
  if (TA) {
    QX_SG(2, 2) else QX_SG(2, 3) else QX_SG(2, 4) else QX_SG(2, 5)
    else QX_SG(3, 2) else QX_SG(3, 3) else QX_SG(3, 4) else QX_SG(3, 5)
    else QX_SG(4, 2) else QX_SG(4, 3) else QX_SG(4, 4) else QX_SG(4, 5)
    else QX_SG(5, 2) else QX_SG(5, 3) else QX_SG(5, 4) else QX_SG(5, 5)
  } else {
    QX_SG(4, 2) else QX_SG(4, 3) else QX_SG(4, 4) else QX_SG(4, 5)
  }
#undef QX_SG
}

// FP32 contractions that ran on the CUDA-core kernel instead of the tensor
// cores (a column map, a device column count or operands outside the TMA
// rules; not the small ones sent there by tc_min_flops), counted for
// qx_gemm_fallbacks().
static std::atomic<long> g_fp32_fallbacks{0};
long fp32_gemm_fallbacks() { return g_fp32_fallbacks.load(); }
void fp32_gemm_fallbacks_add(long n) { g_fp32_fallbacks.fetch_add(n); }

template <typename T>
int gemm(bool ta, bool tb, int M, int N, int K, T alpha, const T *A, long lda, const T *B, long ldb, T beta, T *C,
         long ldc, int gamma, const int *colmap, const int *ncol_dev, cudaStream_t st, void *ws, size_t ws_bytes,
         const T *rowscale, void *pad, size_t pad_bytes) {
  if (M <= 0 || N <= 0) return 0;
  // the workspace opens with the per-tile counters of k_sgemm's split K
  int *cnt = nullptr;
  if (ws && ws_bytes > GEMM_COUNTER_BYTES) {
    cnt = (int *)ws;
    ws = (char *)ws + GEMM_COUNTER_BYTES;
    ws_bytes -= GEMM_COUNTER_BYTES;
  } else {
    ws = nullptr;
    ws_bytes = 0;
  }
  // small FP32 contractions run on the CUDA-core kernel by choice (not counted)
  const bool small = sizeof(T) == sizeof(float) && 2.0 * (double)M * (double)N * (double)K < tc_min_flops();
  if (sizeof(T) == sizeof(float) && K > 0 && !small && (colmap || ncol_dev || !tc_enabled())) ++g_fp32_fallbacks;
  if (rowscale && beta != (T)0) { set_error("gemm: a row scale needs beta = 0"); return 1; }
  if (sizeof(T) == sizeof(float) && !colmap && !ncol_dev && K > 0 && !small) {
    const int r = tc_gemm(ta, tb, M, N, K, (float)alpha, (const float *)A, lda, (const float *)B, ldb, (float)beta,
                          (float *)C, ldc, gamma, st, ws, ws_bytes, (const float *)rowscale, pad, pad_bytes);
    if (r == 0) return 0;
    if (r > 0) {
      set_error("tensor-core GEMM launch failed: %s", cudaGetErrorString(cudaGetLastError()));
      return 2;
    }
    if (tc_enabled()) ++g_fp32_fallbacks;   // operands outside the TMA rules
  }
  if (sizeof(T) == sizeof(double) && K > 0 && dgemm_enabled()) {
    const double *Ad = (const double *)A, *Bd = (const double *)B;
    double *Cd = (double *)C;
    int r;
    if (ta && tb)
      r = launch_dgemm<true, true>(M, N, K, alpha, Ad, lda, Bd, ldb, beta, Cd, ldc, gamma, colmap, ncol_dev, ws,
                                   ws_bytes, st);
    else if (ta)
      r = launch_dgemm<true, false>(M, N, K, alpha, Ad, lda, Bd, ldb, beta, Cd, ldc, gamma, colmap, ncol_dev, ws,
                                    ws_bytes, st);
    else if (tb)
      r = launch_dgemm<false, true>(M, N, K, alpha, Ad, lda, Bd, ldb, beta, Cd, ldc, gamma, colmap, ncol_dev, ws,
                                    ws_bytes, st);
    else
      r = launch_dgemm<false, false>(M, N, K, alpha, Ad, lda, Bd, ldb, beta, Cd, ldc, gamma, colmap, ncol_dev, ws,
                                     ws_bytes, st);
    if (r) return r;
    if (rowscale) scale_rows<T>(M, N, C, ldc, rowscale, colmap, ncol_dev, st);
    return 0;
  }
  if (sizeof(T) == sizeof(float) && !(ta && tb) && sgemm_enabled()) {
    const float *Af = (const float *)A, *Bf = (const float *)B;
    float *Cf = (float *)C;
    if (ta)
      sgemm_launch<true, false>(M, N, K, (float)alpha, Af, lda, Bf, ldb, (float)beta, Cf, ldc, gamma, colmap, ncol_dev,
                                ws, ws_bytes, cnt, st);
    else if (tb)
      sgemm_launch<false, true>(M, N, K, (float)alpha, Af, lda, Bf, ldb, (float)beta, Cf, ldc, gamma, colmap, ncol_dev,
                                ws, ws_bytes, cnt, st);
    else
      sgemm_launch<false, false>(M, N, K, (float)alpha, Af, lda, Bf, ldb, (float)beta, Cf, ldc, gamma, colmap,
                                 ncol_dev, ws, ws_bytes, cnt, st);
    if (rowscale) scale_rows<T>(M, N, C, ldc, rowscale, colmap, ncol_dev, st);
    return 0;
  }
  dim3 g((M + BM - 1) / BM, (N + BN - 1) / BN);
  const long tiles = (long)g.x * g.y;
  int nsplit = 1, kchunk = K;
  if (ws && tiles < 2 * 148 && K >= 4 * 256) {
    nsplit = (int)std::min<long>((2 * 148 + tiles - 1) / tiles, (K + 255) / 256);
    kchunk = ((K + nsplit - 1) / nsplit + BK - 1) / BK * BK;
    nsplit = (K + kchunk - 1) / kchunk;
    if ((size_t)nsplit * M * N * sizeof(T) > ws_bytes) {
      nsplit = (int)(ws_bytes / ((size_t)M * N * sizeof(T)));
      if (nsplit < 2) nsplit = 1;
      else {
        kchunk = ((K + nsplit - 1) / nsplit + BK - 1) / BK * BK;
        nsplit = (K + kchunk - 1) / kchunk;
      }
    }
  }
  T *W = (T *)ws;
  if (ta && tb) launch<T, true, true>(g, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma, colmap, ncol_dev, nsplit, kchunk, W, st);
  else if (ta) launch<T, true, false>(g, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma, colmap, ncol_dev, nsplit, kchunk, W, st);
  else if (tb) launch<T, false, true>(g, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma, colmap, ncol_dev, nsplit, kchunk, W, st);
  else launch<T, false, false>(g, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, gamma, colmap, ncol_dev, nsplit, kchunk, W, st);
  if (rowscale) scale_rows<T>(M, N, C, ldc, rowscale, colmap, ncol_dev, st);
  return 0;
}

template int gemm<float>(bool, bool, int, int, int, float, const float *, long, const float *, long, float, float *,
                         long, int, const int *, const int *, cudaStream_t, void *, size_t, const float *, void *,
                         size_t);
template int gemm<double>(bool, bool, int, int, int, double, const double *, long, const double *, long, double,
                          double *, long, int, const int *, const int *, cudaStream_t, void *, size_t, const double *,
                          void *, size_t);

}  // namespace qx

// ---------------------------------------------------------------------------
// Allocation-free band matrix: the split-K GEMM above with its partial sums in
// a fixed, file-scope device array instead of a caller- or context-owned
// workspace.  For host programs that must not allocate device memory after
// start-up (a memory pool sized once and locked, or a host code that owns all
// device memory itself and forbids cudaMalloc in its time-step loop).
#include <mutex>

#include "../../include/qxmd_b200.h"

// Split-K partials of qx_hmatrix_static: nsplit * nb * nb doubles.  Every
// device that loads this library holds these 16 MiB until the process exits.
static __device__ __align__(256) double g_hmat_scratch[QX_HMATRIX_STATIC_SCRATCH_BYTES / sizeof(double)];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double *g_scratch_ptr[kMaxDevices] = {};

// Device address of g_hmat_scratch on the current device.  In host code the
// symbol only names a host-side shadow; the address the kernels need comes
// from cudaGetSymbolAddress, taken once per device with that device current.
int scratch_address(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    qx::set_error("qx_hmatrix_static: cudaGetDevice: %s", cudaGetErrorString(e));
    return QX_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    qx::set_error("qx_hmatrix_static: device ordinal %d beyond %d", dev, kMaxDevices);
    return QX_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_hmat_scratch);
    if (e != cudaSuccess || !p) {
      qx::set_error("qx_hmatrix_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return QX_ERR_CUDA;
    }
    g_scratch_ptr[dev] = (double *)p;
  }
  *out = g_scratch_ptr[dev];
  return QX_OK;
}
}  // namespace

extern "C" long qx_gemm_fallbacks(void) { return qx::fp32_gemm_fallbacks(); }

extern "C" int qx_hmatrix_static(const double *c, const double *hc, int nplwex, int nb, double *hsub, void *stream) {
  if (!c || !hc || !hsub || nplwex <= 0 || nb <= 0) {
    qx::set_error("qx_hmatrix_static: bad arguments");
    return QX_ERR_ARG;
  }
  if (nb > QX_HMATRIX_STATIC_MAX_NB) {
    qx::set_error("qx_hmatrix_static: nb = %d exceeds %d, the most whose two K-partials fit the %d-byte scratch",
                  nb, QX_HMATRIX_STATIC_MAX_NB, QX_HMATRIX_STATIC_SCRATCH_BYTES);
    return QX_ERR_ARG;
  }
  double *W = nullptr;
  int rc = scratch_address(&W);
  if (rc) return rc;
  // Split K into partials: enough of them to give about two CTAs per SM, each
  // at least 128 deep, as many as the scratch holds (two or more asked for;
  // when nplwex <= BK the chunk rounds up to the whole of K, a single partial
  // and no scratch).  At nb = 1024 the two partials fill the scratch exactly.
  const int tiles_m = (nb + qx::BM - 1) / qx::BM;
  const long tiles = (long)tiles_m * tiles_m;
  const long cap = (long)(QX_HMATRIX_STATIC_SCRATCH_BYTES / (sizeof(double) * (size_t)nb * nb));
  long want = std::max<long>(2, (2 * 148 + tiles - 1) / tiles);
  want = std::min<long>(want, std::max<long>(2, (nplwex + 127) / 128));
  want = std::min<long>(want, cap);
  int kchunk = (int)(((nplwex + want - 1) / want + qx::BK - 1) / qx::BK * qx::BK);
  const int nsplit = (nplwex + kchunk - 1) / kchunk;   // <= want: every partial fits
  // Every partial W[z][n][m], m, n < nb, z < nsplit, is written by its CTA
  // before k_gemm_reduce reads it, so nothing needs clearing between calls.
  dim3 g(tiles_m, tiles_m);
  qx::launch<double, true, false>(g, nb, nb, nplwex, 1.0, c, nplwex, hc, nplwex, 0.0, hsub, nb, 1, nullptr, nullptr,
                                  nsplit, kchunk, W, (cudaStream_t)stream);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    qx::set_error("qx_hmatrix_static: launch: %s", cudaGetErrorString(e));
    return QX_ERR_CUDA;
  }
  return QX_OK;
}
