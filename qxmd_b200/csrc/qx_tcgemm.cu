// Tensor-core GEMM for the FP32 band and projector contractions of the mixed
// precision path: <beta|psi> and its back-application (hckbpp_ib_g,
// nlkbpp.f90:1678-1713), S = C^T C (schmidt.f90:190-237), H_sub = C^T HC
// (engrad.f90:869-895), subgs3 (engrad.f90:1122-1142), C*U
// (eigen.f90:1482-1510) and C*L^-T (schmidt.f90:284-313).
//
// sm_100a only: operands staged by TMA (128-byte swizzles) into a 3-stage
// shared-memory ring, products on the 5th-generation tensor cores
// (tcgen05.mma kind::tf32, 128 x 80 or 128 x 96 tiles, accumulators in TMEM),
// read back with tcgen05.ld.  FP32 accuracy comes from the 3xTF32 split: each operand x
// is cut into x_hi = x rounded to the nearest TF32 value and x_lo = x - x_hi
// rounded the same way, and the tile product is
// A_hi B_hi + A_hi B_lo + A_lo B_hi accumulated in FP32 (relative error about
// 2^-22 per product, unbiased because both parts are rounded to nearest).
// The split is done in shared memory by the epilogue warps between the TMA
// landing and the MMA issue, so HBM traffic is that of a plain FP32 GEMM.
//
// Warp roles (384 threads): warp 0 issues TMA, warp 1 allocates TMEM and
// issues the MMAs (one elected lane), warps 6-11 split the operands, warps
// 2-5 drain the accumulators and run the epilogue (TMEM lane quadrant =
// warp % 4).  Every mbarrier wait is
// bounded by a 2 s clock; on timeout the kernel records an error code, stops
// issuing, drains its own copies and MMAs and frees TMEM.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <array>
#include <map>
#include <mutex>

#include "qx_internal.h"

namespace qx {
namespace tc {

constexpr int BM = 128, BK = 32;
constexpr int A_BYTES = BM * BK * 4;                 // 16 KB
constexpr int NTHREADS = 384;   // TMA, MMA, 4 drain/epilogue warps, 6 split warps
constexpr int NSPLIT_T = NTHREADS - 192;
constexpr int BAR_BYTES = 256;
constexpr unsigned long long WAIT_NS = 2000000000ull;

// Tile width BN (MMA N) and what follows from it: 80 for K-major B, 96 (three
// 32-column chunks) for MN-major B.  TMEM holds two BN-column accumulators
// (at columns 0 and 128), used for alternate k-blocks.
template <int BN_> struct Cfg {
  static constexpr int BN = BN_;
  static constexpr int B_BYTES = BN * BK * 4;
  static constexpr int OFF_AH = 0, OFF_AL = A_BYTES, OFF_BH = 2 * A_BYTES, OFF_BL = 2 * A_BYTES + B_BYTES;
  static constexpr int STAGE_BYTES = 2 * (A_BYTES + B_BYTES);   // a multiple of 1 KB
  static constexpr int STAGES = (4 * STAGE_BYTES <= 212 * 1024) ? 4 : 3;
  static constexpr int TMEM_COLS = 512;
  static constexpr int ACC_STRIDE = 128;   // TMEM column offset of accumulator 1
  static constexpr int TA_BASE = 256;      // A hi/lo of stage s at TA_BASE + 64 s (+ 32 for lo)
  static constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE_BYTES + BAR_BYTES + 1024;   // + alignment slack
  static_assert(BN % 16 == 0 && BN <= ACC_STRIDE, "UMMA N for M = 128, two accumulators in TMEM");
  static_assert(TA_BASE + 64 * STAGES <= TMEM_COLS, "A stages in TMEM");
  static_assert(SMEM_BYTES <= 227 * 1024, "shared memory");
};

__device__ int g_tc_error = 0;

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Non-blocking probe of the phase (acquire semantics).
__device__ __forceinline__ bool mbar_test(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase of parity `parity` to complete, for at most WAIT_NS.
__device__ __noinline__ bool mbar_wait_slow(uint64_t *b, uint32_t parity, int code) {
  if (mbar_try(b, parity)) return true;
  const unsigned long long t0 = now_ns();
  while (true) {
    if (mbar_try(b, parity)) return true;
    if (now_ns() - t0 > WAIT_NS) {
      atomicCAS(&g_tc_error, 0, code);
      return false;
    }
  }
}
// A completed phase is seen by the non-blocking probe at once; a blocking
// try_wait costs a few hundred cycles even then, which on the MMA issuer's
// path of every k-block adds up.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, int code) {
  if (mbar_test(b, parity)) return true;
  return mbar_wait_slow(b, parity, code);
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          su32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(su32(bar))
      : "memory");
}

// Shared-memory matrix descriptor, version 1.  layout 2: 128-byte swizzle of
// 16-byte chunks (K-major tiles); layout 1: 128-byte swizzle of 32-byte
// chunks, the one MN-major layout the tensor cores accept for 32-bit operands.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)layout << 61;
  return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          tmem_d),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}
// A from tensor memory (M rows in lanes, 8 K columns of 32 bits), B from a
// shared-memory descriptor.
__device__ __forceinline__ void mma_tf32_at(uint32_t tmem_d, uint32_t tmem_a, uint64_t bd, uint32_t idesc,
                                            uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(
          tmem_d),
      "r"(tmem_a), "l"(bd), "r"(idesc), "r"(acc));
}
// 32 consecutive 32-bit columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]), "f"(v[9]),
      "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15]), "f"(v[16]), "f"(v[17]), "f"(v[18]),
      "f"(v[19]), "f"(v[20]), "f"(v[21]), "f"(v[22]), "f"(v[23]), "f"(v[24]), "f"(v[25]), "f"(v[26]), "f"(v[27]),
      "f"(v[28]), "f"(v[29]), "f"(v[30]), "f"(v[31])
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}

#define TMEM_LD16(taddr, r)                                                                                          \
  asm volatile(                                                                                                      \
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"      \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),   \
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])                     \
      : "r"(taddr))

struct TcArgs {
  int M, N, K;
  int kb_per_split;      // k-blocks (of BK) per blockIdx.z
  float alpha, beta;
  const float *A;        // for the Gamma-metric epilogue
  long lda;
  const float *B;
  long ldb;
  float *C;
  long ldc;
  int gamma;             // 0 plain, 1 Gamma metric, 2 KB projection metric
  float *W;              // split-K partials W[z][n][m], or null: write C
  const float *rowscale; // C(m, :) scaled by rowscale[m] (beta = 0), or null
};

// Round to the nearest TF32 value (10 stored mantissa bits; ties away from
// zero), by integer arithmetic on the bit pattern.  Values stored this way
// pass through the tensor core's TF32 read unchanged.
__device__ __forceinline__ float tf32_rn(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
// x = hi + lo with hi = tf32_rn(x) (exact TF32, |x - hi| <= 2^-12 |x| with
// either sign) and lo = x - hi in FP32; the tensor core reads lo to TF32,
// losing at most 2^-23 |x|, a bias far below the FP32 rounding of the sums.
__device__ __forceinline__ void split1(float x, float &h, float &l) {
  h = tf32_rn(x);
  l = x - h;
}
template <int N16, int STRIDE>
__device__ __forceinline__ void split_tf32(float4 *hi, float4 *lo, int t) {
#pragma unroll
  for (int i = t; i < N16; i += STRIDE) {
    const float4 x = hi[i];
    float4 h, l;
    split1(x.x, h.x, l.x);
    split1(x.y, h.y, l.y);
    split1(x.z, h.z, l.z);
    split1(x.w, h.w, l.w);
    hi[i] = h;
    lo[i] = l;
  }
}

// A_MN: A stored with M contiguous (A[k*lda + m]); else K contiguous
// (A[m*lda + k]).  B_MN: B stored with N contiguous (B[k*ldb + n]); else K
// contiguous (B[n*ldb + k]).
// ATM: A's hi/lo parts go to tensor memory (warps 6-9, one TMEM lane
// quadrant each) and the MMAs read A there; only B is split in shared memory
// (warps 10-11).  The A tile is then read by the split warps alone: K-major A
// keeps the 128-byte swizzle, MN-major A is loaded without swizzle.
template <bool A_MN, bool B_MN, int BN_, bool ATM>
__global__ void __launch_bounds__(NTHREADS, 1)
    k_tc_gemm(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, TcArgs p) {
  typedef Cfg<BN_> G;
  constexpr int BN = G::BN, STAGES = G::STAGES, STAGE_BYTES = G::STAGE_BYTES;
  constexpr int B_BYTES = G::B_BYTES, OFF_AH = G::OFF_AH, OFF_AL = G::OFF_AL, OFF_BH = G::OFF_BH, OFF_BL = G::OFF_BL;
  extern __shared__ __align__(1024) uint8_t smraw[];
  uint8_t *sm = (uint8_t *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  uint64_t *bars = (uint64_t *)(sm + (size_t)STAGES * STAGE_BYTES);
  uint64_t *full = bars, *conv = bars + STAGES, *empty = bars + 2 * STAGES;
  uint64_t *accf = bars + 3 * STAGES, *acce = accf + 2;   // accumulator full / drained
  uint64_t *fin = acce + 2;                                // all MMAs of this CTA complete
  uint32_t *tmem_slot = (uint32_t *)(fin + 1);
  __shared__ volatile int abort_flag;
  __shared__ float sb0[BN], sb1[BN];   // B(0, n), B(1, n) of the tile (Gamma-metric epilogue)

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int kb0 = blockIdx.z * p.kb_per_split;
  const int nkb_total = (p.K + BK - 1) / BK;
  const int nkb = min(p.kb_per_split, nkb_total - kb0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&conv[s], NSPLIT_T);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 128);
    }
    mbar_init(fin, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                 "r"(G::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int issued = 0;
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % STAGES;
        if (!mbar_wait(&empty[s], ((kb / STAGES) & 1) ^ 1, 1)) { abort_flag = 1; break; }
        if (abort_flag) break;
        uint8_t *st = sm + (size_t)s * STAGE_BYTES;
        mbar_expect_tx(&full[s], A_BYTES + B_BYTES);
        const int k = (kb0 + kb) * BK;
        if (A_MN) {
          for (int c = 0; c < BM / 32; ++c) tma_load_2d(st + OFF_AH + c * 4096, &mapA, m0 + 32 * c, k, &full[s]);
        } else {
          tma_load_2d(st + OFF_AH, &mapA, k, m0, &full[s]);
        }
        if (B_MN) {
          for (int c = 0; c < BN / 32; ++c) tma_load_2d(st + OFF_BH + c * 4096, &mapB, n0 + 32 * c, k, &full[s]);
        } else {
          tma_load_2d(st + OFF_BH, &mapB, k, n0, &full[s]);
        }
        ++issued;
      }
      // drain: every load this thread issued has landed before the CTA exits
      for (int kb = max(0, issued - STAGES); kb < issued; ++kb) mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1, 2);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      // kind::tf32, D F32, M = 128, N = BN
      const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((A_MN && !ATM ? 1u : 0u) << 15) |
                             ((B_MN ? 1u : 0u) << 16) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % STAGES, ab = kb & 1;
        if (!mbar_wait(&conv[s], (kb / STAGES) & 1, 3)) { abort_flag = 1; break; }
        if (!mbar_wait(&acce[ab], ((kb >> 1) & 1) ^ 1, 6)) { abort_flag = 1; break; }
        if (abort_flag) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t st = su32(sm + (size_t)s * STAGE_BYTES);
        const uint32_t dt = tmem + (uint32_t)(ab * G::ACC_STRIDE);
#pragma unroll
        for (int kk = 0; kk < BK / 8; ++kk) {
          // K-major (layout 2): rows of 128 B, 8-row groups 1 KB apart, the
          // k-step is 8 tf32 = 32 B along the swizzled row.  MN-major (layout
          // 1): 32-element MN chunks 4 KB apart (LBO), 4-row K groups 512 B
          // apart (SBO), the k-step is 8 K rows = 1 KB.
          const uint32_t ao = A_MN ? kk * 1024 : kk * 32, bo = B_MN ? kk * 1024 : kk * 32;
          const uint32_t alb = A_MN ? 4096 : 16, blb = B_MN ? 4096 : 16;
          const uint32_t asb = A_MN ? 512 : 1024, bsb = B_MN ? 512 : 1024;
          const uint32_t aly = A_MN ? 1 : 2, bly = B_MN ? 1 : 2;
          const uint64_t bh = sdesc(st + OFF_BH + bo, blb, bsb, bly), bl = sdesc(st + OFF_BL + bo, blb, bsb, bly);
          // each k-block starts its accumulator afresh: the tensor core's
          // accumulation is kept to 12 products deep, the running sum is
          // carried in FP32 registers by the draining warps
          if (ATM) {
            const uint32_t tah = tmem + (uint32_t)(G::TA_BASE + 64 * s + 8 * kk), tal = tah + 32;
            mma_tf32_at(dt, tah, bh, idesc, kk == 0 ? 0u : 1u);
            mma_tf32_at(dt, tah, bl, idesc, 1u);
            mma_tf32_at(dt, tal, bh, idesc, 1u);
          } else {
            const uint64_t ah = sdesc(st + OFF_AH + ao, alb, asb, aly), al = sdesc(st + OFF_AL + ao, alb, asb, aly);
            mma_tf32(dt, ah, bh, idesc, kk == 0 ? 0u : 1u);
            mma_tf32(dt, ah, bl, idesc, 1u);
            mma_tf32(dt, al, bh, idesc, 1u);
          }
        }
        mma_commit(&empty[s]);   // frees the stage when these MMAs are done
        mma_commit(&accf[ab]);   // accumulator ab holds this k-block
      }
      // no MMA of this CTA may still run when TMEM is freed, on any path
      mma_commit(fin);
      mbar_wait(fin, 0, 7);
    }
  } else {
    // ---------------- split (warps 6-11); drain and epilogue (warps 2-5) ----------------
    // The split of a stage runs ahead of the MMAs by up to STAGES k-blocks;
    // the drain of accumulator j overlaps the MMAs of k-block j + 1.
    const bool drains = warp < 6;
    const int quad = warp & 3;
    float acc[BN];
#pragma unroll
    for (int j = 0; j < BN; ++j) acc[j] = 0.f;
    // add the k-block held in accumulator (j & 1) to acc and release it
    auto drain = [&](int j) {
      const int ab = j & 1;
      const bool got = mbar_wait(&accf[ab], (j >> 1) & 1, 5);
      if (!got) abort_flag = 1;
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t base = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(ab * G::ACC_STRIDE);
#pragma unroll
      for (int c = 0; c < BN / 16; ++c) {
        uint32_t r[16];
        TMEM_LD16(base + (uint32_t)(c * 16), r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int q = 0; q < 16; ++q) acc[c * 16 + q] += __uint_as_float(r[q]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      mbar_arrive(&acce[ab]);
    };
    if (!drains && !ATM) {
      const int t = threadIdx.x - 192;   // 0 .. NSPLIT_T - 1 (warps 6-11)
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % STAGES;
        if (!mbar_wait(&full[s], (kb / STAGES) & 1, 4)) abort_flag = 1;
        if (abort_flag) { mbar_arrive(&conv[s]); break; }
        uint8_t *st = sm + (size_t)s * STAGE_BYTES;
        split_tf32<A_BYTES / 16, NSPLIT_T>((float4 *)(st + OFF_AH), (float4 *)(st + OFF_AL), t);
        split_tf32<B_BYTES / 16, NSPLIT_T>((float4 *)(st + OFF_BH), (float4 *)(st + OFF_BL), t);
        // generic-proxy writes -> visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(&conv[s]);
      }
    } else if (!drains && warp < 10) {
      // A: row q * 32 + lane of the tile (q = this warp's TMEM lane quadrant)
      const int m = quad * 32 + lane;
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % STAGES;
        if (!mbar_wait(&full[s], (kb / STAGES) & 1, 4)) abort_flag = 1;
        // warp-uniform exit: the TMEM stores below are .sync.aligned
        if (__any_sync(0xffffffffu, abort_flag != 0)) { mbar_arrive(&conv[s]); break; }
        const float *sa = (const float *)(sm + (size_t)s * STAGE_BYTES + OFF_AH);
        float x[32];
        if (A_MN) {
          // unswizzled 32 (m) x 32 (k) chunks, chunk q holds rows 32 q .. 32 q + 31
#pragma unroll
          for (int k = 0; k < 32; ++k) x[k] = sa[quad * 1024 + k * 32 + lane];
        } else {
          // 128-byte rows, 16-byte chunk j of row m at chunk position j ^ (m & 7)
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const float4 v = *(const float4 *)(sa + m * 32 + ((j ^ (m & 7)) << 2));
            x[4 * j] = v.x;
            x[4 * j + 1] = v.y;
            x[4 * j + 2] = v.z;
            x[4 * j + 3] = v.w;
          }
        }
        float lo[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) split1(x[k], x[k], lo[k]);
        const uint32_t ta = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(G::TA_BASE + 64 * s);
        tmem_st32(ta, x);
        tmem_st32(ta + 32, lo);
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;");
        mbar_arrive(&conv[s]);
      }
    } else if (!drains) {
      const int t = threadIdx.x - 320;   // 0..63 (warps 10-11): B only
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % STAGES;
        if (!mbar_wait(&full[s], (kb / STAGES) & 1, 4)) abort_flag = 1;
        if (abort_flag) { mbar_arrive(&conv[s]); break; }
        uint8_t *st = sm + (size_t)s * STAGE_BYTES;
        split_tf32<B_BYTES / 16, 64>((float4 *)(st + OFF_BH), (float4 *)(st + OFF_BL), t);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(&conv[s]);
      }
    } else {
      for (int kb = 0; kb < nkb; ++kb) {
        if (__any_sync(0xffffffffu, abort_flag != 0)) break;   // warp-uniform: TMEM loads are .sync.aligned
        drain(kb);
      }
    }
    if (drains) {
      // ---------------- epilogue ----------------
      const bool direct = (p.W == nullptr);
      if (direct && p.gamma) {
        for (int j = threadIdx.x - 64; j < BN; j += 128) {   // the 128 threads of warps 2-5
          const int gn = n0 + j;
          sb0[j] = (gn < p.N) ? (B_MN ? p.B[gn] : p.B[(long)gn * p.ldb]) : 0.f;
          sb1[j] = (gn < p.N) ? (B_MN ? p.B[p.ldb + gn] : p.B[(long)gn * p.ldb + 1]) : 0.f;
        }
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");   // the four epilogue warps
      const int gm = m0 + quad * 32 + lane;
      float a0 = 0.f, a1 = 0.f;
      if (direct && p.gamma && gm < p.M) {
        a0 = A_MN ? p.A[gm] : p.A[(long)gm * p.lda];
        a1 = A_MN ? p.A[p.lda + gm] : p.A[(long)gm * p.lda + 1];
      }
      const bool ok = !abort_flag;
      const float alpha = p.alpha, beta = p.beta;
      const float rs = (direct && p.rowscale && gm < p.M) ? p.rowscale[gm] : 1.f;
      if (ok && gm < p.M) {
  #pragma unroll
        for (int c = 0; c < BN / 16; ++c) {
          const int nb = n0 + c * 16;
          if (!direct) {
            float *w = p.W + ((long)blockIdx.z * p.N + nb) * p.M + gm;
  #pragma unroll
            for (int j = 0; j < 16; ++j)
              if (nb + j < p.N) w[(long)j * p.M] = acc[c * 16 + j];
            continue;
          }
          float *cp = p.C + (long)nb * p.ldc + gm;
          float old[16];
          if (beta != 0.f) {
            // issue every load of the chunk before the first store
  #pragma unroll
            for (int j = 0; j < 16; ++j) old[j] = (nb + j < p.N) ? cp[(long)j * p.ldc] : 0.f;
          }
  #pragma unroll
          for (int j = 0; j < 16; ++j) {
            if (nb + j < p.N) {
              float v = acc[c * 16 + j];
              if (p.gamma) {
                v = 2.f * v - a0 * sb0[c * 16 + j];
                if (p.gamma == 2) v -= 2.f * a1 * sb1[c * 16 + j];
              }
              if (p.rowscale) v *= rs;
              cp[(long)j * p.ldc] = (beta == 0.f) ? alpha * v : alpha * v + beta * old[j];
            }
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(G::TMEM_COLS));
  }
}

// ---------------------------------------------------------------------------
// Host side.
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::once_flag g_once;

static bool encode_ready() {
  std::call_once(g_once, [] {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  });
  return g_encode != nullptr;
}

// 2D FP32 tensor: inner extent `inner` (contiguous), `outer` rows `ld` floats
// apart; box 32 x box_rows, out-of-range reads as zero.  Tiles the tensor core
// reads use the 128-byte swizzle of 16-byte chunks (K-major) or of 32-byte
// chunks (MN-major, descriptor layout 1).
// swz: 0 none, 1 the 128-byte swizzle of 16-byte chunks, 2 of 32-byte chunks.
static bool make_map(CUtensorMap *m, const float *base, long inner, long outer, long ld, int box_rows, int swz) {
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
  cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(float)};
  cuuint32_t box[2] = {32u, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1u, 1u};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE,
                        swz == 0 ? CU_TENSOR_MAP_SWIZZLE_NONE
                                 : (swz == 2 ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B : CU_TENSOR_MAP_SWIZZLE_128B),
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

static bool enabled() {
  static int en = -1;
  if (en < 0) {
    const char *e = getenv("QX_TC");
    en = (e && e[0] == '0') ? 0 : 1;
  }
  return en == 1;
}

template <bool A_MN, bool B_MN, int BN, bool ATM>
static int launch_tc(const CUtensorMap &ma, const CUtensorMap &mb, const TcArgs &a, dim3 g, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_tc_gemm<A_MN, B_MN, BN, ATM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Cfg<BN>::SMEM_BYTES) != cudaSuccess)
      return 1;
    attr = true;
  }
  k_tc_gemm<A_MN, B_MN, BN, ATM><<<g, NTHREADS, Cfg<BN>::SMEM_BYTES, st>>>(ma, mb, a);
  note_launch();
  return 0;
}
template <bool A_MN, bool B_MN, int BN>
static int launch_tc(bool atm, const CUtensorMap &ma, const CUtensorMap &mb, const TcArgs &a, dim3 g,
                     cudaStream_t st) {
  return atm ? launch_tc<A_MN, B_MN, BN, true>(ma, mb, a, g, st) : launch_tc<A_MN, B_MN, BN, false>(ma, mb, a, g, st);
}

// QX_TC_ATMEM=0 keeps A in shared memory for the tensor core (read per call).
static bool atmem_enabled() {
  const char *e = getenv("QX_TC_ATMEM");
  return !(e && e[0] == '0');
}

}  // namespace tc

bool tc_enabled() { return tc::enabled(); }

// K-split factors and tile widths chosen by the autotuner, per shape
// (process-wide: contexts of equal sizes share them), and the overrides the
// autotuner times with.
static std::mutex g_split_mu;
static std::map<std::array<long, 6>, std::array<int, 2>> g_split;   // {nsplit, tile width}
thread_local int tc_split_force = 0;
thread_local int tc_tile_force = 0;
int tc_split_lookup(bool ta, bool tb, int M, int N, int K, int gamma) {
  std::lock_guard<std::mutex> lk(g_split_mu);
  auto it = g_split.find({(long)ta, (long)tb, M, N, K, gamma});
  return it == g_split.end() ? 0 : it->second[0];
}
int tc_tile_lookup(bool ta, bool tb, int M, int N, int K, int gamma) {
  std::lock_guard<std::mutex> lk(g_split_mu);
  auto it = g_split.find({(long)ta, (long)tb, M, N, K, gamma});
  return it == g_split.end() ? 0 : it->second[1];
}
void tc_split_store(bool ta, bool tb, int M, int N, int K, int gamma, int nsplit, int tile) {
  std::lock_guard<std::mutex> lk(g_split_mu);
  g_split[{(long)ta, (long)tb, M, N, K, gamma}] = {nsplit, tile};
}
// Tile widths the kernel is built for: K-major B takes any multiple of 16
// (64, 80, 128 here), MN-major B multiples of 32 (64, 96, 128).
bool tc_tile_valid(bool tb, int bn) {
  return tb ? (bn == 64 || bn == 96 || bn == 128) : (bn == 64 || bn == 80 || bn == 128);
}

namespace tc {
// Rows of `inner` floats, `ld` apart, copied to rows `ldp` apart (ldp a
// multiple of 4): an operand whose row stride breaks the 16-byte rule of the
// tensor maps, restaged for the TMA.
// One row per blockIdx.y (rows beyond gridDim.y in steps of it), pairs of
// floats when both strides and both bases allow 8-byte accesses.
__global__ void k_pad_rows(const float *__restrict__ src, long ld, long inner, long rows, float *__restrict__ dst,
                           long ldp) {
  const bool pairs = ((ld | ldp) & 1) == 0 && (((uintptr_t)src | (uintptr_t)dst) & 7) == 0;
  for (long r = blockIdx.y; r < rows; r += gridDim.y) {
    const float *s = src + r * ld;
    float *d = dst + r * ldp;
    if (pairs) {
      const long h = inner >> 1;
      for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < h; i += (long)gridDim.x * blockDim.x)
        reinterpret_cast<float2 *>(d)[i] = reinterpret_cast<const float2 *>(s)[i];
      if ((inner & 1) && blockIdx.x == 0 && threadIdx.x == 0) d[inner - 1] = s[inner - 1];
    } else {
      for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < inner; i += (long)gridDim.x * blockDim.x)
        d[i] = s[i];
    }
  }
}
}  // namespace tc

void pad_rows_f32(const float *src, long ld, long inner, long rows, float *dst, long ldp, cudaStream_t st) {
  if (rows <= 0 || inner <= 0) return;
  tc::k_pad_rows<<<dim3((unsigned)std::min<long>(32, (inner / 2 + 255) / 256 + 1), (unsigned)std::min<long>(rows, 65535)),
                   256, 0, st>>>(src, ld, inner, rows, dst, ldp);
  note_launch();
}

// Tensor-core FP32 GEMM with the semantics of gemm<float> (no column map).
// Returns 0 when launched, -1 when the operands do not meet the TMA rules
// (the caller then uses the CUDA-core kernel), >0 on error.  pad (optional,
// pad_bytes): room to restage an operand whose row stride is not a multiple
// of four floats (or whose base is not 16-byte aligned) before the launch.
int tc_gemm(bool ta, bool tb, int M, int N, int K, float alpha, const float *A, long lda, const float *B, long ldb,
            float beta, float *C, long ldc, int gamma, cudaStream_t st, void *ws, size_t ws_bytes,
            const float *rowscale, void *pad, size_t pad_bytes) {
  using tc::BM;
  using tc::BK;
  if (!tc::enabled() || M <= 0 || N <= 0 || K <= 0) return -1;
  if (!tc::encode_ready()) return -1;
  // A: ta -> K contiguous (A[m*lda + k]); !ta -> M contiguous (A[k*lda + m])
  {
    const bool bad_a = ((uintptr_t)A & 15) || (lda & 3), bad_b = ((uintptr_t)B & 15) || (ldb & 3);
    if (bad_a || bad_b) {
      // restage into pad: rows of the contiguous extent, stride rounded up to 4
      const long a_in = ta ? K : M, a_rows = ta ? M : K, b_in = tb ? N : K, b_rows = tb ? K : N;
      const long a_ld = (a_in + 3) & ~3L, b_ld = (b_in + 3) & ~3L;
      const size_t need = sizeof(float) * ((bad_a ? a_ld * a_rows : 0) + (bad_b ? b_ld * b_rows : 0));
      if (!pad || ((uintptr_t)pad & 15) || need > pad_bytes) return -1;
      float *dst = (float *)pad;
      if (bad_a) {
        pad_rows_f32(A, lda, a_in, a_rows, dst, a_ld, st);
        A = dst;
        lda = a_ld;
        dst += a_ld * a_rows;
      }
      if (bad_b) {
        pad_rows_f32(B, ldb, b_in, b_rows, dst, b_ld, st);
        B = dst;
        ldb = b_ld;
      }
    }
  }
  const bool a_mn = !ta, b_mn = tb;
  const int tm = (M + BM - 1) / BM, nkb = (K + BK - 1) / BK;
  CUtensorMap ma, mb;
  const bool atm = tc::atmem_enabled();
  // tile width: 80 for K-major B, 96 (three 32-column chunks) for MN-major
  // B, unless the autotuner measured another for this shape (A in tensor
  // memory only)
  int bn = b_mn ? 96 : 80;
  {
    // QX_TC_TILE forces a width for every shape where it is valid (tests)
    const char *env = getenv("QX_TC_TILE");
    const int want = tc_tile_force > 0 ? tc_tile_force
                                       : (env && atoi(env) > 0 ? atoi(env) : tc_tile_lookup(ta, tb, M, N, K, gamma));
    if (atm && want > 0 && tc_tile_valid(tb, want)) bn = want;
  }
  const int tn = (N + bn - 1) / bn;
  if (!(a_mn ? tc::make_map(&ma, A, M, K, lda, 32, atm ? 0 : 2) : tc::make_map(&ma, A, K, M, lda, BM, 1))) return -1;
  if (!(b_mn ? tc::make_map(&mb, B, N, K, ldb, 32, 2) : tc::make_map(&mb, B, K, N, ldb, bn, 1))) return -1;
  // split K until the grid covers the SMs, at least 8 k-blocks a split, or
  // as the autotuner measured for this shape
  int nsplit = 1;
  const long tiles = (long)tm * tn;
  const int tuned = ws ? tc_split_lookup(ta, tb, M, N, K, gamma) : 0;
  if (ws && tc_split_force > 0) {
    nsplit = std::min(tc_split_force, nkb);
  } else if (tuned > 0) {
    nsplit = std::min(tuned, nkb);
  } else if (ws && tiles < 100) {
    nsplit = (int)std::min<long>((148 + tiles - 1) / tiles, std::max(1, nkb / 8));
  }
  while (nsplit > 1 && (size_t)nsplit * M * N * sizeof(float) > ws_bytes) --nsplit;
  const int kps = (nkb + nsplit - 1) / nsplit;
  nsplit = (nkb + kps - 1) / kps;
  tc::TcArgs a{M, N, K, kps, alpha, beta, A, lda, B, ldb, C, ldc, gamma, nsplit > 1 ? (float *)ws : nullptr,
               rowscale};
  dim3 g(tm, tn, nsplit);
  int rc;
  if (b_mn) {
    switch (bn) {
      case 64: rc = a_mn ? tc::launch_tc<true, true, 64, true>(ma, mb, a, g, st)
                         : tc::launch_tc<false, true, 64, true>(ma, mb, a, g, st); break;
      case 128: rc = a_mn ? tc::launch_tc<true, true, 128, true>(ma, mb, a, g, st)
                          : tc::launch_tc<false, true, 128, true>(ma, mb, a, g, st); break;
      default: rc = a_mn ? tc::launch_tc<true, true, 96>(atm, ma, mb, a, g, st)
                         : tc::launch_tc<false, true, 96>(atm, ma, mb, a, g, st);
    }
  } else {
    switch (bn) {
      case 64: rc = a_mn ? tc::launch_tc<true, false, 64, true>(ma, mb, a, g, st)
                         : tc::launch_tc<false, false, 64, true>(ma, mb, a, g, st); break;
      case 128: rc = a_mn ? tc::launch_tc<true, false, 128, true>(ma, mb, a, g, st)
                          : tc::launch_tc<false, false, 128, true>(ma, mb, a, g, st); break;
      default: rc = a_mn ? tc::launch_tc<true, false, 80>(atm, ma, mb, a, g, st)
                         : tc::launch_tc<false, false, 80>(atm, ma, mb, a, g, st);
    }
  }
  if (rc) return rc;
  if (nsplit > 1)
    gemm_reduce_f32(ta, tb, M, N, nsplit, alpha, A, lda, B, ldb, beta, C, ldc, gamma, (const float *)ws, st,
                    rowscale);
  return 0;
}

// Error code recorded by a tensor-core GEMM whose wait timed out (0: none);
// reading clears it.
int tc_error_take() {
  int h = 0, z = 0;
  if (cudaMemcpyFromSymbol(&h, tc::g_tc_error, sizeof(int)) != cudaSuccess) return -1;
  if (h) cudaMemcpyToSymbol(tc::g_tc_error, &z, sizeof(int));
  return h;
}

}  // namespace qx
