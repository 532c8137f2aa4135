// TDDFT-FSSH surface hopping in the density-matrix representation
// (tddft_fssh_dm, tddft_fssh.f90:1989-2402), one spin channel, on the device.
//
// For a window of nst adiabatic states, state s (occupied, with an empty
// neighbour within nupdn = 3) carries a 7 x 7 complex density matrix
// rho(j, k), j, k in [s-3, s+3] clipped to the window.  Over one MD step of
// length dtmd it is integrated with RK4 in nstep = int(dtmd / dttddft)
// substeps of
//   d rho_r/dt = (e_j - e_k) rho_i - rho_r d + d rho_r,
//   d rho_i/dt = -(e_j - e_k) rho_r - rho_i d + d rho_i,
// d(k, j) = -(A(k, j) - A(j, k)) / (2 dtmd) the nonadiabatic couplings from
// the overlap A(k, j) = <psi_k(t)|psi_j(t+dt)>, while the ratio
// Re rho(iud, 0) / Re rho(0, 0) is summed per neighbour.  Then one thread
// walks the states and neighbours in the reference's order, forms the hop
// probabilities 2 d(news, s) dttddft * sum (with the Boltzmann factor on
// one-state-up hops), accumulates them, and compares their running sum with
// one Park-Miller draw (rnd00, funcs.f90:1673-1689) to accept at most one
// transition.
//
// All arithmetic is FP64 with explicitly rounded operations (no fused
// multiply-add) in the reference's evaluation order, so the amplitudes and
// the hop sequence are those of a CPU evaluation of the same expressions.
//
// Layout (all double, one buffer set per context): dnr/dni [nst][7][7] with
// rho(j, k) at [s][j + 3][k + 3]; probinteg and bkl [nst][7]; accum(news, s)
// at [news + s * nst]; occ_rec and occ_store [nst]; rndx [1].
#include "qx_internal.h"

namespace qx {

namespace {
constexpr int FN = 3, FW = 7;

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// d(k, j) = -(A(k, j) - A(j, k)) / 2 / dtmd (tddft_fssh.f90:2098)
__device__ __forceinline__ double dkj(const double *A, int nst, int k, int j, double dtmd) {
  return dvd(dvd(-sub(A[k + (long)j * nst], A[j + (long)k * nst]), 2.0), dtmd);
}

// The state takes part when it is occupied and a neighbour within 3 is not
// full (tddft_fssh.f90:2110-2121).
__device__ __forceinline__ bool fs_active(const double *occ, int nst, int s) {
  if (!(occ[s] > 0.5)) return false;
  bool any = false;
  for (int iud = -FN; iud <= FN; ++iud) {
    const int ns = s + iud;
    if (ns < 0 || ns >= nst || ns == s) continue;
    if (occ[ns] > 1.5) continue;
    any = true;
  }
  return any;
}

// One CTA of 128 threads per state s: thread t < 98 owns the real (t even) or
// imaginary (t odd) part of rho(a - 3, b - 3), (a, b) = (e / 7, e % 7),
// e = t / 2.  Each thread carries one chain of the reference's sum, in the
// reference's order.  The couplings of the element's row a and column b and
// its energy difference stay in registers for the whole MD step; the RK
// stage matrices go through two shared buffers in turn, so one barrier per
// stage suffices.  Outside the window the matrices are zero and the
// couplings too: the extra terms add exact zeros, so the sums equal those
// over the window alone.
constexpr int FT_PROP = 128;
__global__ void __launch_bounds__(FT_PROP) k_fssh_prop(int nst, const double *A, const double *eig, double dtmd,
                                                      double dttddft, double *dnr, double *dni,
                                                      const double *occ_store, double *probinteg) {
  const int s = blockIdx.x;
  const int t = threadIdx.x;
  __shared__ double D[FW][FW], E[FW];
  __shared__ double S[2][2][FW][FW];   // [buffer][re, im][a][b]
  if (t < FW) probinteg[(long)s * FW + t] = 0.0;
  if (!fs_active(occ_store, nst, s)) return;
  const int n1 = max(-FN, -s), n2 = min(FN, nst - 1 - s);
  if (t < FW * FW) {
    const int a = t / FW, b = t % FW;
    const bool ok = a - FN >= n1 && a - FN <= n2 && b - FN >= n1 && b - FN <= n2;
    D[a][b] = ok ? dkj(A, nst, s + a - FN, s + b - FN, dtmd) : 0.0;
  }
  for (int i = t; i < 2 * 2 * FW * FW; i += FT_PROP) (&S[0][0][0][0])[i] = 0.0;
  if (t < FW) E[t] = (t - FN >= n1 && t - FN <= n2) ? eig[s + t - FN] : 0.0;
  __syncthreads();
  const int e = min(t >> 1, FW * FW - 1), part = t & 1;
  const int a = e / FW, b = e % FW;
  const bool own = t < 2 * FW * FW && a - FN >= n1 && a - FN <= n2 && b - FN >= n1 && b - FN <= n2;
  double *g = (part ? dni : dnr) + (long)s * FW * FW + e;
  double dv = own ? *g : 0.0;
  const double de = part ? -sub(E[a], E[b]) : sub(E[a], E[b]);
  double drow[FW], dcol[FW];
#pragma unroll
  for (int l = 0; l < FW; ++l) {
    drow[l] = D[a][l];   // d(j, l)
    dcol[l] = D[l][b];   // d(l, k)
  }
  const double rkc[4] = {0.0, dvd(dttddft, 2.0), dvd(dttddft, 2.0), dttddft};
  const int nstep = (int)(dtmd / dttddft);
  // probability integral of the neighbour owned here (real part of element (iud + 3, 3))
  const bool pown = own && part == 0 && b == FN && a != FN;
  double pint = 0.0;
  if (own) S[0][part][a][b] = dv;
  __syncthreads();
  for (int step = 0; step < nstep; ++step) {
    double k[4];
#pragma unroll
    for (int irk = 0; irk < 4; ++irk) {
      const int cur = irk & 1;
      // real part: (e_j - e_k) Im rho + sum_l (-Re rho(j, l) d(l, k) + Re rho(l, k) d(j, l));
      // imaginary part: -(e_j - e_k) Re rho + the same sum over Im rho
      const double(*X)[FW] = S[cur][part];
      double r = mul(de, S[cur][1 - part][a][b]);
#pragma unroll
      for (int l = 0; l < FW; ++l) r = add(sub(r, mul(X[a][l], dcol[l])), mul(X[l][b], drow[l]));
      k[irk] = r;
      if (own) {
        if (irk < 3) {
          S[1 - cur][part][a][b] = add(dv, mul(rkc[irk + 1], r));
        } else {
          // RK4 update: rho + (k1 + 2 k2 + 2 k3 + k4) dttddft / 6 (tddft_fssh.f90:2168-2177)
          const double sm = add(add(add(k[0], mul(2.0, k[1])), mul(2.0, k[2])), k[3]);
          dv = add(dv, dvd(mul(sm, dttddft), 6.0));
          S[0][part][a][b] = dv;
        }
      }
      __syncthreads();
    }
    if (pown) pint = add(pint, dvd(S[0][0][a][FN], S[0][0][FN][FN]));
  }
  if (own) *g = dv;
  if (pown) probinteg[(long)s * FW + a] = pint;
}

// Park-Miller rnd00: rndx <- mod(16807 rndx, 2147483647), rn = rndx / 2147483647.
__device__ __forceinline__ double rnd00(double *rndx) {
  const double rnd = mul(16807.0, *rndx);
  *rndx = fmod(rnd, 0.2147483647e10);
  return dvd(*rndx, 0.2147483647e10);
}

// Hop probabilities and the hop (tddft_fssh.f90:2219-2366), one thread.
__global__ void k_fssh_hop(int nst, const double *A, const double *eig, double dtmd, double dttddft, int boltz,
                           double treq, int hop, const double *probinteg, const double *occ_store, double *occ_rec,
                           double *accum, double *rndx, double *bkl_out, int *trans_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double rn = rnd00(rndx);
  double probsum = 0.0;
  int trans = -1;
  for (long i = 0; i < (long)nst * FW; ++i) bkl_out[i] = 0.0;
  for (int s = 0; s < nst; ++s) {
    if (!(occ_store[s] > 0.5)) continue;
    for (int iud = -FN; iud <= FN; ++iud) {
      const int ns = s + iud;
      if (ns < 0 || ns >= nst || ns == s) continue;
      if (occ_store[ns] > 1.5) continue;
      const double boltzmn = (boltz && iud == 1) ? exp(dvd(-sub(eig[ns], eig[s]), treq)) : 1.0;
      const double bkl0 = mul(mul(mul(2.0, dkj(A, nst, ns, s, dtmd)), dttddft), probinteg[(long)s * FW + iud + FN]);
      const double bkl = mul(bkl0, boltzmn);
      bkl_out[(long)s * FW + iud + FN] = bkl;
      if (bkl > 0.0) accum[ns + (long)s * nst] = add(accum[ns + (long)s * nst], bkl);
      const double pb = bkl > 0.0 ? bkl : 0.0;
      if (hop && probsum <= rn && rn < add(probsum, pb)) {
        trans = s * nst + ns;
        occ_rec[s] = sub(occ_rec[s], 1.0);
        occ_rec[ns] = add(occ_rec[ns], 1.0);
      }
      probsum = add(probsum, pb);
    }
  }
  *trans_out = trans;
}

__global__ void k_fssh_init(int nst, double *dnr, double *dni, double *accum) {
  const long n = (long)nst * FW * FW;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    dnr[i] = (i % (FW * FW)) == FN * FW + FN ? 1.0 : 0.0;
    dni[i] = 0.0;
  }
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (long)nst * nst; i += (long)gridDim.x * blockDim.x)
    accum[i] = 0.0;
}
}  // namespace

void fssh_init(int nst, double *dnr, double *dni, double *accum, cudaStream_t st) {
  k_fssh_init<<<std::max(1, std::min(148, (nst * FW * FW + 255) / 256)), 256, 0, st>>>(nst, dnr, dni, accum);
  note_launch();
}

void fssh_step(int nst, const double *A, const double *eig, double dtmd, double dttddft, int boltz, double treq,
               int hop, double *dnr, double *dni, const double *occ_store, double *occ_rec, double *probinteg,
               double *accum, double *rndx, double *bkl, int *trans, cudaStream_t st) {
  k_fssh_prop<<<nst, FT_PROP, 0, st>>>(nst, A, eig, dtmd, dttddft, dnr, dni, occ_store, probinteg);
  note_launch();
  k_fssh_hop<<<1, 32, 0, st>>>(nst, A, eig, dtmd, dttddft, boltz, treq, hop, probinteg, occ_store, occ_rec, accum,
                               rndx, bkl, trans);
  note_launch();
}

}  // namespace qx
