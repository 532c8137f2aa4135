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

// One warp per state s: lane e < 49 owns rho(a - 3, b - 3) with
// (a, b) = (e / 7, e % 7), lanes 0..16 also e + 32.  The couplings of an
// element's row a and column b and its energy difference stay in registers
// for the whole MD step; the stage matrix is shared through shared memory,
// zero outside the window (the zero couplings there add exact zeros, so the
// sums equal those over the window alone).
__global__ void __launch_bounds__(32) k_fssh_prop(int nst, const double *A, const double *eig, double dtmd,
                                                 double dttddft, double *dnr, double *dni, const double *occ_store,
                                                 double *probinteg) {
  const int s = blockIdx.x;
  const int lane = threadIdx.x;
  __shared__ double D[FW][FW], E[FW], Sr[FW][FW], Si[FW][FW];
  if (lane < FW) probinteg[(long)s * FW + lane] = 0.0;
  if (!fs_active(occ_store, nst, s)) return;
  const int n1 = max(-FN, -s), n2 = min(FN, nst - 1 - s);
  for (int e = lane; e < FW * FW; e += 32) {
    const int a = e / FW, b = e % FW;
    const bool ok = a - FN >= n1 && a - FN <= n2 && b - FN >= n1 && b - FN <= n2;
    D[a][b] = ok ? dkj(A, nst, s + a - FN, s + b - FN, dtmd) : 0.0;
    Sr[a][b] = 0.0;
    Si[a][b] = 0.0;
  }
  if (lane < FW) E[lane] = (lane - FN >= n1 && lane - FN <= n2) ? eig[s + lane - FN] : 0.0;
  __syncwarp();
  // own elements, their couplings and energy differences
  int ea[2], eb[2];
  bool own[2];
  double dr[2], di[2], de[2], drow[2][FW], dcol[2][FW];
  double *gr = dnr + (long)s * FW * FW, *gi = dni + (long)s * FW * FW;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const int e = lane + 32 * t;
    ea[t] = min(e / FW, FW - 1);
    eb[t] = e % FW;
    own[t] = e < FW * FW && ea[t] - FN >= n1 && ea[t] - FN <= n2 && eb[t] - FN >= n1 && eb[t] - FN <= n2;
    dr[t] = own[t] ? gr[e] : 0.0;
    di[t] = own[t] ? gi[e] : 0.0;
    de[t] = sub(E[ea[t]], E[eb[t]]);
#pragma unroll
    for (int l = 0; l < FW; ++l) {
      drow[t][l] = D[ea[t]][l];   // d(j, l)
      dcol[t][l] = D[l][eb[t]];   // d(l, k)
    }
  }
  const double rkc[4] = {0.0, dvd(dttddft, 2.0), dvd(dttddft, 2.0), dttddft};
  const int nstep = (int)(dtmd / dttddft);
  // probability integrals of the neighbours this lane owns (elements (iud + 3, 3))
  bool pown[2];
  double pint[2] = {0.0, 0.0};
#pragma unroll
  for (int t = 0; t < 2; ++t) pown[t] = own[t] && eb[t] == FN && ea[t] != FN;
  for (int step = 0; step < nstep; ++step) {
    double kr[4][2], ki[4][2];
#pragma unroll
    for (int irk = 0; irk < 4; ++irk) {
      __syncwarp();   // every lane has read the previous stage input
#pragma unroll
      for (int t = 0; t < 2; ++t)
        if (own[t]) {
          Sr[ea[t]][eb[t]] = irk == 0 ? dr[t] : add(dr[t], mul(rkc[irk], kr[irk - 1][t]));
          Si[ea[t]][eb[t]] = irk == 0 ? di[t] : add(di[t], mul(rkc[irk], ki[irk - 1][t]));
        }
      __syncwarp();
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int a = ea[t], b = eb[t];
        double r = mul(de[t], Si[a][b]);
        double m = mul(-de[t], Sr[a][b]);
#pragma unroll
        for (int l = 0; l < FW; ++l) {
          r = add(sub(r, mul(Sr[a][l], dcol[t][l])), mul(Sr[l][b], drow[t][l]));
          m = add(sub(m, mul(Si[a][l], dcol[t][l])), mul(Si[l][b], drow[t][l]));
        }
        kr[irk][t] = r;
        ki[irk][t] = m;
      }
    }
    // RK4 update: rho + (k1 + 2 k2 + 2 k3 + k4) dttddft / 6 (tddft_fssh.f90:2168-2177)
#pragma unroll
    for (int t = 0; t < 2; ++t)
      if (own[t]) {
        const double sr = add(add(add(kr[0][t], mul(2.0, kr[1][t])), mul(2.0, kr[2][t])), kr[3][t]);
        const double si = add(add(add(ki[0][t], mul(2.0, ki[1][t])), mul(2.0, ki[2][t])), ki[3][t]);
        dr[t] = add(dr[t], dvd(mul(sr, dttddft), 6.0));
        di[t] = add(di[t], dvd(mul(si, dttddft), 6.0));
      }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < 2; ++t)
      if (own[t]) Sr[ea[t]][eb[t]] = dr[t];
    __syncwarp();
#pragma unroll
    for (int t = 0; t < 2; ++t)
      if (pown[t]) pint[t] = add(pint[t], dvd(Sr[ea[t]][FN], Sr[FN][FN]));
  }
#pragma unroll
  for (int t = 0; t < 2; ++t)
    if (own[t]) {
      const int e = lane + 32 * t;
      gr[e] = dr[t];
      gi[e] = di[t];
    }
#pragma unroll
  for (int t = 0; t < 2; ++t)
    if (pown[t]) probinteg[(long)s * FW + ea[t]] = pint[t];
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
  k_fssh_prop<<<nst, 32, 0, st>>>(nst, A, eig, dtmd, dttddft, dnr, dni, occ_store, probinteg);
  note_launch();
  k_fssh_hop<<<1, 32, 0, st>>>(nst, A, eig, dtmd, dttddft, boltz, treq, hop, probinteg, occ_store, occ_rec, accum,
                               rndx, bkl, trans);
  note_launch();
}

}  // namespace qx
