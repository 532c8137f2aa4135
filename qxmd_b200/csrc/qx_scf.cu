// Density-side kernels of one SCF iteration, all FP64: Hartree potential
// (harting, engrad.f90:1673-1743), Perdew-Zunger LDA (xclda/VXC,
// vxc.f90:961-1018, 2063-2108, with the reference's single-precision
// literals), glocal assembly (pwlda.f90:1984-2024) and Kerker-filtered
// linear density mixing.  Reductions write per-block partial sums that a
// single block adds in a fixed order, so results are deterministic.
#include "qx_internal.h"
#include "qx_scf.h"

namespace qx {

constexpr int RB = 256;

__device__ __forceinline__ double block_sum_rb(double v, double *red) { return block_sum(v, red); }

// |G|^2 of every grid point, or -1 outside the density sphere (and 0 at G=0).
__global__ void k_grid_g2(int k1, int k2, int k3, double c00, double c01, double c02, double c10, double c11,
                          double c12, double c20, double c21, double c22, double ecutdens, double *__restrict__ g2) {
  const long n = (long)k1 * k2 * k3;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int i1 = (int)(i % k1), i2 = (int)((i / k1) % k2), i3 = (int)(i / ((long)k1 * k2));
    const double d1 = i1 <= k1 / 2 ? i1 : i1 - k1;
    const double d2 = i2 <= k2 / 2 ? i2 : i2 - k2;
    const double d3 = i3 <= k3 / 2 ? i3 : i3 - k3;
    const double gx = c00 * d1 + c01 * d2 + c02 * d3;
    const double gy = c10 * d1 + c11 * d2 + c12 * d3;
    const double gz = c20 * d1 + c21 * d2 + c22 * d3;
    const double s = gx * gx + gy * gy + gz * gz;
    g2[i] = (s <= ecutdens) ? s : -1.0;
  }
}

__global__ void k_real_to_cplx(const double *__restrict__ r, const double *__restrict__ r2, double2 *__restrict__ z,
                               long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    z[i] = make_double2(r2 ? r[i] - r2[i] : r[i], 0.0);
}

// V_H(G) = 8 pi rho(G) / |G|^2 inside the density sphere; E_H partial sums
// (Omega/2) sum_G V_H(G) conj(rho(G)).
__global__ void __launch_bounds__(RB) k_hartree(double2 *__restrict__ z, const double *__restrict__ g2, long n,
                                                double half_vol, double *__restrict__ part) {
  __shared__ double red[RB / 32];
  double e = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double q = g2[i];
    double2 v = z[i];
    if (q > 0.0) {
      const double f = 8.0 * 3.14159265358979323846 / q;
      e += f * (v.x * v.x + v.y * v.y);
      v.x *= f; v.y *= f;
    } else {
      v.x = 0.0; v.y = 0.0;
    }
    z[i] = v;
  }
  e = block_sum_rb(e, red);
  if (threadIdx.x == 0) part[blockIdx.x] = e * half_vol;
}

// Kerker filter of a density difference in G space: d(G) *= G^2/(G^2+q0^2)
// inside the density sphere, 0 at G = 0 and outside.
__global__ void k_kerker(double2 *__restrict__ z, const double *__restrict__ g2, long n, double q02) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double q = g2[i];
    double2 v = z[i];
    const double f = (q > 0.0) ? q / (q + q02) : 0.0;
    v.x *= f; v.y *= f;
    z[i] = v;
  }
}

// PZ LDA on rho, glocal = vloc + Re(vh) + vxc; partial sums of
// eps_xc*rho and vxc*rho (times rdelv).
template <typename T>
__global__ void __launch_bounds__(RB) k_xc_glocal(const double *__restrict__ rho, const double *__restrict__ vloc,
                                                  const double2 *__restrict__ vh, long n, double rdelv,
                                                  double *__restrict__ glocal, T *__restrict__ glocal_t,
                                                  double *__restrict__ part) {
  __shared__ double red[RB / 32];
  const double pi4 = 12.56637061436;
  const double a1 = -0.4582, b1 = -0.1423, b2 = (double)1.0529f, b3 = (double)0.3334f;
  const double c1 = -0.0480, c2 = (double)0.0311f, c3 = (double)-0.0116f, c4 = (double)0.0020f;
  double sx = 0.0, sv = 0.0;
  for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < n; m += (long)gridDim.x * blockDim.x) {
    const double rh = rho[m];
    double vexc = 0.0, eexc = 0.0;
    if (rh >= 1e-30) {
      const double rs = cbrt(3.0 / (pi4 * rh));
      const double ex = a1 / rs, vx = 4.0 * ex / 3.0;
      double ec, vc;
      if (rs >= 1.0) {
        const double srs = sqrt(rs);
        const double bunb = 1.0 + b2 * srs + b3 * rs;
        ec = b1 / bunb;
        vc = ec * (1.0 + (b2 * srs / 6.0 + b3 * rs / 3.0) / bunb);
      } else {
        const double lr = log(rs);
        ec = c1 + c2 * lr + c3 * rs + c4 * rs * lr;
        vc = ec - (c2 + (c3 + c4) * rs + c4 * rs * lr) / 3.0;
      }
      vexc = 2.0 * (vx + vc);
      eexc = 2.0 * (ex + ec);
    }
    const double g = vloc[m] + vh[m].x + vexc;
    glocal[m] = g;
    glocal_t[m] = (T)g;
    sx += eexc * rh;
    sv += vexc * rh;
  }
  sx = block_sum_rb(sx, red);
  sv = block_sum_rb(sv, red);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sx * rdelv;
    part[2 * blockIdx.x + 1] = sv * rdelv;
  }
}

// rho_in += beta * Re(filtered difference); partial sums of the residual
// |rho_out - rho_in|^2 * rdelv taken before the update.
__global__ void __launch_bounds__(RB) k_mix(double *__restrict__ rho_in, const double *__restrict__ rho_out,
                                            const double2 *__restrict__ dfilt, long n, double beta, double rdelv,
                                            double *__restrict__ part) {
  __shared__ double red[RB / 32];
  double s = 0.0;
  for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < n; m += (long)gridDim.x * blockDim.x) {
    const double d = rho_out[m] - rho_in[m];
    s += d * d;
    rho_in[m] += beta * dfilt[m].x;
  }
  s = block_sum_rb(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s * rdelv;
}

// out[k] = sum over nblk partial sums with stride `stride` and offset k.
// One warp per output: lane-strided partial sums, then a shuffle tree (a fixed
// order, so the result does not change from run to run).
// Fixed-order sums of the partials: lane l of a warp adds blocks l, l + 32,
// ... four at a time into four running sums (the loads of a round are
// independent), then the lanes are combined by shuffles.
__global__ void k_reduce(const double *__restrict__ part, int nblk, int stride, int nk, double *__restrict__ out) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = w; k < nk; k += blockDim.x >> 5) {
    double s4[4] = {0.0, 0.0, 0.0, 0.0};
    int b = lane;
    for (; b + 96 < nblk; b += 128)
#pragma unroll
      for (int u = 0; u < 4; ++u) s4[u] += part[(long)(b + 32 * u) * stride + k];
    for (; b < nblk; b += 32) s4[0] += part[(long)b * stride + k];
    double s = (s4[0] + s4[1]) + (s4[2] + s4[3]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[k] = s;
  }
}

// sum_b occ_b * w_b, one warp: lane l takes bands l, l + 32, ...
__global__ void k_band_energy(const double *__restrict__ w, const double *__restrict__ occ, int nb,
                              double *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int b = lane; b < nb; b += 32) s += occ[b] * w[b];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) *out = s;
}

// ---- Pulay mixing -------------------------------------------------------------
// Device state (PulayState): cnt entries of history, order[] their slots
// (oldest first), A[slot][slot] the residual metric, coef[] the mixing
// coefficients by order position, slot the entry being added.  The host
// never reads any of it, so a mixing step has no host round trip.

// Start a step: a fresh history after a reset or a full one, else append;
// the new entry takes the lowest free slot.
__global__ void k_pulay_push(PulayState p, int reset) {
  if (threadIdx.x != 0) return;
  if (reset || p.s->reset_next || p.s->cnt >= p.itratn) {
    p.s->cnt = 0;
    p.s->reset_next = 0;
  }
  int slot = 0;
  for (; slot < p.itratn; ++slot) {
    bool used = false;
    for (int i = 0; i < p.s->cnt; ++i) used |= (p.s->order[i] == slot);
    if (!used) break;
  }
  p.s->order[p.s->cnt++] = slot;
  p.s->slot = slot;
}

// z = rho_in + i (rho_out - rho_in): both real fields in one complex FFT.
__global__ void k_pack2(const double *__restrict__ rin, const double *__restrict__ rout, double2 *__restrict__ z,
                        long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    z[i] = make_double2(rin[i], rout[i] - rin[i]);
}

// Unpack the transform of two real fields: with Z = F(a + i b),
// A(G) = (Z(G) + Z(-G)^*)/2 and B(G) = (Z(G) - Z(-G)^*)/(2i).  u = A (every G),
// d = B inside the density sphere without G = 0, else 0.
__global__ void k_pulay_store(const double2 *__restrict__ z, const double *__restrict__ g2, int k1, int k2, int k3,
                              PulayState p) {
  const long n = (long)k1 * k2 * k3;
  const int slot = p.s->slot;
  double2 *u = p.u + slot * n, *d = p.d + slot * n;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int i1 = (int)(i % k1), i2 = (int)((i / k1) % k2), i3 = (int)(i / ((long)k1 * k2));
    const long j = (i1 ? k1 - i1 : 0) + (long)k1 * ((i2 ? k2 - i2 : 0) + (long)k2 * (i3 ? k3 - i3 : 0));
    const double2 a = z[i], b = z[j];
    u[i] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
    d[i] = g2[i] > 0.0 ? make_double2(0.5 * (a.y + b.y), -0.5 * (a.x - b.x)) : make_double2(0.0, 0.0);
  }
}

// Partial sums of Omega sum_G Re(d_i^* d_new) w(G), w = (G^2 + q1)/G^2, for
// every history entry i (order position) against the new one.
__global__ void __launch_bounds__(RB) k_pulay_dots(const double *__restrict__ g2, long n, PulayState p, double rvol,
                                                   double *__restrict__ part) {
  __shared__ double red[RB / 32];
  const int cnt = p.s->cnt;
  const double2 *dn = p.d + p.s->slot * n;
  const double2 *di[PULAY_MAX];
#pragma unroll
  for (int i = 0; i < PULAY_MAX; ++i) di[i] = p.d + (i < cnt ? p.s->order[i] : 0) * n;
  double acc[PULAY_MAX];
#pragma unroll
  for (int i = 0; i < PULAY_MAX; ++i) acc[i] = 0.0;
  for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < n; m += (long)gridDim.x * blockDim.x) {
    const double q = g2[m];
    if (q <= 0.0) continue;
    const double w = (q + p.q1) / q;
    const double2 b = dn[m];
#pragma unroll
    for (int i = 0; i < PULAY_MAX; ++i)
      if (i < cnt) {
        const double2 a = di[i][m];
        acc[i] += (a.x * b.x + a.y * b.y) * w;
      }
  }
#pragma unroll
  for (int i = 0; i < PULAY_MAX; ++i) {
    if (i >= cnt) break;   // cnt is uniform across the block
    const double t = block_sum_rb(acc[i], red);
    if (threadIdx.x == 0) part[(long)blockIdx.x * PULAY_MAX + i] = t * rvol;
  }
}

// Mixing coefficients (one thread; cnt <= PULAY_MAX): record the new metric
// row, then c = rowsums(A^-1) / sum(A^-1) over the history, dropping the
// oldest entry while A is singular and restarting from the new entry when
// its centre element is tiny (chgdns.f90:1013-1096).  The inverse is Gauss-
// Jordan elimination with partial pivoting of A / max|A_ij|; "singular"
// means |det| < 1e-30 as in INVERS (funcs.f90:1-56).
__global__ void k_pulay_solve(PulayState p, const double *__restrict__ adot) {
  if (threadIdx.x != 0) return;
  PulayDev &s = *p.s;
  const int M = PULAY_MAX;
  for (int i = 0; i < s.cnt; ++i) {
    s.A[s.order[i] * M + s.slot] = adot[i];
    s.A[s.slot * M + s.order[i]] = adot[i];
  }
  double w[M * M], inv[M * M];
  for (;;) {
    const int k = s.cnt;
    if (k == 1) {
      s.coef[0] = 1.0;
      break;
    }
    const int c = (k + 1) / 2 - 1;
    const double amax = fabs(s.A[s.order[c] * M + s.order[c]]);
    if (amax < 1.0e-15) {
      s.order[0] = s.slot;
      s.cnt = 1;
      continue;
    }
    double elmax = 0.0;
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j) elmax = fmax(elmax, fabs(s.A[s.order[i] * M + s.order[j]]));
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j) {
        w[i * M + j] = s.A[s.order[i] * M + s.order[j]] / elmax;
        inv[i * M + j] = (i == j) ? 1.0 : 0.0;
      }
    double det = 1.0;
    for (int col = 0; col < k; ++col) {
      int piv = col;
      for (int r = col + 1; r < k; ++r)
        if (fabs(w[r * M + col]) > fabs(w[piv * M + col])) piv = r;
      if (piv != col) {
        det = -det;
        for (int j = 0; j < k; ++j) {
          double t = w[col * M + j]; w[col * M + j] = w[piv * M + j]; w[piv * M + j] = t;
          t = inv[col * M + j]; inv[col * M + j] = inv[piv * M + j]; inv[piv * M + j] = t;
        }
      }
      const double pv = w[col * M + col];
      det *= pv;
      if (pv == 0.0) break;
      const double rp = 1.0 / pv;
      for (int j = 0; j < k; ++j) { w[col * M + j] *= rp; inv[col * M + j] *= rp; }
      for (int r = 0; r < k; ++r) {
        if (r == col) continue;
        const double f = w[r * M + col];
        if (f == 0.0) continue;
        for (int j = 0; j < k; ++j) { w[r * M + j] -= f * w[col * M + j]; inv[r * M + j] -= f * inv[col * M + j]; }
      }
    }
    if (!(fabs(det) >= 1.0e-30)) {
      for (int i = 0; i + 1 < k; ++i) s.order[i] = s.order[i + 1];
      s.cnt = k - 1;
      continue;
    }
    // rows of (A/elmax)^-1; the common factor cancels in c
    double tot = 0.0;
    for (int i = 0; i < k; ++i) {
      double r = 0.0;
      for (int j = 0; j < k; ++j) r += inv[i * M + j];
      s.coef[i] = r;
      tot += r;
    }
    for (int i = 0; i < k; ++i) s.coef[i] /= tot;
    break;
  }
  if (s.cnt == p.itratn) s.reset_next = 1;
}

// z(G) = sum_i c_i (u_i(G) + K(G) d_i(G)), K = aslh G^2/(G^2 + bslh) inside
// the density sphere (0 at G = 0 and outside, where d_i is 0 anyway).
__global__ void k_pulay_new(const double *__restrict__ g2, long n, PulayState p, double aslh, double bslh,
                            double2 *__restrict__ z) {
  const int cnt = p.s->cnt;
  for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < n; m += (long)gridDim.x * blockDim.x) {
    const double q = g2[m];
    const double kf = q > 0.0 ? aslh * q / (q + bslh) : 0.0;
    double2 r = make_double2(0.0, 0.0);
    for (int i = 0; i < cnt; ++i) {
      const long o = p.s->order[i] * n + m;
      const double c = p.s->coef[i];
      const double2 u = p.u[o], d = p.d[o];
      r.x += c * (u.x + kf * d.x);
      r.y += c * (u.y + kf * d.y);
    }
    z[m] = r;
  }
}

// rho_in <- Re z; partial sums of |rho_out - rho_in|^2 * rdelv before the update.
__global__ void __launch_bounds__(RB) k_take_real(double *__restrict__ rho_in, const double *__restrict__ rho_out,
                                                  const double2 *__restrict__ z, long n, double rdelv,
                                                  double *__restrict__ part) {
  __shared__ double red[RB / 32];
  double s = 0.0;
  for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < n; m += (long)gridDim.x * blockDim.x) {
    const double d = rho_out[m] - rho_in[m];
    s += d * d;
    rho_in[m] = z[m].x;
  }
  s = block_sum_rb(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s * rdelv;
}

// ---- launchers -------------------------------------------------------------
void pulay_push(const PulayState &p, int reset, cudaStream_t st) { k_pulay_push<<<1, 32, 0, st>>>(p, reset); note_launch(); }
void pack2(const double *rin, const double *rout, double2 *z, long n, cudaStream_t st) {
  k_pack2<<<148 * 4, 256, 0, st>>>(rin, rout, z, n); note_launch();
}
void pulay_store(const double2 *z, const double *g2, int k1, int k2, int k3, const PulayState &p, cudaStream_t st) {
  k_pulay_store<<<148 * 4, 256, 0, st>>>(z, g2, k1, k2, k3, p); note_launch();
}
void pulay_coef(const double *g2, long n, const PulayState &p, double rvol, double *part, double *adot,
                cudaStream_t st) {
  k_pulay_dots<<<SCF_NBLK, RB, 0, st>>>(g2, n, p, rvol, part); note_launch();
  k_reduce<<<1, 32 * PULAY_MAX, 0, st>>>(part, SCF_NBLK, PULAY_MAX, PULAY_MAX, adot); note_launch();
  k_pulay_solve<<<1, 32, 0, st>>>(p, adot); note_launch();
}
void pulay_new(const double *g2, long n, const PulayState &p, double aslh, double bslh, double2 *z, cudaStream_t st) {
  k_pulay_new<<<148 * 4, 256, 0, st>>>(g2, n, p, aslh, bslh, z); note_launch();
}
void take_real(double *rho_in, const double *rho_out, const double2 *z, long n, double rdelv, double *part,
               double *out, cudaStream_t st) {
  k_take_real<<<SCF_NBLK, RB, 0, st>>>(rho_in, rho_out, z, n, rdelv, part); note_launch();
  k_reduce<<<1, 32, 0, st>>>(part, SCF_NBLK, 1, 1, out); note_launch();
}

void grid_g2(int k1, int k2, int k3, const double *cross, double ecutdens, double *g2, cudaStream_t st) {
  k_grid_g2<<<148 * 4, 256, 0, st>>>(k1, k2, k3, cross[0], cross[3], cross[6], cross[1], cross[4], cross[7],
                                    cross[2], cross[5], cross[8], ecutdens, g2); note_launch();
}

void real_to_cplx(const double *r, const double *r2, double2 *z, long n, cudaStream_t st) {
  k_real_to_cplx<<<148 * 4, 256, 0, st>>>(r, r2, z, n); note_launch();
}

void hartree_g(double2 *z, const double *g2, long n, double half_vol, double *part, double *out, cudaStream_t st) {
  k_hartree<<<SCF_NBLK, RB, 0, st>>>(z, g2, n, half_vol, part); note_launch();
  k_reduce<<<1, 32, 0, st>>>(part, SCF_NBLK, 1, 1, out); note_launch();
}

void kerker(double2 *z, const double *g2, long n, double q02, cudaStream_t st) {
  k_kerker<<<148 * 4, 256, 0, st>>>(z, g2, n, q02); note_launch();
}

template <typename T>
void xc_glocal(const double *rho, const double *vloc, const double2 *vh, long n, double rdelv, double *glocal,
               T *glocal_t, double *part, double *out2, cudaStream_t st) {
  k_xc_glocal<T><<<SCF_NBLK, RB, 0, st>>>(rho, vloc, vh, n, rdelv, glocal, glocal_t, part); note_launch();
  k_reduce<<<1, 64, 0, st>>>(part, SCF_NBLK, 2, 2, out2); note_launch();
}
template void xc_glocal<float>(const double *, const double *, const double2 *, long, double, double *, float *,
                               double *, double *, cudaStream_t);
template void xc_glocal<double>(const double *, const double *, const double2 *, long, double, double *, double *,
                                double *, double *, cudaStream_t);

void mix(double *rho_in, const double *rho_out, const double2 *dfilt, long n, double beta, double rdelv, double *part,
         double *out, cudaStream_t st) {
  k_mix<<<SCF_NBLK, RB, 0, st>>>(rho_in, rho_out, dfilt, n, beta, rdelv, part); note_launch();
  k_reduce<<<1, 32, 0, st>>>(part, SCF_NBLK, 1, 1, out); note_launch();
}

void band_energy(const double *w, const double *occ, int nb, double *out, cudaStream_t st) {
  k_band_energy<<<1, 32, 0, st>>>(w, occ, nb, out); note_launch();
}

}  // namespace qx
