/*
 * ORACLE -- test infrastructure only.  CPU FP64 restatement of QXMD's Kohn-Sham
 * hot path, used by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg as the checker.  It is never linked into or called by the
 * product library.
 *
 * PARITY UNPINNED: QXMD is Fortran + FFTW 3.3.8 and neither a Fortran
 * compiler nor FFTW exists where this was written, and the reference ships no
 * test vectors.  This file follows the reference statement by statement where
 * cited; its own FFT is checked against a direct DFT and numpy's pocketfft in
 * tests/test_oracle.py.
 *
 * Layouts follow the Fortran arrays: a wavefunction band is a real vector of
 * nplwex = 2*(nplw+1) numbers (Re, Im of c(G) for the Gamma-point half
 * sphere), bands are stored one after another (column-major gdcr(nplwex,nb));
 * the FFT grid index is n1 + (n2 + n3*k2)*k1 (n1 fastest), 0-based.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* Host threads of the band-parallel loops.  Every parallel loop below gives
 * each output element to one thread and keeps the serial order of its sums,
 * so results do not depend on the thread count. */
void orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Mixed-radix complex FFT (recursive decimation in time, any factorisation). */
/* out[k] = sum_j in[j] exp(sign*2*pi*i*j*k/n), unscaled.                     */
/* ------------------------------------------------------------------------ */
static int smallest_factor(int n) {
  for (int p = 2; p * p <= n; ++p)
    if (n % p == 0) return p;
  return n;
}

static void fft_rec(const cplx *in, long is, cplx *out, int n, const cplx *w,
                    long wstride, cplx *tmp) {
  if (n == 1) { out[0] = in[0]; return; }
  int p = smallest_factor(n), m = n / p;
  for (int r = 0; r < p; ++r)
    fft_rec(in + r * is, is * p, out + (long)r * m, m, w, wstride * p, tmp);
  for (int k = 0; k < m; ++k)
    for (int q = 0; q < p; ++q) {
      cplx s = 0;
      long kk = k + (long)q * m;
      for (int r = 0; r < p; ++r) {
        long t = ((long)r * kk) % n;
        s += w[t * wstride] * out[(long)r * m + k];
      }
      tmp[kk] = s;
    }
  memcpy(out, tmp, sizeof(cplx) * n);
}

void orc_fft1(cplx *x, int n, int sign) {
  cplx *w = malloc(sizeof(cplx) * n), *in = malloc(sizeof(cplx) * n),
       *tmp = malloc(sizeof(cplx) * n);
  const double tp = 2.0 * acos(-1.0);
  for (int t = 0; t < n; ++t) w[t] = cos(tp * t / n) + sign * I * sin(tp * t / n);
  memcpy(in, x, sizeof(cplx) * n);
  fft_rec(in, 1, x, n, w, 1, tmp);
  free(w); free(in); free(tmp);
}

/* 3D transform along all three axes; sign=+1 backward (unscaled), -1 forward
 * (unscaled -- callers apply 1/N as rfft3 key=1 does, fft3.f90:160-170). */
void orc_fft3(cplx *a, int k1, int k2, int k3, int sign) {
  int nmax = k1 > k2 ? k1 : k2; nmax = nmax > k3 ? nmax : k3;
  cplx *line = malloc(sizeof(cplx) * nmax), *res = malloc(sizeof(cplx) * nmax),
       *tmp = malloc(sizeof(cplx) * nmax), *w = malloc(sizeof(cplx) * nmax);
  const double tp = 2.0 * acos(-1.0);
  int dims[3] = {k1, k2, k3};
  long strides[3] = {1, k1, (long)k1 * k2};
  for (int ax = 0; ax < 3; ++ax) {
    int n = dims[ax];
    for (int t = 0; t < n; ++t) w[t] = cos(tp * t / n) + sign * I * sin(tp * t / n);
    long st = strides[ax];
    long nl = (long)k1 * k2 * k3 / n;
    for (long l = 0; l < nl; ++l) {
      /* decompose line id into base offset */
      long base;
      if (ax == 0) base = l * k1;
      else if (ax == 1) base = (l % k1) + (l / k1) * (long)k1 * k2;
      else base = l;
      for (int j = 0; j < n; ++j) line[j] = a[base + j * st];
      fft_rec(line, 1, res, n, w, 1, tmp);
      for (int j = 0; j < n; ++j) a[base + j * st] = res[j];
    }
  }
  free(line); free(res); free(tmp); free(w);
}

/* Gamma-point inner product 2*sum x*y - x(1)*y(1) (eigen.f90:382-386). */
double orc_dot(const double *x, const double *y, int nplwex) {
  double s = 0.0;
  for (int i = 0; i < nplwex; ++i) s += x[i] * y[i];
  return 2.0 * s - x[0] * y[0];
}

/* wvg2r: half-sphere coefficients -> real psi(r) on the FFT grid
 * (engrad.f90:1527-1546): Hermitian fill at +G/-G, backward transform. */
void orc_wvg2r(const double *c, int nplw, const int *ijk_pos, const int *ijk_neg,
               int k1, int k2, int k3, double *psir) {
  long n = (long)k1 * k2 * k3;
  cplx *z = calloc(n, sizeof(cplx));
  z[ijk_pos[0]] = c[0];
  for (int ig = 1; ig <= nplw; ++ig) {
    z[ijk_pos[ig]] = c[2 * ig] + I * c[2 * ig + 1];
    z[ijk_neg[ig]] = c[2 * ig] - I * c[2 * ig + 1];
  }
  orc_fft3(z, k1, k2, k3, +1);
  for (long i = 0; i < n; ++i) psir[i] = creal(z[i]);
  free(z);
}

/* calnlc: real-space KB projection and back-application
 * (nlkbppr.f90:1773-1900); apk += sum_l vnl_l * (rdelv*clalp_l*sum vnl_l*psi). */
void orc_calnlc(int natom, int lmx, const int *off, const int *mesh,
                const double *vnl, const double *clalp, double rdelv,
                const double *psir, double *apk, double *sumr_out) {
  double sumr[16];
  for (int ia = 0; ia < natom; ++ia) {
    for (int l = 0; l < lmx; ++l) {
      double s = 0.0;
      for (int mm = off[ia]; mm < off[ia + 1]; ++mm) s += vnl[(long)mm * lmx + l] * psir[mesh[mm]];
      sumr[l] = s * rdelv * clalp[l];
      if (sumr_out) sumr_out[ia * lmx + l] = sumr[l];
    }
    for (int l = 0; l < lmx; ++l)
      for (int mm = off[ia]; mm < off[ia + 1]; ++mm)
        apk[mesh[mm]] += vnl[(long)mm * lmx + l] * sumr[l];
  }
}

/* Hamiltonian tables (the module state the Fortran routines read). */
typedef struct {
  int k1, k2, k3, nplw, nplwex;
  const int *ijk_pos, *ijk_neg;
  const double *dkgnrm;   /* nplwex */
  const double *glocal;   /* kfft0 */
  int nlmode;             /* 0 none, 1 G-space KB, 2 real-space KB */
  int nproj;              /* G-space */
  const double *kbg;      /* nplwex * nproj, projector-major */
  const double *vclalp;   /* nproj */
  int natom, lmx;         /* real-space */
  const int *off, *mesh;
  const double *vnl, *clalp;
  double rdelv;
} orc_ham;

/* hcnonloc (engrad.f90:411-606): rhcr += FFT^-1-space V_loc*psi (+ real-space KB),
 * forward transform scaled 1/N, picked at +G for ig = 0..nplw. */
void orc_hcnonloc(const orc_ham *h, const double *c, double *rhcr) {
  long n = (long)h->k1 * h->k2 * h->k3;
  double *psir = malloc(sizeof(double) * n);
  orc_wvg2r(c, h->nplw, h->ijk_pos, h->ijk_neg, h->k1, h->k2, h->k3, psir);
  cplx *z = malloc(sizeof(cplx) * n);
  for (long i = 0; i < n; ++i) z[i] = h->glocal[i] * psir[i];
  if (h->nlmode == 2) {
    double *apk = calloc(n, sizeof(double));
    orc_calnlc(h->natom, h->lmx, h->off, h->mesh, h->vnl, h->clalp, h->rdelv, psir, apk, NULL);
    for (long i = 0; i < n; ++i) z[i] += apk[i];
    free(apk);
  }
  orc_fft3(z, h->k1, h->k2, h->k3, -1);
  const double fin = 1.0 / (double)n;
  for (int ig = 0; ig <= h->nplw; ++ig) {
    cplx v = z[h->ijk_pos[ig]] * fin;
    rhcr[2 * ig] += creal(v);
    rhcr[2 * ig + 1] += cimag(v);
  }
  free(psir); free(z);
}

/* hckbpp_ib_g (nlkbpp.f90:1623-1721): t = 2*sum_{ig>=3} B*c + B(1)*c(1);
 * rhcr += vclalp*B*t.  Projections returned in slm if given. */
void orc_hckbpp(const orc_ham *h, const double *c, double *rhcr, double *slm) {
  int ne = h->nplwex;
  for (int j = 0; j < h->nproj; ++j) {
    const double *b = h->kbg + (long)j * ne;
    double t = 0.0;
    for (int ig = 2; ig < ne; ++ig) t += b[ig] * c[ig];
    t = 2.0 * t + b[0] * c[0];
    if (slm) slm[j] = t;
    double f = h->vclalp[j] * t;
    for (int ig = 0; ig < ne; ++ig) rhcr[ig] += b[ig] * f;
  }
}

/* One full H*x for one vector in the eigen_BKL order (eigen.f90:516-551):
 * kinetic, G-space KB, then local (+ real-space KB). */
void orc_hpsi1(const orc_ham *h, const double *c, double *hc) {
  for (int i = 0; i < h->nplwex; ++i) hc[i] = h->dkgnrm[i] * c[i];
  if (h->nlmode == 1) orc_hckbpp(h, c, hc, NULL);
  orc_hcnonloc(h, c, hc);
}

void orc_hpsi(const orc_ham *h, const double *c, double *hc, int nb) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < nb; ++b) orc_hpsi1(h, c + (long)b * h->nplwex, hc + (long)b * h->nplwex);
}

/* ekinetic2 (engrad.f90:75-127): ekib(i) = 2*<c|T|c>; returns sum occ*<c|T|c>. */
double orc_ekinetic(const orc_ham *h, const double *c, int nb, const double *occ, double *ekib) {
  double ekin = 0.0;
  int ne = h->nplwex;
  for (int b = 0; b < nb; ++b) {
    const double *x = c + (long)b * ne;
    double s = 0.0;
    for (int i = 0; i < ne; ++i) s += h->dkgnrm[i] * x[i] * x[i];
    s = 2.0 * s - h->dkgnrm[0] * x[0] * x[0];
    if (occ) ekin += occ[b] * s;
    if (ekib) ekib[b] = 2.0 * s;
  }
  return ekin;
}

/* prpcg (eigen.f90:1093-1113): Teter-Payne-Allan preconditioner. */
static void prpcg(double ekib, const double *dkgnrm, int ne, double *prcd) {
  for (int ig = 0; ig < ne; ++ig) {
    double e15 = 1.5 * ekib;
    double x = dkgnrm[ig] / e15;
    double t = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x));
    double x2 = x * x, x4 = x2 * x2;
    t = t / (t + 16.0 * x4);
    prcd[ig] = t * 2.0 / e15;
  }
}

typedef struct {
  int itermx, iteremx, noband;
  double tolera, roughfzan, roughfeig, threinn, wdinner;
  int ccreal4;          /* 1: the lower-band snapshot cgjr is real*4 */
  int sequential;       /* 1: one rank holds all bands (Gauss-Seidel order) */
} orc_cgparm;

/* eigen_BKL (eigen.f90:199-938) for all bands.  Band ib is projected
 * against the snapshot cgjr of bands 0..ib-1 (subgs3, engrad.f90:1072-1191),
 * itself (subgs4, engrad.f90:1196-1248), and updated by the BKL 2x2 step.
 * pm->sequential = 0: the snapshot is the entry copy of every band, which is
 * the reference run with one band per rank.  pm->sequential = 1: after band
 * ib's last step its final vector replaces its snapshot column
 * (cgjr(:,ib) = gdcr(:,ibb), eigen.f90:699), which is the reference run on
 * one rank, where later bands see the updated lower bands.
 * lhcunt=.true., lortho=.false.: rhcr holds H*gdcr on entry.
 * Outputs eig, bzan (final residual) and nriter per band. */
/* The CG steps of one band ib (the body of the band loop of eigen_BKL,
 * eigen.f90:283-776) against the snapshot snap of bands 0..ib-1; work arrays
 * prcd, gnk, hnk (ne) and prod (ib). */
static void bkl_band(const orc_ham *h, const orc_cgparm *pm, int ib, double *gdcr, double *rhcr,
                     const double *ekib, const double *snap, double *eig, double *bzan, int *nriter,
                     double *prcd, double *gnk, double *hnk, double *prod) {
  int ne = h->nplwex;
  {
    double *x = gdcr + (long)ib * ne, *hx = rhcr + (long)ib * ne;
    prpcg(ekib[ib], h->dkgnrm, ne, prcd);
    double e = orc_dot(x, hx, ne);
    for (int i = 0; i < ne; ++i) gnk[i] = e * x[i] - hx[i];
    double zansa = orc_dot(gnk, gnk, ne);
    int iter = 0, izcnt = 0, lreset = 1;
    double zansab = zansa, z000re = zansa, x000re = 1.0e10, eigb = e, dinnerx = 0.0, betk = 0.0;
    for (;;) {
      ++iter;
      for (int i = 0; i < ne; ++i) gnk[i] *= prcd[i];
      double zansap = orc_dot(gnk, gnk, ne);
      double beta = 0.0;
      if (lreset) { for (int i = 0; i < ne; ++i) hnk[i] = 0.0; }
      else beta = zansap / betk;
      lreset = 0;
      for (int i = 0; i < ne; ++i) hnk[i] = gnk[i] + beta * hnk[i];
      betk = zansap;
      /* subgs3 against the snapshot of lower bands */
      for (int jb = 0; jb < ib; ++jb) prod[jb] = orc_dot(snap + (long)jb * ne, hnk, ne);
      for (int jb = 0; jb < ib; ++jb) {
        const double *cj = snap + (long)jb * ne;
        for (int i = 0; i < ne; ++i) hnk[i] -= prod[jb] * cj[i];
      }
      /* subgs4 against the current vector */
      double hhx = orc_dot(x, hnk, ne);
      for (int i = 0; i < ne; ++i) hnk[i] -= hhx * x[i];
      double cai = orc_dot(hnk, hx, ne);
      orc_hpsi1(h, hnk, gnk);
      double cbi = orc_dot(hnk, gnk, ne);
      double hhi = orc_dot(hnk, hnk, ne);
      double dtnew, alpsq;
      if (hhi > 0.0) {
        double h11 = e, h12 = cai / sqrt(hhi), h21 = h12, h22 = cbi / hhi;
        double enew = 0.5 * (h11 + h22 - sqrt((h11 + h22) * (h11 + h22) - 4.0 * (h11 * h22 - h12 * h21)));
        dtnew = (enew - h11) / h12 / sqrt(hhi);
        double alpsq2 = 1.0 / (1.0 + dtnew * (0.0 + dtnew * hhi));
        alpsq = sqrt(alpsq2);
        e = enew;
      } else {
        /* line minimisation (eigen.f90:624-695), reached only for h = 0 */
        hhx = orc_dot(hnk, x, ne);
        double c0 = e, c1 = cai, c2 = cbi, c3 = hhi, c4 = 2.0 * hhx;
        double s0 = c0 * c4 - c1, s1 = c0 * c3 - c2, s2 = c1 * c3 - c2 * c4;
        double sr = s1 * s1 - s2 * s0;
        dtnew = (sr > 0.0) ? (-s1 - sqrt(sr)) / s2 : -1.0;
        if (dtnew > 0.0) {
          double dinner = sqrt(1.0 / (1.0 + dtnew * dtnew * hhi));
          if (dinner < pm->threinn) dtnew = 0.0;
          if (dinner < dinnerx * pm->wdinner) dtnew = 0.0;
          if (dinner > dinnerx) dinnerx = dinner;
        }
        double d2 = dtnew * dtnew;
        double alpsq2 = 1.0 / (1.0 + dtnew * c4 + d2 * c3);
        e = (c0 + dtnew * c1 + d2 * c2) * alpsq2;
        alpsq = sqrt(alpsq2);
      }
      for (int i = 0; i < ne; ++i) x[i] = alpsq * (x[i] + dtnew * hnk[i]);
      for (int i = 0; i < ne; ++i) hx[i] = alpsq * (hx[i] + dtnew * gnk[i]);
      for (int i = 0; i < ne; ++i) gnk[i] = e * x[i] - hx[i];
      zansa = orc_dot(gnk, gnk, ne);
      double de = fabs(eigb - e);
      int stop = (ib < pm->noband && iter >= pm->itermx) ||
                 (ib >= pm->noband && iter >= pm->iteremx) || zansa < pm->tolera ||
                 de < pm->tolera || zansa < z000re * pm->roughfzan ||
                 (iter > 1 && de < x000re * pm->roughfeig);
      if (stop) break;
      if (iter == 1) x000re = de;
      if (zansa > zansab) {
        if (++izcnt > 20) { izcnt = 0; lreset = 1; }
      }
      zansab = zansa;
      eigb = e;
    }
    eig[ib] = e;
    if (bzan) bzan[ib] = zansa;
    if (nriter) nriter[ib] = iter;
  }
}

/* eigen_BKL for all bands (see bkl_band).  In the one-band-per-rank order
 * every band reads only the entry snapshot, so the bands run in parallel;
 * the one-rank order is serial. */
void orc_eigen_bkl(const orc_ham *h, const orc_cgparm *pm, int nb, double *gdcr,
                   double *rhcr, const double *ekib, double *eig, double *bzan, int *nriter) {
  int ne = h->nplwex;
  double *snap = malloc(sizeof(double) * ne * (long)nb);
  for (long i = 0; i < (long)ne * nb; ++i)
    snap[i] = pm->ccreal4 ? (double)(float)gdcr[i] : gdcr[i];
  if (pm->sequential) {
    double *prcd = malloc(sizeof(double) * ne), *gnk = malloc(sizeof(double) * ne),
           *hnk = malloc(sizeof(double) * ne), *prod = malloc(sizeof(double) * (nb + 1));
    for (int ib = 0; ib < nb; ++ib) {
      bkl_band(h, pm, ib, gdcr, rhcr, ekib, snap, eig, bzan, nriter, prcd, gnk, hnk, prod);
      const double *x = gdcr + (long)ib * ne;
      for (int i = 0; i < ne; ++i) snap[(long)ib * ne + i] = pm->ccreal4 ? (double)(float)x[i] : x[i];
    }
    free(prcd); free(gnk); free(hnk); free(prod);
  } else {
#pragma omp parallel
    {
      double *prcd = malloc(sizeof(double) * ne), *gnk = malloc(sizeof(double) * ne),
             *hnk = malloc(sizeof(double) * ne), *prod = malloc(sizeof(double) * (nb + 1));
#pragma omp for schedule(dynamic, 1)
      for (int ib = 0; ib < nb; ++ib)
        bkl_band(h, pm, ib, gdcr, rhcr, ekib, snap, eig, bzan, nriter, prcd, gnk, hnk, prod);
      free(prcd); free(gnk); free(hnk); free(prod);
    }
  }
  free(snap);
}

/* rsdecmp + rsinvcd (schmidt.f90:428-544): Cholesky S = L L^T then L^-1, both
 * in the lower triangle of s (column-major n x n).  Returns 0, or 1+i if the
 * pivot of row i is not > 1e-30 (schmidt.f90:256-267). */
int orc_cholinv(double *s, int n) {
  const double zero = 1.0e-30;
#define S(i, j) s[(long)(j) * n + (i)]
  int bad = 0;
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < i; ++k) S(i, i) -= S(i, k) * S(i, k);
    if (S(i, i) > zero) {
      S(i, i) = sqrt(S(i, i));
      for (int k = 0; k < i; ++k) {
        double sik = S(i, k);
        for (int j = i + 1; j < n; ++j) S(j, i) -= S(j, k) * sik;
      }
      double r = 1.0 / S(i, i);
      for (int j = i + 1; j < n; ++j) S(j, i) *= r;
    } else {
      for (int j = i; j < n; ++j) S(j, i) = 0.0;
      if (!bad) bad = 1 + i;
    }
  }
  for (int i = 0; i < n - 1; ++i)
    for (int j = i + 1; j < n; ++j) S(i, j) = 0.0;
  if (bad) return bad;
  double *w = malloc(sizeof(double) * n);
  for (int i = 0; i < n; ++i) {
    double r = 1.0 / S(i, i);
    for (int j = i + 1; j < n; ++j) S(j, i) *= r;
    S(i, i) = r;
  }
  for (int j = n - 2; j >= 0; --j) {
    for (int i = j + 1; i < n; ++i) w[i] = 0.0;
    for (int k = j + 1; k < n; ++k) {
      double skj = S(k, j);
      for (int i = j + 1; i < n; ++i) w[i] += S(i, k) * skj;
    }
    for (int i = j + 1; i < n; ++i) S(i, j) = -w[i];
  }
  free(w);
#undef S
  return 0;
}

/* schmidt2 (schmidt.f90:117-378): S = C^T C (Gamma metric), Cholesky, L^-1,
 * C(:,ib) <- sum_{jb<=ib} Linv(ib,jb) C(:,jb).  Returns orc_cholinv's code;
 * the lower-triangular L^-1 is left in linv (n x n, column-major) if given. */
int orc_schmidt(double *c, int ne, int nb, double *linv) {
  double *s = calloc((long)nb * nb, sizeof(double));
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j <= i; ++j) s[(long)j * nb + i] = orc_dot(c + (long)j * ne, c + (long)i * ne, ne);
  int rc = orc_cholinv(s, nb);
  if (rc) { free(s); return rc; }
  /* the in-place update of schmidt.f90:284-313 runs ib downwards so that
   * column ib still reads the old columns jb <= ib; writing into a copy gives
   * the same sums and lets the columns run in parallel */
  double *out = malloc(sizeof(double) * (long)ne * nb);
#pragma omp parallel for schedule(dynamic, 1)
  for (int ib = nb - 1; ib >= 0; --ib) {
    double *buf = out + (long)ib * ne;
    for (int i = 0; i < ne; ++i) buf[i] = 0.0;
    for (int jb = 0; jb <= ib; ++jb) {
      double p = s[(long)jb * nb + ib];
      const double *cj = c + (long)jb * ne;
      for (int i = 0; i < ne; ++i) buf[i] += p * cj[i];
    }
  }
  memcpy(c, out, sizeof(double) * (long)ne * nb);
  if (linv) memcpy(linv, s, sizeof(double) * nb * nb);
  free(s); free(out);
  return 0;
}

/* hmatrix2 (engrad.f90:845-956): H(jb,ib) = <c_jb|hc_ib>, symmetric fill,
 * eig(ib) = H(ib,ib). */
void orc_hmatrix(const double *c, const double *hc, int ne, int nb, double *hm, double *eig) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int ib = 0; ib < nb; ++ib)
    for (int jb = 0; jb <= ib; ++jb) {
      double p = orc_dot(hc + (long)ib * ne, c + (long)jb * ne, ne);
      hm[(long)ib * nb + jb] = p;
      hm[(long)jb * nb + ib] = p;
      if (jb == ib && eig) eig[ib] = p;
    }
}

/* gradresnv (engrad.f90:1013-1067): per-band squared residual norms; returns
 * max in zmax and occupation-weighted sum in zsum. */
void orc_gradres(const double *c, const double *hc, const double *eig, const double *occ,
                 int ne, int nb, double *prod, double *zmax, double *zsum) {
  double m = 0.0, s = 0.0;
  for (int ib = 0; ib < nb; ++ib) {
    const double *x = c + (long)ib * ne, *y = hc + (long)ib * ne;
    double p = 0.0;
    for (int i = 0; i < ne; ++i) { double r = eig[ib] * x[i] - y[i]; p += r * r; }
    double r0 = eig[ib] * x[0] - y[0];
    p = 2.0 * p - r0 * r0;
    if (prod) prod[ib] = p;
    if (p > m) m = p;
    s += p * occ[ib];
  }
  *zmax = m; *zsum = s;
}

/* Symmetric eigen-decomposition by cyclic Jacobi rotations in round-robin
 * pair order (Brent-Luk), FP64.  a (n x n column-major) is destroyed; v gets
 * the eigenvectors as columns sorted by ascending eigenvalue, each with its
 * largest-magnitude component made positive (first such index on ties).
 * Returns the number of sweeps, or -1 if not converged in maxsweep. */
int orc_jacobi(double *a, int n, double *w, double *v, int maxsweep) {
#define A(i, j) a[(long)(j) * n + (i)]
#define V(i, j) v[(long)(j) * n + (i)]
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) V(i, j) = (i == j) ? 1.0 : 0.0;
  int m = n + (n & 1);
  int *top = malloc(sizeof(int) * m);
  for (int i = 0; i < m; ++i) top[i] = i;
  int sweeps = -1;
  for (int sw = 0; sw < maxsweep; ++sw) {
    double off = 0.0, tot = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) { double x = A(i, j) * A(i, j); tot += x; if (i != j) off += x; }
    if (off <= 1e-30 * tot || off == 0.0) { sweeps = sw; break; }
    for (int r = 0; r < m - 1; ++r) {
      for (int k = 0; k < m / 2; ++k) {
        int p = top[k], q = top[m - 1 - k];
        if (p >= n || q >= n) continue;
        if (p > q) { int t = p; p = q; q = t; }
        double apq = A(p, q);
        if (apq == 0.0) continue;
        double app = A(p, p), aqq = A(q, q);
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int i = 0; i < n; ++i) {            /* columns p, q */
          double aip = A(i, p), aiq = A(i, q);
          A(i, p) = c * aip - s * aiq;
          A(i, q) = s * aip + c * aiq;
        }
        for (int i = 0; i < n; ++i) {            /* rows p, q */
          double api = A(p, i), aqi = A(q, i);
          A(p, i) = c * api - s * aqi;
          A(q, i) = s * api + c * aqi;
        }
        for (int i = 0; i < n; ++i) {
          double vip = V(i, p), viq = V(i, q);
          V(i, p) = c * vip - s * viq;
          V(i, q) = s * vip + c * viq;
        }
      }
      /* rotate positions 1..m-1 */
      int last = top[m - 1];
      for (int i = m - 1; i > 1; --i) top[i] = top[i - 1];
      top[1] = last;
    }
  }
  free(top);
  for (int i = 0; i < n; ++i) w[i] = A(i, i);
  /* selection sort ascending with column swaps */
  for (int i = 0; i < n; ++i) {
    int k = i;
    for (int j = i + 1; j < n; ++j) if (w[j] < w[k]) k = j;
    if (k != i) {
      double t = w[i]; w[i] = w[k]; w[k] = t;
      for (int r = 0; r < n; ++r) { double x = V(r, i); V(r, i) = V(r, k); V(r, k) = x; }
    }
  }
  for (int j = 0; j < n; ++j) {
    int k = 0; double mx = -1.0;
    for (int i = 0; i < n; ++i) if (fabs(V(i, j)) > mx) { mx = fabs(V(i, j)); k = i; }
    if (V(k, j) < 0.0) for (int i = 0; i < n; ++i) V(i, j) = -V(i, j);
  }
#undef A
#undef V
  return sweeps;
}

/* untrycore (eigen.f90:1456-1514): C <- C*U for C (ne x nb), U (nb x nb). */
void orc_rotate(double *c, int ne, int nb, const double *u) {
  double *out = malloc(sizeof(double) * (long)ne * nb);
#pragma omp parallel for schedule(static)
  for (int ib = 0; ib < nb; ++ib)
    for (int i = 0; i < ne; ++i) {
      double s = 0.0;
      for (int jb = 0; jb < nb; ++jb) s += u[(long)ib * nb + jb] * c[(long)jb * ne + i];
      out[(long)ib * ne + i] = s;
    }
  memcpy(c, out, sizeof(double) * (long)ne * nb);
  free(out);
}

/* softchg (chgdns.f90:388-454): rho(r) = sum_b occ_b/Omega * psi_b(r)^2. */
void orc_softchg(const orc_ham *h, const double *c, int nb, const double *occ, double rvol,
                 double *rho) {
  long n = (long)h->k1 * h->k2 * h->k3;
  /* bands in chunks: psi(r) of a chunk in parallel, then every grid point
   * sums its chunk in band order, which keeps the serial order of the sums */
  int chunk = 2 * orc_get_threads();
  if (chunk > nb) chunk = nb;
  if (chunk < 1) chunk = 1;
  double *psir = malloc(sizeof(double) * n * chunk);
  for (long i = 0; i < n; ++i) rho[i] = 0.0;
  for (int b0 = 0; b0 < nb; b0 += chunk) {
    int m = nb - b0 < chunk ? nb - b0 : chunk;
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < m; ++k)
      orc_wvg2r(c + (long)(b0 + k) * h->nplwex, h->nplw, h->ijk_pos, h->ijk_neg, h->k1, h->k2, h->k3,
                psir + (long)k * n);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
      double r = rho[i];
      for (int k = 0; k < m; ++k) {
        double p = psir[(long)k * n + i];
        r += p * p * (occ[b0 + k] / rvol);
      }
      rho[i] = r;
    }
  }
  free(psir);
}

/* xclda + VXC (vxc.f90:961-1018, 2063-2108): Perdew-Zunger LDA with the
 * reference's single-precision literals; vexc/eexc in Ry.  Returns the four
 * energy sums (eexc, evexc, ecor, evcor) times 2*rdelv. */
void orc_xclda(const double *rho, long n, double rdelv, double *vexc, double *eeexc, double *en4) {
  const double pi4 = 12.56637061436;
  const double a1 = -0.4582, b1 = -0.1423, b2 = (double)1.0529f, b3 = (double)0.3334f;
  const double c1 = -0.0480, c2 = (double)0.0311f, c3 = (double)-0.0116f, c4 = (double)0.0020f;
  double s[4] = {0, 0, 0, 0};
  for (long m = 0; m < n; ++m) {
    double rh = rho[m];
    if (rh < 1e-30) { vexc[m] = 0.0; if (eeexc) eeexc[m] = 0.0; continue; }
    double rs = pow(3.0 / (pi4 * rh), 1.0 / 3.0);
    double ex = a1 / rs, vx = 4.0 * ex / 3.0, ec, vc;
    if (rs >= 1.0) {
      double bunb = 1.0 + b2 * sqrt(rs) + b3 * rs;
      ec = b1 / bunb;
      vc = ec * (1.0 + (b2 * sqrt(rs) / 6.0 + b3 * rs / 3.0) / bunb);
    } else {
      ec = c1 + c2 * log(rs) + c3 * rs + c4 * rs * log(rs);
      vc = ec - (c2 + (c3 + c4) * rs + c4 * rs * log(rs)) / 3.0;
    }
    vexc[m] = 2.0 * (vx + vc);
    if (eeexc) eeexc[m] = 2.0 * (ex + ec);
    s[0] += ex * rh; s[1] += vx * rh; s[2] += ec * rh; s[3] += vc * rh;
  }
  for (int i = 0; i < 4; ++i) en4[i] = s[i] * 2.0 * rdelv;
}

/* ------------------------------------------------------------------------ */
/* TDDFT-FSSH in the density-matrix representation: tddft_fssh_dm
 * (tddft_fssh.f90:1989-2402) for one spin channel (nspnmx = 1), without the
 * decoherence branch (lfssh_dish = .false.).  States s = 0..nst-1 of a band
 * window (noband = noccmx = nst); phis(k, j) = <psi_k(t)|psi_j(t+dt)> at
 * phis[k + j*nst]; eig(nst) in Ry.  Per state s a (2*3+1)^2 complex density
 * matrix dn[s][j+3][k+3] (nupdn = 3) is integrated by RK4 over
 * nstep = int(dtmd/dttddft) substeps; then the hop probabilities and one
 * Park-Miller draw (rnd00, funcs.f90:1673-1689) decide a transition.
 * Every expression keeps the reference's evaluation order (left to right).
 * accum(news, s) at accum[news + s*nst]; bkl_out[s*7 + iud+3] the hop
 * probability of each pair (0 where none).  Returns -1, or s*nst + news of
 * the accepted transition. */
#define FS_N 3
#define FS_W 7
static double rnd00(double *rndx) {
  const double rnda = 16807.0, rndm = 0.2147483647e10;
  double rnd = rnda * *rndx;
  *rndx = fmod(rnd, rndm);
  return *rndx / rndm;
}

double orc_rnd00(double *rndx) { return rnd00(rndx); }

int orc_fssh_dm(int nst, const double *phis, const double *eig, double dtmd, double dttddft, int boltz,
                double treq, int hop, double *dnr, double *dni, double *accum, double *occ_rec, double *rndx,
                double *bkl_out) {
#define PH(k, j) phis[(long)(k) + (long)(j) * nst]
#define DKJ(k, j) (-(PH(k, j) - PH(j, k)) / 2.0 / dtmd)
#define DR(s, j, k) dnr[((long)(s) * FS_W + (j) + FS_N) * FS_W + (k) + FS_N]
#define DI(s, j, k) dni[((long)(s) * FS_W + (j) + FS_N) * FS_W + (k) + FS_N]
  double rn = rnd00(rndx);
  double *occ_store = malloc(sizeof(double) * nst);
  double *probinteg = calloc((size_t)nst * FS_W, sizeof(double));
  memcpy(occ_store, occ_rec, sizeof(double) * nst);
  const double rkc[4] = {0.0, dttddft / 2.0, dttddft / 2.0, dttddft};
  const int nstep = (int)(dtmd / dttddft);
  double kr[4][FS_W][FS_W], ki[4][FS_W][FS_W], dmtr[FS_W][FS_W], dmti[FS_W][FS_W];
  for (int s = 0; s < nst; ++s) {
    int ldm = 0;
    if (occ_store[s] > 0.5)
      for (int iud = -FS_N; iud <= FS_N; ++iud) {
        int ns = s + iud;
        if (ns < 0 || ns >= nst || ns == s) continue;
        if (occ_store[ns] > 1.5) continue;
        ldm = 1;
      }
    if (!ldm) continue;
    const int n1 = -FS_N > -s ? -FS_N : -s, n2 = FS_N < nst - 1 - s ? FS_N : nst - 1 - s;
    for (int i = 0; i < nstep; ++i) {
      /* stage 1 from dn itself (tddft_fssh.f90:2126-2141) */
      for (int kb = n1; kb <= n2; ++kb)
        for (int jb = n1; jb <= n2; ++jb) {
          const int k = s + kb, j = s + jb;
          double r = (eig[j] - eig[k]) * DI(s, jb, kb);
          double m = -(eig[j] - eig[k]) * DR(s, jb, kb);
          for (int lb = n1; lb <= n2; ++lb) {
            const int l = s + lb;
            r = r - DR(s, jb, lb) * DKJ(l, k) + DR(s, lb, kb) * DKJ(j, l);
            m = m - DI(s, jb, lb) * DKJ(l, k) + DI(s, lb, kb) * DKJ(j, l);
          }
          kr[0][jb + FS_N][kb + FS_N] = r;
          ki[0][jb + FS_N][kb + FS_N] = m;
        }
      /* stages 2-4 (2143-2166) */
      for (int irk = 1; irk < 4; ++irk) {
        for (int kb = n1; kb <= n2; ++kb)
          for (int jb = n1; jb <= n2; ++jb) {
            dmtr[jb + FS_N][kb + FS_N] = DR(s, jb, kb) + rkc[irk] * kr[irk - 1][jb + FS_N][kb + FS_N];
            dmti[jb + FS_N][kb + FS_N] = DI(s, jb, kb) + rkc[irk] * ki[irk - 1][jb + FS_N][kb + FS_N];
          }
        for (int kb = n1; kb <= n2; ++kb)
          for (int jb = n1; jb <= n2; ++jb) {
            const int k = s + kb, j = s + jb;
            double r = (eig[j] - eig[k]) * dmti[jb + FS_N][kb + FS_N];
            double m = -(eig[j] - eig[k]) * dmtr[jb + FS_N][kb + FS_N];
            for (int lb = n1; lb <= n2; ++lb) {
              const int l = s + lb;
              r = r - dmtr[jb + FS_N][lb + FS_N] * DKJ(l, k) + dmtr[lb + FS_N][kb + FS_N] * DKJ(j, l);
              m = m - dmti[jb + FS_N][lb + FS_N] * DKJ(l, k) + dmti[lb + FS_N][kb + FS_N] * DKJ(j, l);
            }
            kr[irk][jb + FS_N][kb + FS_N] = r;
            ki[irk][jb + FS_N][kb + FS_N] = m;
          }
      }
      /* RK4 update (2168-2177) */
      for (int kb = n1; kb <= n2; ++kb)
        for (int jb = n1; jb <= n2; ++jb) {
          const int a = jb + FS_N, b = kb + FS_N;
          DR(s, jb, kb) = DR(s, jb, kb) + (kr[0][a][b] + 2.0 * kr[1][a][b] + 2.0 * kr[2][a][b] + kr[3][a][b]) *
                                              dttddft / 6.0;
          DI(s, jb, kb) = DI(s, jb, kb) + (ki[0][a][b] + 2.0 * ki[1][a][b] + 2.0 * ki[2][a][b] + ki[3][a][b]) *
                                              dttddft / 6.0;
        }
      /* transition probability integral (2179-2188) */
      for (int iud = -FS_N; iud <= FS_N; ++iud) {
        int ns = s + iud;
        if (ns < 0 || ns >= nst || ns == s) continue;
        probinteg[(long)s * FS_W + iud + FS_N] += DR(s, iud, 0) / DR(s, 0, 0);
      }
    }
  }
  /* probabilities and the hop (2219-2366) */
  int trans = -1;
  double probsum = 0.0;
  if (bkl_out) for (long i = 0; i < (long)nst * FS_W; ++i) bkl_out[i] = 0.0;
  for (int s = 0; s < nst; ++s) {
    if (!(occ_store[s] > 0.5)) continue;
    for (int iud = -FS_N; iud <= FS_N; ++iud) {
      int ns = s + iud;
      if (ns < 0 || ns >= nst || ns == s) continue;
      if (occ_store[ns] > 1.5) continue;
      double boltzmn = (boltz && iud == 1) ? exp(-(eig[ns] - eig[s]) / treq) : 1.0;
      double bkl0 = 2.0 * DKJ(ns, s) * dttddft * probinteg[(long)s * FS_W + iud + FS_N];
      double bkl = bkl0 * boltzmn;
      if (bkl_out) bkl_out[(long)s * FS_W + iud + FS_N] = bkl;
      if (bkl > 0.0) accum[(long)ns + (long)s * nst] += bkl;
      double pb = bkl > 0.0 ? bkl : 0.0;
      if (hop && probsum <= rn && rn < probsum + pb) {
        trans = s * nst + ns;
        occ_rec[s] = occ_rec[s] - 1.0;
        occ_rec[ns] = occ_rec[ns] + 1.0;
      }
      probsum = probsum + pb;
    }
  }
  free(occ_store);
  free(probinteg);
  return trans;
#undef PH
#undef DKJ
#undef DR
#undef DI
}
