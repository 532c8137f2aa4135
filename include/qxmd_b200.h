/*
 * qxmd_b200 -- C ABI of the B200 (sm_100a) Kohn-Sham hot path of QXMD.
 *
 * Plain C: opaque context, host or device pointers and sizes, int status.
 * Layouts are those of the Fortran arrays the reference subroutines take:
 * a wavefunction block gdcr(nplwex, nband) is column-major real*8 with
 * nplwex = 2*(nplw+1) (Re, Im of c(G) on the Gamma-point half sphere); the
 * FFT grid index is n1 + (n2 + n3*k2)*k1 with n1 fastest.
 *
 * Two precisions per context: QX_PREC_FP64 (the plain drop-in) keeps every
 * device array in FP64; QX_PREC_MIXED keeps wavefunctions, FFTs and the band
 * contractions in FP32 and the nband x nband Cholesky / eigen-decomposition,
 * energies and density in FP64.  Host transfer functions always take real*8.
 *
 * Every function returns QX_OK (0) or an error code; qx_last_error() gives
 * the message.  Nothing here falls back to the CPU.
 */
#ifndef QXMD_B200_H
#define QXMD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define QX_OK 0
#define QX_ERR_ARG 1       /* bad argument or unsupported size          */
#define QX_ERR_CUDA 2      /* CUDA runtime error                        */
#define QX_ERR_NOTPD 3     /* <psi_i|psi_j> not positive definite       */
#define QX_ERR_EIG 4       /* subspace eigen-decomposition not converged */
#define QX_ERR_STATE 5     /* call order (e.g. untryt before hmatrix)   */

#define QX_PREC_FP64 0
#define QX_PREC_MIXED 1

#define QX_NL_NONE 0
#define QX_NL_GSPACE 1     /* KB projectors in G space (lking = .false.) */
#define QX_NL_RSPACE 2     /* KB projectors in real space (lking = .true.) */

/* qx_hpsi flags */
#define QX_HPSI_KINETIC 1
#define QX_HPSI_NONLOCAL 2
#define QX_HPSI_ACCUMULATE 4

/* Real-space KB: at most 9 projectors per atom (s, three p, five d). */
#define QX_KBR_MAX_LMX 9

typedef struct qx_ctx qx_ctx;

/* Convergence controls of the CG band update; defaults of
 * modules.f90:171-182 (toleig, roughfeig, roughfzan, threinn, wdinner,
 * itermx, iteremx) and noband (number of occupied bands). */
typedef struct {
  int itermx, iteremx, noband;
  double tolera, roughfzan, roughfeig, threinn, wdinner;
  int ccreal4;   /* FP64 contexts: round the lower-band snapshot to real*4 */
  int sequential; /* 0: all bands at once against the entry vectors (the
                   * reference run with one band per rank); 1: bands one after
                   * another, each against the final vectors of the bands below
                   * (the reference run on one rank; one graph launch per call) */
} qx_cgparm;

/* Result of one SCF iteration (energies in Ry). */
typedef struct {
  double etot;       /* band energy - E_H + E_xc - int V_xc rho + E_ion   */
  double eband;      /* sum occ * eigenvalue (after subspace rotation)  */
  double ehartree;
  double exc;
  double evxc;
  double resid;      /* int (rho_out - rho_in)^2                         */
  double zmax;       /* max band residual before the CG (gradres)        */
  int ncg_hpsi;      /* H|psi> band applications spent in the CG        */
  int eig_clusters;     /* eigenvalue clusters of the subspace problem */
} qx_scf_out;

const char *qx_last_error(void);
int qx_version(void);
/* Number of kernels this library has launched in the process (all contexts). */
long qx_launch_count(void);
/* FP32 band contractions in the process that ran on the CUDA-core GEMM
 * instead of the tensor cores (a column map or device column count, or
 * operands outside the TMA rules that could not be restaged). */
long qx_gemm_fallbacks(void);

/* ---- set-up (module state of the reference, uploaded once per geometry) -- */

/* Grid and G sphere: the outputs of reclat/set_rciprl (reclat.f90:167-475,
 * modules.f90:1402-1603).  ijkgd: 2*nplw+1 zero-based grid indices of G index
 * -nplw..nplw (ijkgd(-nplw:nplw) of reclat.f90:256-274 minus one);
 * dkgnrm: |G|^2 per real component, 2*(nplw+1).  stream: cudaStream_t or 0. */
int qx_create(qx_ctx **ctx, int precision, int kfft1, int kfft2, int kfft3, int nplw, const int *ijkgd,
              const double *dkgnrm, int nband, void *stream);
int qx_destroy(qx_ctx *ctx);

/* glocal(kfft0): total local potential on the FFT grid (pwlda.f90:1984-2024). */
int qx_set_glocal(qx_ctx *ctx, const double *glocal);
/* G-space KB tables, eqlmr_(nplwex, nproj) and vclalp(nproj)
 * (setbgq nlkbpp.f90:2135-2187, setnlc_g nlkbpp.f90:1236-1279). */
int qx_set_kb_g(qx_ctx *ctx, int nproj, const double *eqlmr, const double *vclalp);
/* The same tables built on the device, for MD steps.  Once per cell
 * (setqlm nlkbpp.f90:2196-2247 with tbqlma of ppkb.f90:3228-3236):
 *   ntype species of lmx projector channels each, channel ch = l + lmx * it;
 *   tbqlm((mxqlm + 1), lmx * ntype): radial tables at |G| = k * dlqlm(it);
 *   qlm((nplw + 1), nlm): angular factors; channel ch uses column lmidx[ch];
 *   even[ch]: 1 for even l (litoll: cos/-sin), 0 for odd l (-sin/-cos);
 *   vclalp(lmx * ntype): KB energy of each channel;
 *   ngabc(3, nplw + 1): integer coordinates of the half-sphere G vectors.
 * The radial table must reach the largest |G| (2 int(|G|/(2 dl)) + 2 <= mxqlm). */
int qx_set_kb_builder(qx_ctx *ctx, int ntype, int lmx, int mxqlm, const double *dlqlm, const double *tbqlm, int nlm,
                      const double *qlm, const int *lmidx, const int *even, const double *vclalp, const int *ngabc);
/* Once per geometry (setbgq nlkbpp.f90:2135-2187 with the phases of
 * stscfn_pw pwlda.f90:5711-5850): eqlmr_ and vclalp of natom atoms of
 * species ityp(natom) (0-based) at fractional coordinates satm(3, natom),
 * projector j = l + lmx * a.  Reuses the table buffers when the projector
 * count is unchanged, so captured SCF-iteration graphs stay valid.  When
 * force tables were set (qx_set_force_tables, same natom and projector
 * count) their species, phases and KB derivative tables follow the new
 * geometry too, so qx_forces needs no new qx_set_force_tables. */
int qx_build_kb_g(qx_ctx *ctx, int natom, const int *ityp, const double *satm);
/* Reads back the G-space KB tables in use (eqlmr_(nplwex, nproj), vclalp(nproj);
 * either pointer may be null), converted to double. */
int qx_get_kb_g(qx_ctx *ctx, double *eqlmr, double *vclalp);
/* Real-space KB tables (setnlc nlkbppr.f90:1010-1768, used by calnlc
 * nlkbppr.f90:1773-1900): atom a owns points off[a]..off[a+1]-1 with
 * zero-based grid index mesh[] and projector values vnl[point*lmx + l];
 * clalp(lmx) = clalp_ncr; rdelv = volume per grid point.  1 <= lmx <=
 * QX_KBR_MAX_LMX; species with fewer projectors than lmx carry zero columns
 * (the reference's lmx(it) differs by species; one stride serves all here). */
int qx_set_kb_r(qx_ctx *ctx, int natom, int lmx, const int *off, const int *mesh, const double *vnl,
                const double *clalp, double rdelv);
/* The real-space tables built on the device, for MD steps (setnlc
 * nlkbppr.f90:1010-1560).  Once per cell: ntype species of lmx projectors each
 * (1 <= lmx <= QX_KBR_MAX_LMX; s, p, d), radial tables tabnl((mxnl + 1),
 * lmx * ntype) at r = k * dltnl(it), projector
 * radius rcut(ntype), dtabnl (nullable, same shape): g'(r)/r of each radial
 * table g, for the projector gradients of the forces (tbfnl of fnnlcl2),
 * poly(lmx * ntype): the real solid-harmonic polynomial
 * that multiplies each channel's radial value (0: 1; 1-3: x, y, z; 4-8: xy,
 * yz, zx, x^2 - y^2, 3z^2 - r^2 of the displacement from the atom), clalp(lmx)
 * KB energies, rdelv the volume per grid point, rba(3, 3) the lattice
 * vectors as columns (row-major here: rba[3 * x + j] = component x of
 * vector j).  The sphere must fit in half the cell along every axis. */
int qx_set_kb_r_builder(qx_ctx *ctx, int ntype, int lmx, int mxnl, const double *dltnl, const double *rcut,
                        const double *tabnl, const double *dtabnl, const int *poly, const double *clalp, double rdelv,
                        const double *rba);
/* Per-channel projector radii (rmxnlc(la, it) of setnlc nlkbppr.f90:1405-1431,
 * which gives each angular channel la its own point list, numsnl(la, i) points
 * of meshnl): rcl(lmx, ntype), rcl[l + lmx * it] the radius of the channel of
 * projector l of species it, each in (0, rcut(it)]; the species radius given
 * to qx_set_kb_r_builder must be the largest of its channels'.  The device
 * keeps one list per atom, the points within rcut(it), and a projector is zero
 * (value and gradient) beyond its own channel's radius, so that calnlc's
 * per-channel sums and fnnlcl2's are reproduced exactly (the added terms are
 * zeros).  Until this is called every channel has the species radius.  Takes
 * effect at the next qx_build_kb_r. */
int qx_set_kb_r_channel_radii(qx_ctx *ctx, const double *rcl);
/* Once per geometry: the points of every atom (species ityp(natom), 0-based,
 * fractional coordinates satm(3, natom)) within its projector radius, their
 * projector values, and the x-line index of the real-space KB kernels.  The
 * buffers grow by 25 % when the point count outgrows them (captured graphs
 * are then dropped); otherwise they are reused in place. */
int qx_build_kb_r(qx_ctx *ctx, int natom, const int *ityp, const double *satm);
/* Reads back the real-space tables in use: *npts, and when not null
 * off(natom + 1), mesh(npts), vnl(lmx * npts) (double). */
int qx_get_kb_r(qx_ctx *ctx, int *npts, int *off, int *mesh, double *vnl);
int qx_set_nlmode(qx_ctx *ctx, int mode);
/* occ(nband) and the cell volume (softchg weights occ/rvol, chgdns.f90:421). */
int qx_set_occ(qx_ctx *ctx, const double *occ, double rvol);

/* ---- host <-> device (real*8 host arrays) ------------------------------ */
int qx_put_psi(qx_ctx *ctx, const double *gdcr);
int qx_get_psi(qx_ctx *ctx, double *gdcr);
int qx_put_hpsi(qx_ctx *ctx, const double *rhcr);
int qx_get_hpsi(qx_ctx *ctx, double *rhcr);
int qx_get_eig(qx_ctx *ctx, double *eig);
int qx_get_rho(qx_ctx *ctx, double *rho);
int qx_put_rho(qx_ctx *ctx, const double *rho);
int qx_get_glocal(qx_ctx *ctx, double *glocal);
/* Device pointers of the resident arrays: 0 psi, 1 hpsi, 2 rho_in (double),
 * 3 rho_out (double), 4 eig (double), 5 the local pseudopotential of
 * qx_scf_init / qx_build_vloc (double, kfft0).  psi/hpsi are double or float
 * by precision. */
void *qx_dev_ptr(qx_ctx *ctx, int which);
int qx_sync(qx_ctx *ctx);

/* ---- hot path on device-resident data ---------------------------------- */

/* hc = [hc +] T c + V_loc c [+ V_NL c] for nb bands of device array c
 * (leading dimension nplwex, the context's precision): hcnonloc
 * (engrad.f90:411-606) with the kinetic term (eigen.f90:335) and KB part
 * (hckbpp_ib_g nlkbpp.f90:1623-1721 or calnlc) chosen by flags. */
int qx_hpsi(qx_ctx *ctx, const void *c, void *hc, int nb, int flags);
/* ekinetic2 (engrad.f90:75-127): ekib(b) = 2 <psi_b|T|psi_b>; *ekin = sum occ <T>. */
int qx_ekinetic(qx_ctx *ctx, double *ekin, double *ekib);
/* enonloc2 + ekinetic2 HC products for all bands: hpsi = H psi. */
int qx_enonloc(qx_ctx *ctx);
/* hmatrix2 (engrad.f90:845-956): H_sub = <psi|H|psi>, eig = diag. */
int qx_hmatrix(qx_ctx *ctx, double *hsub);
/* Allocation-free band matrix.  No counterpart in the reference: an extra
 * entry point for host programs that cannot call cudaMalloc once their run
 * has started -- codes that carve all device memory out of one pool sized at
 * start-up, or run where a further allocation could fail or stall the time
 * step.  It computes what qx_hmatrix computes before symmetrising, on device
 * arrays the caller owns and without a context:
 *   hsub(j, i) = 2 sum_g c(g, j) hc(g, i) - c(1, j) hc(1, i)
 * for all j, i < nb (FP64, column-major nb x nb, leading dimension nb; c and
 * hc column-major nplwex x nb), as a split-K GEMM whose partial sums live in
 * a 16 MiB file-scope device array (QX_HMATRIX_STATIC_SCRATCH_BYTES) that
 * every GPU loading this library holds until exit.  Returns QX_ERR_ARG for
 * nb > QX_HMATRIX_STATIC_MAX_NB (two nb x nb partials must fit).  The first
 * call on each device looks up that array's device address (with the device
 * current) and should come before any stream capture.  Under CUDA's lazy
 * module loading (the default) the array is reserved when its code module
 * first loads on a device, which in a program that calls only this entry
 * point is that first call: a caller that sizes and locks its memory pool at
 * start-up should make one call then (or run with CUDA_MODULE_LOADING=EAGER,
 * which reserves it when the library loads).  All calls share the
 * one array and it keeps the last call's partials; each call writes every
 * partial it reads, so nothing needs clearing, but calls that overlap on the
 * GPU (other streams, other host threads) race on it.  Enqueued on `stream`
 * (cudaStream_t or 0); the result is ready when that stream is. */
#define QX_HMATRIX_STATIC_SCRATCH_BYTES 16777216
#define QX_HMATRIX_STATIC_MAX_NB 1024
int qx_hmatrix_static(const double *c, const double *hc, int nplwex, int nb, double *hsub, void *stream);
/* gradresnv (engrad.f90:1013-1067). */
int qx_gradres(qx_ctx *ctx, double *prod, double *zmax, double *zsum);
/* untryt2 (eigen.f90:1171-1331): diagonalise the last H_sub, psi <- psi U;
 * eigenvalues ascending into ev (nullable). */
int qx_untryt(qx_ctx *ctx, double *ev);
/* untryhc2 (eigen.f90:1383-1451): hpsi <- hpsi U with the same U. */
int qx_untryhc(qx_ctx *ctx);
/* eigen_BKL (eigen.f90:199-938) for all bands; needs hpsi = H psi and the
 * ekib of the last qx_ekinetic.  nriter (nullable): iterations per band. */
int qx_eigen(qx_ctx *ctx, const qx_cgparm *p, int *nriter, int *nhpsi);
/* schmidt2 (schmidt.f90:117-378): psi <- psi L^-T. */
int qx_schmidt(qx_ctx *ctx);
/* softchg (chgdns.f90:388-454): rho_out(r) = sum occ/Omega psi(r)^2. */
int qx_softchg(qx_ctx *ctx);

/* ---- one SCF iteration (pwlda.f90:1628-3700 order) --------------------- */
/* vloc(kfft0): local pseudopotential on the grid; cross: 2*pi*reciprocal
 * vectors, column-major 3x3; eion: ion-ion energy added to etot. */
int qx_scf_init(qx_ctx *ctx, const double *vloc, const double *cross, double ecutdens, double eion, double mixbeta,
                double kerker_q0);
/* Density mixing after qx_scf_init.  itratn >= 2: Pulay mixing
 * (mxchgg_pulay, chgdns.f90:954-1120; imxchg = 1) with itratn history entries
 * (at most 16), residual metric (G^2 + q1)/G^2 from cmetric
 * (chgdns.f90:661-668), Kerker factor mixbeta G^2/(G^2 + kerker_q0^2) (aslh,
 * bslh of qx_scf_init); itratn 0 or 1: Kerker-filtered linear mixing (the
 * default).  Reference defaults: itratn 10, cmetric 20, aslh 0.8, bslh 0.64. */
int qx_scf_mixing(qx_ctx *ctx, int itratn, double cmetric);
/* rho_in <- rho_out of the current psi (start of an SCF run; restarts the
 * Pulay history). */
int qx_scf_rho_from_psi(qx_ctx *ctx);
int qx_scf_iteration(qx_ctx *ctx, const qx_cgparm *p, qx_scf_out *out);
/* One SCF iteration on host arrays, for a host program that keeps gdcr on
 * the host between iterations (pwlda_md's loop, S/pwlda.f90:1628-3700):
 * psi_in (nplwex x nband, real*8) is uploaded while the iteration builds
 * the potential from the density, which does not need it (null: keep the
 * device wavefunctions), H|psi> waits for it, and the results are read back
 * as soon as each is final, on a stream of their own: psi_out after
 * schmidt2, while the density and the mixing still run; rho_out (kfft0, the
 * output density of softchg) after softchg; eig_out (nband) at the end.  Any
 * pointer may be null; page-locked host buffers let the copies overlap the
 * iteration (pageable ones still work, synchronously).  psi_in and psi_out
 * may be the same buffer.  Returns when every copy has landed. */
int qx_scf_iteration_host(qx_ctx *ctx, const qx_cgparm *p, qx_scf_out *out, const double *psi_in, double *psi_out,
                          double *rho_out, double *eig_out);
/* The same iteration in two halves, for many cells at once: qx_scf_launch
 * enqueues it on the context's stream (graph replay, nothing waits);
 * qx_scf_result waits for that stream and reads the results.  Launching every
 * cell before reading any lets independent cells run concurrently. */
int qx_scf_launch(qx_ctx *ctx, const qx_cgparm *p);
int qx_scf_result(qx_ctx *ctx, qx_scf_out *out);

/* ---- FP64 refinement sweep --------------------------------------------- */
/* dst (an FP64 context of the same cell, after qx_scf_init) takes over src's
 * state on the device: psi widened to FP64, src's rho_out as the next input
 * density, the Pulay history restarted.  A few qx_scf_iteration calls on dst
 * then refine a mixed-precision SCF solution to FP64. */
int qx_refine_from(qx_ctx *dst, qx_ctx *src);

/* ---- autotuner --------------------------------------------------------- */
/* Times this context's launch choices on its own buffers and keeps the
 * fastest: the K-split of each tensor-core contraction shape (shared by
 * contexts of equal sizes) and, for FP32, the fused plane kernels against the
 * generic y/x passes of the FFT pipeline.  Overwrites only scratch buffers;
 * call after set-up and before the SCF iterations (captured iteration graphs
 * are dropped).  report (nullable): a one-line summary. */
int qx_autotune(qx_ctx *ctx, char *report, int report_len);

/* ---- TDDFT-FSSH nonadiabatic overlaps --------------------------------- */
/* Keep the current psi as the previous step's wavefunctions (gdcr_rec). */
int qx_tddft_store(qx_ctx *ctx);
/* tddft_fssh_cal_matrix (tddft_fssh.f90:1344-1414): aij(i, j) = <prev_i|psi_j>
 * with the Gamma metric 2 sum - x(1) y(1), aij column-major nband x nband
 * (element (i, j) at aij[i + j * nband]); tensor cores (3xTF32) in mixed
 * contexts.  The FP64 amplitude propagation and hops stay with the caller. */
int qx_tddft_overlap(qx_ctx *ctx, double *aij);

/* ---- TDDFT-FSSH surface hopping (tddft_fssh_dm, tddft_fssh.f90:1989-2402) -- */
/* Density-matrix representation, one spin channel, no decoherence branch
 * (lfssh_dish = .false.).  The states are the band window b0 .. b0+nstate-1
 * (the reference's noband = noccmx states); each occupied state with a
 * not-full neighbour within nupdn = 3 carries a 7 x 7 complex density
 * matrix, integrated over each MD step in FP64 by RK4 in int(dtmd/dttddft)
 * substeps with the couplings d(k, j) = -(A(k, j) - A(j, k)) / (2 dtmd) of the
 * overlap A(k, j) = <psi_k(t)|psi_j(t+dt)> (tddft_fssh.f90:2098); then the hop
 * probabilities and one Park-Miller draw (rnd00, funcs.f90:1673-1689) decide
 * at most one transition (tddft_fssh.f90:2219-2366).  Times in Rydberg units
 * (1 fs = 20.67), energies in Ry. */
#define QX_FSSH_MAX_STATES 1024
typedef struct {
  int b0, nstate;      /* first band of the window, number of states        */
  double dtmd;         /* MD step                                           */
  double dttddft;      /* electronic substep (reference default 0.02)       */
  int boltzmann;       /* lfssh_boltzmn: exp(-(e_news - e_s)/treq) on hops one state up */
  double treq;         /* temperature (Ry) of that factor                   */
  int hop;             /* lfssh_switch: accept transitions                  */
  double seed;         /* rseed_fssh: state of rnd00 (0 < seed < 2147483647) */
} qx_fssh_parm;
/* Starts the surface hopping: density matrices set to the pure state,
 * accumulated probabilities cleared, occupations occ(nstate) of the window,
 * and the current psi kept as the previous step's wavefunctions. */
int qx_fssh_init(qx_ctx *ctx, const qx_fssh_parm *p, const double *occ);
/* One MD step.  phis (nullable): the overlap A as nstate x nstate column-major
 * host array (a caller that reorders crossing states, as
 * tddft_fssh_set_matrix2 does, passes its own); null: the overlap of the kept
 * previous psi with the current psi on the device (tensor cores in mixed
 * contexts), after which the current psi is kept for the next step.  eig
 * (nullable): the window's eigenvalues, else the context's current ones.
 * Outputs (nullable): occ(nstate) after the step, *transition = s * nstate +
 * news of an accepted hop or -1, bkl(7, nstate): the hop probability of
 * state s to s + iud at bkl[s * 7 + iud + 3]. */
int qx_fssh_step(qx_ctx *ctx, const double *phis, const double *eig, double *occ, int *transition, double *bkl);
/* Reads the state: dnr, dni (7, 7, nstate) with rho(j, k) of state s at
 * [(s * 7 + j + 3) * 7 + k + 3]; accum(nstate, nstate) with the accumulated
 * probability of s -> news at [news + s * nstate]; *rndx the rnd00 state.
 * Any pointer may be null. */
int qx_fssh_state(qx_ctx *ctx, double *dnr, double *dni, double *accum, double *rndx);

/* ---- Hellmann-Feynman forces (force.f90:5-860 terms floc and fnlc) ------ */
/* Geometry tables, set once per geometry after the KB tables (qx_set_kb_g)
 * and qx_scf_init:
 *   natom, ntype, ityp(natom): 0-based species of each atom;
 *   satm(3, natom): fractional coordinates (the phases cos, sin of 2 pi k s
 *     are built on the device by the recurrence of stscfn, bulk.f90:2086-2175);
 *   n5: G vectors of the density half sphere, G = 0 first; ijk5(n5): 0-based
 *     grid index of +G; ngabc(3, n5): integer coordinates (nga, ngb, ngc);
 *   gvec5(3, n5): cartesian G (gx, gy, gz);
 *   svco(n5, ntype): local form factor of each species (Ry; flocal_g);
 *   gw(3, nplw + 1): cartesian G of the wavefunction half sphere.
 * KB projector j of atom a is j = l + lmx * a with lmx = nproj / natom. */
int qx_set_force_tables(qx_ctx *ctx, int natom, int ntype, const int *ityp, const double *satm, int n5,
                        const int *ijk5, const int *ngabc, const double *gvec5, const double *svco,
                        const double *gw);
/* The local pseudopotential of the current geometry on the device, in place
 * of the one given to qx_scf_init (vlocal_g, nlkbpp.f90:862-1036):
 * v(r) = sum_G V(G) e^{iG.r} over the density sphere,
 * V(G) = (1/Omega) sum_a svco(G, ityp_a) e^{-iG.R_a}, from the form factors and
 * phases of qx_set_force_tables (a later qx_build_kb_g moves the phases to its
 * geometry).  Together with qx_build_kb_g this moves every geometry table of
 * an SCF iteration without a host upload, for MD steps. */
int qx_build_vloc(qx_ctx *ctx);
/* Forces (Ry/bohr, (3, natom) each) of the current psi and its density
 * rho = sum occ/Omega |psi|^2:
 *   floc: local pseudopotential in G space (flocal_g, nlkbpp.f90:1037-1120),
 *     2 sum_{G != 0} G svco(G) (Re rho(G) sin G.R + Im rho(G) cos G.R);
 *   fnl: G-space KB (kbnlpp_frc2, nlkbpp.f90:1878-2130),
 *     4 sum_n occ_n sum_l vclalp_l <beta|psi_n> sum_{G != 0} G (beta_re psi_im - beta_im psi_re).
 * The ion-ion (Ewald) term is geometry only and stays with the caller. */
int qx_forces(qx_ctx *ctx, double *floc, double *fnl);
/* Real-space KB forces (Ry/bohr, (3, natom)) of the current psi (fnnlcl2,
 * nlkbppr.f90:2024-3120): F_a = 2 sum_n occ_n / Omega sum_l clalp_l P_l D_l,
 * P_l = rdelv sum_points vnl_l psi_n, D_l = rdelv sum_points grad vnl_l psi_n,
 * psi_n(r) from the inverse FFT passes; needs the tables of qx_build_kb_r
 * with the gradient table (dtabnl) given to qx_set_kb_r_builder. */
int qx_forces_nl_r(qx_ctx *ctx, double *fnl);

/* ---- drop-in shims with the reference's host-array arguments ----------- */
/* kbnlpp_frc2 (nlkbpp.f90:1878): fnlc(3, natom) += the G-space KB forces of
 * cgjr(nplwex, nband) with the occupations of qx_set_occ. */
int qxgpu_kbnlpp_frc2(qx_ctx *ctx, const double *cgjr, double *fnlc);
/* fnnlcl2 (nlkbppr.f90:2024): fnlc(3, natom) += the real-space KB forces of
 * cgjr(nplwex, nband) (tables of qx_build_kb_r with gradients). */
int qxgpu_fnnlcl2(qx_ctx *ctx, const double *cgjr, double *fnlc);
/* hcnonloc: rhcr(nplwex, nb) += local (+ real-space KB) H products of cgjr. */
int qxgpu_hcnonloc(qx_ctx *ctx, const double *cgjr, double *rhcr, int nb);
/* hckbpp_g (nlkbpp.f90:1284-1393): rhcr += G-space KB products of cgjr. */
int qxgpu_hckbpp_g(qx_ctx *ctx, const double *cgjr, double *rhcr, int nb);
/* ekinetic + enonloc: rhcr = H cgjr for all nband bands; ekib(nband). */
int qxgpu_enonloc(qx_ctx *ctx, const double *cgjr, double *rhcr, double *ekib);
/* eigen (eigen.f90:52): gdcr, rhcr updated in place; eig out. */
int qxgpu_eigen(qx_ctx *ctx, double *gdcr, double *rhcr, const double *ekib, double *eig, const qx_cgparm *p);
/* schmidt (schmidt.f90:71): cgjr orthonormalised in place. */
int qxgpu_schmidt(qx_ctx *ctx, double *cgjr);
/* hmatrix (engrad.f90:804): dmtrxr(nband, nband) and eig from cgjr, rhcr. */
int qxgpu_hmatrix(qx_ctx *ctx, const double *cgjr, const double *rhcr, double *dmtrxr, double *eig);
/* untryt + untryhc (eigen.f90:1118, 1336) after qxgpu_hmatrix: gdcr, rhcr rotated in place. */
int qxgpu_untryt(qx_ctx *ctx, double *gdcr, double *rhcr, double *ev);
/* softchg: glocal(kfft0) = sum occ/rvol |psi(r)|^2 of cgjr. */
int qxgpu_softchg(qx_ctx *ctx, const double *cgjr, double *rho);
/* rfft3 (fft3.f90:113-232) on the full grid: key = 1 forward real -> complex
 * scaled 1/kfft0 (fft3x = Re, fft3y = Im on the full grid), key = 2 backward
 * complex -> real (fft3x out, fft3y zeroed). */
int qxgpu_rfft3(qx_ctx *ctx, int key, double *fft3x, double *fft3y);

#ifdef __cplusplus
}
#endif
#endif
