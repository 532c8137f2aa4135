// C ABI of the hot path: context, plan construction and the entry points that
// mirror the reference subroutines (see include/qxmd_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <string>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/qxmd_b200.h"
#include "qx_cg.h"
#include "qx_internal.h"
#include "qx_scf.h"

#include <atomic>

namespace qx {
static std::atomic<long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
static thread_local char g_err[512] = "";
void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
}  // namespace qx

using namespace qx;

#define CK(x)                                                                          \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) {                                                           \
      set_error("%s:%d %s: %s", __FILE__, __LINE__, #x, cudaGetErrorString(e_));       \
      return QX_ERR_CUDA;                                                              \
    }                                                                                  \
  } while (0)

#define CKL()                                                                          \
  do {                                                                                 \
    cudaError_t e_ = cudaGetLastError();                                               \
    if (e_ != cudaSuccess) {                                                           \
      set_error("%s:%d launch: %s", __FILE__, __LINE__, cudaGetErrorString(e_));       \
      return QX_ERR_CUDA;                                                              \
    }                                                                                  \
  } while (0)

#define TRY(x)                   \
  do {                           \
    int r_ = (x);                \
    if (r_) return r_;           \
  } while (0)

struct qx_ctx {
  int prec = 0;
  cudaStream_t st = 0;
  Plan pl;
  int nb = 0, ne = 0, npair_all = 0;
  int nlmode = 0;
  double rvol = 0.0;
  bool have_occ = false, have_glocal = false, have_hsub = false, have_u = false, have_kbg = false, have_kbr = false;
  // FP64 small arrays
  double *d_dk = nullptr, *d_occ = nullptr, *d_wocc = nullptr, *d_eig = nullptr, *d_ekib = nullptr, *d_w = nullptr;
  double *d_hsub = nullptr, *d_mat = nullptr, *d_V = nullptr;   // nb*nb, nb*nb, 2*nb*nb
  double *d_prod = nullptr;
  double *d_eigws = nullptr;   // eigensolver work, 8*nb*nb + 1024*nb
  int *d_info = nullptr;
  int *d_allpairs = nullptr;
  // state arrays in the context precision
  void *psi = nullptr, *hpsi = nullptr, *g = nullptr, *h = nullptr, *gh = nullptr, *snap = nullptr, *tmp = nullptr;
  void *mat_t = nullptr;   // nb*nb in T
  void *proj = nullptr;    // nproj*nb in T
  void *gws = nullptr;     // split-K GEMM workspace
  size_t gws_bytes = 0;
  // FP32 contractions whose band arrays have a row stride (nplwex) that is not
  // a multiple of four floats: room to restage operands for the tensor maps
  void *tcpad = nullptr;
  size_t tcpad_bytes = 0;
  // FP32 KB projector table rows at stride nplwex rounded up to four floats
  // (made once in qx_set_kb_g when nplwex % 4 != 0, so that the <beta|psi>
  // contractions restage only the band operand)
  float *kbgp = nullptr;
  long kbgp_ld = 0;
  CgState cg;
  // density side
  double *d_rho_in = nullptr, *d_rho_out = nullptr, *d_vloc = nullptr, *d_glocal = nullptr, *d_g2 = nullptr;
  double2 *d_zg = nullptr;
  double *d_part = nullptr, *d_sc = nullptr;
  double eion = 0.0, mixbeta = 0.3, q02 = 1.0;
  // Pulay mixing (itratn > 1) or Kerker-filtered linear mixing
  int itratn = 0;
  double cmetric = 20.0, g2min = 0.0, g2max = 0.0;
  bool pulay_reset = true;
  PulayDev *d_pulay = nullptr;
  double2 *d_pu = nullptr, *d_pd = nullptr;
  double *d_ppart = nullptr, *d_adot = nullptr;
  bool scf_ready = false;
  // sequential CG: device band cursor, dot-product buffer and the captured
  // while-loop graph (rebuilt when its buffers or parameters change)
  int *d_seqi = nullptr;   // cur, pairs[2], list[1]
  double *d_seqw = nullptr;
  int seqw_len = 0;
  cudaStream_t cap_st = nullptr;
  // second stream of H|psi>: the G-space KB contractions run there beside the
  // FFT pipeline (fork / join events; captured as parallel graph branches)
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // host I/O of qx_scf_iteration_host: psi and rho are read back on io_st as
  // soon as the iteration has made them final (events recorded inside it,
  // captured as event-record nodes of the iteration graph)
  cudaStream_t io_st = nullptr;
  cudaEvent_t ev_psi_final = nullptr, ev_rho_final = nullptr;
  cudaEvent_t ev_psi_in = nullptr;   // psi uploaded on io_st; the iteration waits for it before H|psi>
  // set by the first qx_scf_iteration_host: only then do the iteration's
  // graphs carry the event nodes (they slow the replay of many small graphs)
  bool host_io = false;
  double *d_io = nullptr;
  long io_len = 0;
  cudaGraph_t seq_graph = nullptr;
  cudaGraphExec_t seq_exec = nullptr;
  std::vector<char> seq_key;
  long seq_body_launches = 0;
  double *d_stage = nullptr;   // host-transfer staging (mixed precision)
  long stage_len = 0;
  // SCF iteration without host round trips: results go to device slots
  // (d_sc[5..6] gradres max/sum, d_info[0] eigen clusters, d_info[1] Cholesky
  // status, d_info[2] CG band applications) read once at the end, and the
  // whole iteration is captured as a graph per buffer arrangement
  // Hellmann-Feynman force tables (qx_set_force_tables)
  int f_natom = 0, f_ntype = 0, f_n5 = 0, f_km[3] = {0, 0, 0}, f_ktot = 0, f_nproj = 0;
  int *d_ityp = nullptr, *d_ijk5 = nullptr, *d_ngabc = nullptr;
  double *d_satm = nullptr, *d_gvec5 = nullptr, *d_svco = nullptr, *d_gw = nullptr, *d_dcq = nullptr,
         *d_dsq = nullptr, *d_force = nullptr;
  void *prev = nullptr;    // wavefunctions of the previous MD step (gdcr_rec), context precision
  bool have_prev = false;
  // TDDFT-FSSH state of the band window (qx_fssh.cu)
  qx_fssh_parm fs{};
  bool have_fssh = false;
  int fs_cap = 0;
  double *d_fs_dnr = nullptr, *d_fs_dni = nullptr, *d_fs_pint = nullptr, *d_fs_bkl = nullptr,
         *d_fs_accum = nullptr, *d_fs_occ = nullptr, *d_fs_occ0 = nullptr, *d_fs_rndx = nullptr,
         *d_fs_A = nullptr, *d_fs_eig = nullptr;
  int *d_fs_trans = nullptr;
  void *dtab = nullptr;    // 3 nproj x nplwex derivative tables (context precision)
  void *dproj = nullptr;   // 3 nproj x nb
  bool have_ftab = false;
  // G-space KB table builder (qx_set_kb_builder, qx_build_kb_g)
  int kb_ntype = 0, kb_lmx = 0, kb_km[3] = {0, 0, 0}, kb_ktot = 0, kb_natom_cap = 0;
  double *d_kb_zzz = nullptr, *d_kb_vclt = nullptr, *d_kb_dcq = nullptr, *d_kb_dsq = nullptr, *d_kb_satm = nullptr;
  int *d_kb_even = nullptr, *d_kb_ngabc = nullptr, *d_kb_ityp = nullptr;
  bool have_kb_builder = false;
  // real-space table builder (qx_set_kb_r_builder, qx_build_kb_r)
  KbrGeom kbr_geom = {};
  int kbr_ntype = 0, kbr_mxnl = 0, kbr_natom = 0, kbr_lmx = 4;
  long kbr_cap = 0;
  double *d_kbr_dl = nullptr, *d_kbr_rcut = nullptr, *d_kbr_tab = nullptr, *d_kbr_satm = nullptr;
  int *d_kbr_poly = nullptr, *d_kbr_ityp = nullptr, *d_kbr_cnt = nullptr, *d_kbr_off = nullptr,
      *d_kbr_mesh = nullptr, *d_kbr_ptatom = nullptr, *d_kbr_lcnt = nullptr, *d_kbr_loff = nullptr,
      *d_kbr_cursor = nullptr;
  int4 *d_kbr_lent = nullptr;
  void *d_kbr_vnl = nullptr, *d_kbr_sumr = nullptr, *d_kbr_bufR = nullptr;
  double *d_kbr_rcl = nullptr;    // radius of each projector's channel (lmx * ntype)
  std::vector<double> kbr_rcut_h; // species radii (the largest channel's)
  double *d_kbr_dtab = nullptr;   // g'(r)/r tables (optional)
  void *d_kbr_dvnl = nullptr;     // projector gradients per point (with d_kbr_dtab)
  long kbr_dvnl_cap = 0;
  double *d_kbr_fpart = nullptr, *d_kbr_fout = nullptr;
  long kbr_fpart_n = 0;
  bool have_kbr_builder = false;
  bool defer = false;
  struct ScfGraph {
    std::vector<char> key;
    cudaGraphExec_t exec = nullptr;
    void *psi = nullptr, *hpsi = nullptr, *tmp = nullptr;   // pointer arrangement after the iteration
    long launches = 0;
    long fallbacks = 0;   // FP32 contractions on the CUDA-core GEMM per replay
  };
  std::vector<ScfGraph> scf_graphs;
  std::vector<void *> allocs;
  size_t tsize() const { return prec == QX_PREC_FP64 ? sizeof(double) : sizeof(float); }
};

static int dalloc(qx_ctx *c, void **p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  CK(cudaMalloc(p, bytes));
  c->allocs.push_back(*p);
  return 0;
}
template <typename P>
static int dalloc(qx_ctx *c, P **p, size_t bytes) {
  void *v = nullptr;
  TRY(dalloc(c, &v, bytes));
  *p = (P *)v;
  return 0;
}

// Captured SCF-iteration graphs hold the table pointers of their capture:
// every call that replaces a table buffer drops them (the next iteration
// captures again).
static void drop_scf_graphs(qx_ctx *c) {
  for (auto &g : c->scf_graphs) cudaGraphExecDestroy(g.exec);
  c->scf_graphs.clear();
}

// Frees a context buffer that a new one replaces (a table that grew, a
// projector or atom count that changed), so that memory does not pile up over
// an MD run: waits for the context's streams (kernels in flight may still
// read it), drops every captured graph (they hold its address) and takes it
// off the context's list.  p may be null.
static int dfree(qx_ctx *c, void *p) {
  if (!p) return 0;
  CK(cudaStreamSynchronize(c->st));
  if (c->st2) CK(cudaStreamSynchronize(c->st2));
  drop_scf_graphs(c);
  if (c->seq_exec) { cudaGraphExecDestroy(c->seq_exec); c->seq_exec = nullptr; }
  if (c->seq_graph) { cudaGraphDestroy(c->seq_graph); c->seq_graph = nullptr; }
  auto it = std::find(c->allocs.begin(), c->allocs.end(), p);
  if (it != c->allocs.end()) c->allocs.erase(it);
  CK(cudaFree(p));
  return 0;
}
// dfree(*p), then a new buffer of `bytes` into *p.
template <typename P>
static int dregrow(qx_ctx *c, P **p, size_t bytes) {
  TRY(dfree(c, (void *)*p));
  *p = nullptr;
  return dalloc(c, p, bytes);
}

extern "C" const char *qx_last_error(void) { return g_err; }
extern "C" int qx_version(void) { return 1; }
extern "C" long qx_launch_count(void) { return g_launches.load(); }

// ---------------------------------------------------------------------------
// The stage plan of a length from an explicit radix sequence (product n,
// each 2..9, at most 8 stages) and the layout of its stage tables.
static bool plan_len(int n, const int *radix, int nstage, FftLen &L) {
  if (nstage < 0 || nstage > 8) return false;
  long prod = 1;
  for (int s = 0; s < nstage; ++s) {
    if (radix[s] < 2 || radix[s] > 9) return false;
    prod *= radix[s];
  }
  if (prod != n) return false;
  L.n = n;
  L.nstage = nstage;
  for (int s = 0; s < nstage; ++s) L.radix[s] = radix[s];
  int ns = 1, st = 0, ob = 0;
  for (int s = 0; s < L.nstage; ++s) {
    const int R = L.radix[s], nr = n / R;
    L.st_off[s] = st;
    L.ob_off[s] = ob;
    st += nr * (R - 1);
    ob += nr;
    ns *= R;
  }
  L.nst = st;
  L.nob = ob;
  return true;
}

static bool factor_len(int n, FftLen &L) {
  int m = n, nst = 0, radix[8];
  // largest radices first: fewer passes through shared memory (the default
  // plan; qx_autotune may pick another)
  const int rad[8] = {9, 8, 7, 6, 5, 4, 3, 2};
  while (m > 1) {
    int r = 0;
    for (int c : rad)
      if (m % c == 0) { r = c; break; }
    if (!r || nst >= 8) return false;
    radix[nst++] = r;
    m /= r;
  }
  return plan_len(n, radix, nst, L);
}

// Every ordered factorisation of n into radices 2..9 with at most maxst
// stages (the autotuner's candidate plans).
static void radix_plans(int n, int maxst, std::vector<std::vector<int>> &out, std::vector<int> &cur) {
  if (n == 1) {
    if (!cur.empty()) out.push_back(cur);
    return;
  }
  if ((int)cur.size() >= maxst) return;
  for (int r = 9; r >= 2; --r)
    if (n % r == 0) {
      cur.push_back(r);
      radix_plans(n / r, maxst, out, cur);
      cur.pop_back();
    }
}

// Stage output bases (precision independent) of the three lengths.
static void stage_bases(const FftLen &L, std::vector<int> &out) {
  int ns = 1;
  for (int s = 0; s < L.nstage; ++s) {
    const int R = L.radix[s], nr = L.n / R;
    for (int j = 0; j < nr; ++j) out.push_back((j / ns) * ns * R + j % ns);
    ns *= R;
  }
}

template <typename T>
static int upload_tw(qx_ctx *c) {
  typedef typename c2t<T>::type C;
  Plan &pl = c->pl;
  const double tp = 2.0 * std::acos(-1.0);
  std::vector<C> base, stg;
  for (int d = 0; d < 3; ++d) {
    const FftLen &L = pl.L[d];
    const int n = L.n;
    for (int t = 0; t < n; ++t) {
      C w;
      w.x = (T)std::cos(tp * t / n);
      w.y = (T)-std::sin(tp * t / n);
      base.push_back(w);
    }
    int ns = 1;
    for (int s = 0; s < L.nstage; ++s) {
      const int R = L.radix[s], nr = n / R, tstep = n / (ns * R);
      for (int j = 0; j < nr; ++j) {
        const int k = j % ns;
        for (int r = 1; r < R; ++r) {
          const long idx = ((long)k * r * tstep) % n;
          C w;
          w.x = (T)std::cos(tp * idx / n);
          w.y = (T)-std::sin(tp * idx / n);
          stg.push_back(w);
        }
      }
      ns *= R;
    }
  }
  C *dp = nullptr, *ds = nullptr;
  // a new plan replaces the tables of the old one
  TRY(dfree(c, pl.bufs<T>().tw));
  TRY(dfree(c, pl.bufs<T>().stw));
  pl.bufs<T>().tw = nullptr;
  pl.bufs<T>().stw = nullptr;
  TRY(dalloc(c, &dp, sizeof(C) * base.size()));
  TRY(dalloc(c, &ds, sizeof(C) * std::max<size_t>(stg.size(), 1)));
  CK(cudaMemcpy(dp, base.data(), sizeof(C) * base.size(), cudaMemcpyHostToDevice));
  if (!stg.empty()) CK(cudaMemcpy(ds, stg.data(), sizeof(C) * stg.size(), cudaMemcpyHostToDevice));
  pl.bufs<T>().tw = dp;
  pl.bufs<T>().stw = ds;
  return 0;
}

template <typename T>
static int alloc_pipe(qx_ctx *c) {
  typedef typename c2t<T>::type C;
  Plan &pl = c->pl;
  Bufs<T> &b = pl.bufs<T>();
  const long per_pair = (long)pl.k3 * pl.P2 * pl.P1 + (long)pl.k3 * pl.k2 * pl.P1 + (long)(pl.nplw + 1) * 2;
  // band pairs per pipeline launch: a chunk's z-transformed planes stay in
  // L2 between the passes (Si64 FP32: 80 pairs, 25 MB of bufA, one chunk)
  const char *env = getenv("QX_CHUNK_MB");
  const double mb = env ? atof(env) : 160.0;
  long ch = (long)(mb * 1048576.0 / (sizeof(C) * (double)per_pair));
  ch = std::max(1L, std::min(ch, (long)c->npair_all));
  pl.chunk = (int)ch;
  TRY(dalloc(c, &b.bufA, sizeof(C) * ch * pl.k3 * pl.P2 * pl.P1));
  TRY(dalloc(c, &b.bufB, sizeof(C) * ch * pl.k3 * pl.k2 * pl.P1));
  TRY(dalloc(c, &b.zsph, sizeof(C) * ch * (pl.nplw + 1) * 2));
  TRY(dalloc(c, &b.vloc, sizeof(T) * pl.n));
  CK(cudaMemset(b.vloc, 0, sizeof(T) * pl.n));
  if (sizeof(T) == sizeof(float) && plane_length_supported(pl.k1, pl.k2))
    TRY(dalloc(c, &b.rho_part, sizeof(double) * RHO_GROUPS * pl.n));
  TRY(upload_tw<T>(c));
  // shared-memory opt-in for the largest launch of this plan
  const size_t need = fft_smem_need<T>(pl);
  if (need > 227 * 1024) {
    set_error("FFT tile needs %zu bytes of shared memory (> 227 KB)", need);
    return QX_ERR_ARG;
  }
  set_fft_smem_limits<T>(need);
  CKL();
  return 0;
}

// Restaging room for the tensor-core contractions when nplwex is not a
// multiple of four (rows of band arrays then break the 16-byte stride rule
// of the tensor maps): `rows` rows of nplwex rounded up to four floats.
static int tcpad_reserve(qx_ctx *c, long rows) {
  if (c->prec != QX_PREC_MIXED || (c->ne & 3) == 0) return 0;
  const size_t need = sizeof(float) * (size_t)rows * (size_t)((c->ne + 3) & ~3L);
  if (need <= c->tcpad_bytes) return 0;
  void *p = nullptr;
  TRY(dalloc(c, &p, need));
  c->tcpad = p;
  c->tcpad_bytes = need;
  return 0;
}

extern "C" int qx_create(qx_ctx **out, int precision, int k1, int k2, int k3, int nplw, const int *ijkgd,
                         const double *dkgnrm, int nband, void *stream) {
  if (!out || !ijkgd || !dkgnrm || k1 <= 0 || k2 <= 0 || k3 <= 0 || nplw < 0 || nband <= 0 ||
      (precision != QX_PREC_FP64 && precision != QX_PREC_MIXED)) {
    set_error("qx_create: bad arguments");
    return QX_ERR_ARG;
  }
  qx_ctx *c = new qx_ctx();
  *out = nullptr;
  c->prec = precision;
  c->st = (cudaStream_t)stream;
  c->nb = nband;
  c->ne = 2 * (nplw + 1);
  c->npair_all = (nband + 1) / 2;
  Plan &pl = c->pl;
  pl.k1 = k1; pl.k2 = k2; pl.k3 = k3;
  pl.n = (long)k1 * k2 * k3;
  pl.nplw = nplw;
  pl.nplwex = c->ne;
  if (!factor_len(k1, pl.L[0]) || !factor_len(k2, pl.L[1]) || !factor_len(k3, pl.L[2])) {
    set_error("qx_create: FFT sizes must be products of 2,3,5,7 (got %d %d %d)", k1, k2, k3);
    delete c;
    return QX_ERR_ARG;
  }
  if (init_fft_roots()) {
    set_error("qx_create: cannot write FFT roots to the device: %s", cudaGetErrorString(cudaGetLastError()));
    delete c;
    return QX_ERR_CUDA;
  }
  // QX_FFT_PLAN = "r1xr2x...": that radix sequence for every axis whose
  // length it multiplies to (tests pin the stage kernels on chosen plans)
  if (const char *fp = getenv("QX_FFT_PLAN")) {
    int rad[8], nr = 0;
    for (const char *q = fp; *q && nr < 8;) {
      rad[nr++] = atoi(q);
      while (*q && *q != 'x') ++q;
      if (*q == 'x') ++q;
    }
    for (int d = 0; d < 3; ++d) {
      FftLen L;
      if (plan_len(pl.L[d].n, rad, nr, L)) pl.L[d] = L;
    }
  }
  pl.tw_off[0] = 0; pl.tw_off[1] = k1; pl.tw_off[2] = k1 + k2;
  pl.stw_off[0] = 0; pl.stw_off[1] = pl.L[0].nst; pl.stw_off[2] = pl.L[0].nst + pl.L[1].nst;
  pl.sob_off[0] = 0; pl.sob_off[1] = pl.L[0].nob; pl.sob_off[2] = pl.L[0].nob + pl.L[1].nob;
  // sphere geometry from ijkgd
  std::vector<int> n1(nplw + 1), n2(nplw + 1), i3v(nplw + 1);
  int m1 = 0, m2 = 0, m3 = 0;
  for (int ig = 0; ig <= nplw; ++ig) {
    const long ijk = ijkgd[nplw + ig];
    if (ijk < 0 || ijk >= pl.n) { set_error("qx_create: ijkgd out of range"); delete c; return QX_ERR_ARG; }
    const int a = (int)(ijk % k1), b = (int)((ijk / k1) % k2), d = (int)(ijk / ((long)k1 * k2));
    n1[ig] = a <= k1 / 2 ? a : a - k1;
    n2[ig] = b <= k2 / 2 ? b : b - k2;
    const int n3 = d <= k3 / 2 ? d : d - k3;
    i3v[ig] = d;
    m1 = std::max(m1, std::abs(n1[ig]));
    m2 = std::max(m2, std::abs(n2[ig]));
    m3 = std::max(m3, std::abs(n3));
    // -G must sit at the mirrored index
    const long ijm = ijkgd[nplw - ig];
    const int am = (int)(ijm % k1), bm = (int)((ijm / k1) % k2), dm = (int)(ijm / ((long)k1 * k2));
    if (am != (k1 - a) % k1 || bm != (k2 - b) % k2 || dm != (k3 - d) % k3) {
      set_error("qx_create: ijkgd(-G) is not the mirror of ijkgd(G) at G index %d", ig);
      delete c;
      return QX_ERR_ARG;
    }
  }
  if (2 * m1 + 1 > k1 || 2 * m2 + 1 > k2 || 2 * m3 + 1 > k3) {
    set_error("qx_create: wavefunction sphere does not fit the grid");
    delete c;
    return QX_ERR_ARG;
  }
  pl.m1 = m1; pl.m2 = m2; pl.m3 = m3;
  pl.P1 = 2 * m1 + 1; pl.P2 = 2 * m2 + 1;
  // row CSR of the +G and -G positions
  struct Ent { int j2, a, i3, ig, sgn; };
  std::vector<Ent> ents;
  ents.reserve(2 * nplw + 1);
  for (int ig = 0; ig <= nplw; ++ig) {
    ents.push_back({n2[ig] + m2, n1[ig] + m1, i3v[ig], ig, +1});
    if (ig) ents.push_back({-n2[ig] + m2, -n1[ig] + m1, (k3 - i3v[ig]) % k3, ig, -1});
  }
  std::vector<int> lo(pl.P2, 1 << 30), hi(pl.P2, -1), cnt(pl.P2 + 1, 0);
  for (auto &e : ents) {
    lo[e.j2] = std::min(lo[e.j2], e.a);
    hi[e.j2] = std::max(hi[e.j2], e.a);
    cnt[e.j2 + 1]++;
  }
  for (int j = 0; j < pl.P2; ++j) {
    if (hi[j] < 0) { lo[j] = 1; hi[j] = 0; }
    cnt[j + 1] += cnt[j];
  }
  std::vector<int4> rent(ents.size());
  std::vector<int> fill(cnt.begin(), cnt.end() - 1);
  for (auto &e : ents) rent[fill[e.j2]++] = make_int4(e.a - lo[e.j2], e.i3, e.ig, e.sgn);
  // z-columns: every (j2, a) with lo <= a <= hi, row by row
  std::vector<int> col_ja, colq((size_t)pl.P2 * pl.P1, -1);
  for (int j = 0; j < pl.P2; ++j)
    for (int a = lo[j]; a <= hi[j]; ++a) {
      colq[(size_t)j * pl.P1 + a] = (int)col_ja.size();
      col_ja.push_back(j * pl.P1 + a);
    }
  pl.ncol = (int)col_ja.size();
  std::vector<int> col_ig((size_t)k3 * std::max(1, pl.ncol), 0);
  for (auto &e : ents) col_ig[(size_t)e.i3 * pl.ncol + colq[(size_t)e.j2 * pl.P1 + e.a]] = e.sgn > 0 ? e.ig + 1 : -(e.ig + 1);
  int rc = 0;
#define FAIL(x) do { rc = (x); if (rc) { qx_destroy(c); return rc; } } while (0)
  FAIL(dalloc(c, &pl.d_row_lo, sizeof(int) * pl.P2));
  FAIL(dalloc(c, &pl.d_row_hi, sizeof(int) * pl.P2));
  FAIL(dalloc(c, &pl.d_row_off, sizeof(int) * (pl.P2 + 1)));
  FAIL(dalloc(c, &pl.d_row_ent, sizeof(int4) * rent.size()));
  FAIL(dalloc(c, &pl.d_col_ja, sizeof(int) * std::max<size_t>(1, col_ja.size())));
  FAIL(dalloc(c, &pl.d_col_ig, sizeof(int) * col_ig.size()));
  if (cudaMemcpy(pl.d_row_lo, lo.data(), sizeof(int) * pl.P2, cudaMemcpyHostToDevice) ||
      cudaMemcpy(pl.d_row_hi, hi.data(), sizeof(int) * pl.P2, cudaMemcpyHostToDevice) ||
      cudaMemcpy(pl.d_row_off, cnt.data(), sizeof(int) * (pl.P2 + 1), cudaMemcpyHostToDevice) ||
      cudaMemcpy(pl.d_row_ent, rent.data(), sizeof(int4) * rent.size(), cudaMemcpyHostToDevice) ||
      (pl.ncol && cudaMemcpy(pl.d_col_ja, col_ja.data(), sizeof(int) * col_ja.size(), cudaMemcpyHostToDevice)) ||
      cudaMemcpy(pl.d_col_ig, col_ig.data(), sizeof(int) * col_ig.size(), cudaMemcpyHostToDevice)) {
    set_error("qx_create: upload failed: %s", cudaGetErrorString(cudaGetLastError()));
    qx_destroy(c);
    return QX_ERR_CUDA;
  }
  {
    std::vector<int> sob;
    for (int d = 0; d < 3; ++d) stage_bases(pl.L[d], sob);
    FAIL(dalloc(c, &pl.d_sob, sizeof(int) * std::max<size_t>(sob.size(), 1)));
    if (!sob.empty() && cudaMemcpy(pl.d_sob, sob.data(), sizeof(int) * sob.size(), cudaMemcpyHostToDevice)) {
      qx_destroy(c);
      return QX_ERR_CUDA;
    }
  }
  // small FP64 arrays
  const int nb = nband, ne = c->ne;
  FAIL(dalloc(c, &c->d_dk, sizeof(double) * ne));
  if (cudaMemcpy(c->d_dk, dkgnrm, sizeof(double) * ne, cudaMemcpyHostToDevice)) { qx_destroy(c); return QX_ERR_CUDA; }
  FAIL(dalloc(c, &c->d_occ, sizeof(double) * nb));
  FAIL(dalloc(c, &c->d_wocc, sizeof(double) * nb));
  FAIL(dalloc(c, &c->d_eig, sizeof(double) * nb));
  FAIL(dalloc(c, &c->d_ekib, sizeof(double) * nb));
  FAIL(dalloc(c, &c->d_w, sizeof(double) * nb));
  FAIL(dalloc(c, &c->d_prod, sizeof(double) * nb));
  FAIL(dalloc(c, &c->d_hsub, sizeof(double) * nb * nb));
  FAIL(dalloc(c, &c->d_mat, sizeof(double) * nb * nb));
  FAIL(dalloc(c, &c->d_V, sizeof(double) * 2 * nb * nb));
  FAIL(dalloc(c, &c->d_eigws, sizeof(double) * (8 * (size_t)nb * nb + 1024 * (size_t)nb)));
  FAIL(dalloc(c, &c->d_info, sizeof(int) * 4));
  std::vector<int> pairs(2 * c->npair_all);
  for (int p = 0; p < c->npair_all; ++p) {
    pairs[2 * p] = 2 * p;
    pairs[2 * p + 1] = (2 * p + 1 < nb) ? 2 * p + 1 : -1;
  }
  FAIL(dalloc(c, &c->d_allpairs, sizeof(int) * pairs.size()));
  cudaMemcpy(c->d_allpairs, pairs.data(), sizeof(int) * pairs.size(), cudaMemcpyHostToDevice);
  // state arrays
  const size_t ts = c->tsize(), blk = ts * (size_t)nb * ne;
  FAIL(dalloc(c, &c->psi, blk));
  FAIL(dalloc(c, &c->hpsi, blk));
  FAIL(dalloc(c, &c->g, blk));
  FAIL(dalloc(c, &c->h, blk));
  FAIL(dalloc(c, &c->gh, blk));
  FAIL(dalloc(c, &c->snap, blk));
  FAIL(dalloc(c, &c->tmp, blk));
  FAIL(dalloc(c, &c->mat_t, ts * nb * nb));
  c->gws_bytes = sizeof(double) * (size_t)64 * 1024 * 1024 / 8;   // 64 MB
  FAIL(dalloc(c, &c->gws, c->gws_bytes));
  // the split-K tile counters, zero before the first GEMM on the context's stream
  if (cudaMemsetAsync(c->gws, 0, GEMM_COUNTER_BYTES, c->st) != cudaSuccess) {
    set_error("qx_create: clearing the GEMM counters failed");
    qx_destroy(c);
    return QX_ERR_CUDA;
  }
  FAIL(tcpad_reserve(c, 2L * nb));
  cudaMemset(c->psi, 0, blk);
  cudaMemset(c->hpsi, 0, blk);
  // CG state
  CgState &s = c->cg;
  double **dd[] = {&s.eig, &s.zansa, &s.zansab, &s.z000re, &s.x000re, &s.eigb, &s.betk, &s.dinnerx, &s.cai};
  for (auto p : dd) FAIL(dalloc(c, p, sizeof(double) * nb));
  s.ekib = c->d_ekib;
  int **ii[] = {&s.iter, &s.izcnt, &s.lreset, &s.active, &s.list};
  for (auto p : ii) FAIL(dalloc(c, p, sizeof(int) * nb));
  FAIL(dalloc(c, &s.pairs, sizeof(int) * 2 * c->npair_all));
  FAIL(dalloc(c, &s.nact, sizeof(int)));
  FAIL(dalloc(c, &s.npair, sizeof(int)));
  // pipeline buffers for the context precision (FP64 density FFTs always)
  if (c->prec == QX_PREC_FP64) {
    FAIL(alloc_pipe<double>(c));
  } else {
    FAIL(alloc_pipe<float>(c));
    TRY(upload_tw<double>(c));
    set_fft_smem_limits<double>(227 * 1024);
  }
  // read-back stream and the events the iteration records for it
  if (cudaStreamCreateWithFlags(&c->io_st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_psi_final, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_rho_final, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_psi_in, cudaEventDisableTiming) != cudaSuccess) {
    set_error("qx_create: stream or event creation failed");
    qx_destroy(c);
    return QX_ERR_CUDA;
  }
  if (cudaGetLastError() != cudaSuccess) { set_error("qx_create: CUDA error during set-up"); qx_destroy(c); return QX_ERR_CUDA; }
#undef FAIL
  *out = c;
  return QX_OK;
}

extern "C" int qx_destroy(qx_ctx *c) {
  if (!c) return QX_OK;
  cudaStreamSynchronize(c->st);
  for (auto &g : c->scf_graphs) cudaGraphExecDestroy(g.exec);
  if (c->seq_exec) cudaGraphExecDestroy(c->seq_exec);
  if (c->seq_graph) cudaGraphDestroy(c->seq_graph);
  if (c->cap_st) cudaStreamDestroy(c->cap_st);
  if (c->st2) cudaStreamSynchronize(c->st2);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->st2) cudaStreamDestroy(c->st2);
  if (c->io_st) cudaStreamDestroy(c->io_st);
  if (c->ev_psi_final) cudaEventDestroy(c->ev_psi_final);
  if (c->ev_rho_final) cudaEventDestroy(c->ev_rho_final);
  if (c->ev_psi_in) cudaEventDestroy(c->ev_psi_in);
  for (void *p : c->allocs) cudaFree(p);
  delete c;
  return QX_OK;
}

// ---------------------------------------------------------------------------
// FP64 staging area of a mixed-precision context for host transfers; grown
// on demand and kept, so repeated transfers allocate nothing.
static int stage(qx_ctx *c, long n, double **out) {
  if (c->stage_len < n) {
    TRY(dregrow(c, &c->d_stage, sizeof(double) * n));
    c->stage_len = n;
  }
  *out = c->d_stage;
  return 0;
}

template <typename T>
static int upload_conv(qx_ctx *c, T *dst, const double *src, long n) {
  if (sizeof(T) == sizeof(double)) {
    CK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
    return 0;
  }
  double *tmp = nullptr;
  TRY(stage(c, n, &tmp));
  CK(cudaMemcpyAsync(tmp, src, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  convert<double, T>(tmp, dst, n, c->st);
  CKL();
  return 0;
}

template <typename T>
static int download_conv(qx_ctx *c, double *dst, const T *src, long n) {
  if (sizeof(T) == sizeof(double)) {
    CK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
  }
  double *tmp = nullptr;
  TRY(stage(c, n, &tmp));
  convert<T, double>(src, tmp, n, c->st);
  CK(cudaMemcpyAsync(dst, tmp, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

static int up(qx_ctx *c, void *dst, const double *src, long n) {
  return c->prec == QX_PREC_FP64 ? upload_conv<double>(c, (double *)dst, src, n)
                                 : upload_conv<float>(c, (float *)dst, src, n);
}
static int down(qx_ctx *c, double *dst, const void *src, long n) {
  return c->prec == QX_PREC_FP64 ? download_conv<double>(c, dst, (const double *)src, n)
                                 : download_conv<float>(c, dst, (const float *)src, n);
}

extern "C" int qx_set_glocal(qx_ctx *c, const double *glocal) {
  if (!c || !glocal) { set_error("qx_set_glocal: null"); return QX_ERR_ARG; }
  if (!c->d_glocal) TRY(dalloc(c, &c->d_glocal, sizeof(double) * c->pl.n));
  CK(cudaMemcpyAsync(c->d_glocal, glocal, sizeof(double) * c->pl.n, cudaMemcpyHostToDevice, c->st));
  if (c->prec == QX_PREC_FP64)
    convert<double, double>(c->d_glocal, c->pl.b64.vloc, c->pl.n, c->st);
  else
    convert<double, float>(c->d_glocal, c->pl.b32.vloc, c->pl.n, c->st);
  CKL();
  c->have_glocal = true;
  return QX_OK;
}

// The KB projector table as a contraction operand: the padded FP32 copy
// where there is one, else the table itself at stride nplwex.
template <typename T>
static const T *kbg_operand(const qx_ctx *c, long *ld) {
  if (sizeof(T) == sizeof(float) && c->kbgp) {
    *ld = c->kbgp_ld;
    return (const T *)c->kbgp;
  }
  *ld = c->ne;
  return c->pl.bufs<T>().kbg;
}

extern "C" int qx_set_kb_g(qx_ctx *c, int nproj, const double *eqlmr, const double *vclalp) {
  if (!c || nproj <= 0 || !eqlmr || !vclalp) { set_error("qx_set_kb_g: bad arguments"); return QX_ERR_ARG; }
  const size_t ts = c->tsize();
  void *kbg = c->prec == QX_PREC_FP64 ? (void *)c->pl.b64.kbg : (void *)c->pl.b32.kbg;
  void *vcl = c->prec == QX_PREC_FP64 ? (void *)c->pl.b64.vclalp : (void *)c->pl.b32.vclalp;
  void *proj = c->proj;
  if (!c->have_kbg || c->pl.nproj != nproj) {
    // a new projector count: new buffers (the old ones freed); the same count
    // (a new geometry) rewrites the tables in place, so captured SCF graphs
    // stay valid
    TRY(dregrow(c, &kbg, ts * (size_t)nproj * c->ne));
    TRY(dregrow(c, &vcl, ts * nproj));
    TRY(dregrow(c, &proj, ts * (size_t)nproj * c->nb));
    TRY(dfree(c, c->kbgp));
    c->kbgp = nullptr;
    c->kbgp_ld = 0;
    c->pl.nproj = nproj;
    drop_scf_graphs(c);
    TRY(tcpad_reserve(c, (long)nproj + c->nb));
    if (c->prec == QX_PREC_FP64) { c->pl.b64.kbg = (double *)kbg; c->pl.b64.vclalp = (double *)vcl; }
    else {
      c->pl.b32.kbg = (float *)kbg;
      c->pl.b32.vclalp = (float *)vcl;
      if (c->ne & 3) {
        c->kbgp_ld = (c->ne + 3) & ~3L;
        TRY(dalloc(c, &c->kbgp, sizeof(float) * (size_t)nproj * c->kbgp_ld));
      }
    }
    c->proj = proj;
  }
  TRY(up(c, kbg, eqlmr, (long)nproj * c->ne));
  TRY(up(c, vcl, vclalp, nproj));
  if (c->kbgp) {
    pad_rows_f32((const float *)kbg, c->ne, c->ne, nproj, c->kbgp, c->kbgp_ld, c->st);
    CKL();
  }
  c->have_kbg = true;
  return QX_OK;
}

extern "C" int qx_set_kb_builder(qx_ctx *c, int ntype, int lmx, int mxqlm, const double *dlqlm, const double *tbqlm,
                                 int nlm, const double *qlm, const int *lmidx, const int *even, const double *vclalp,
                                 const int *ngabc) {
  if (!c || ntype <= 0 || lmx <= 0 || mxqlm < 2 || nlm <= 0 || !dlqlm || !tbqlm || !qlm || !lmidx || !even ||
      !vclalp || !ngabc) {
    set_error("qx_set_kb_builder: bad arguments");
    return QX_ERR_ARG;
  }
  if (lmx > 256) { set_error("qx_set_kb_builder: at most 256 projectors per atom"); return QX_ERR_ARG; }
  const int nplw1 = c->ne / 2, nchan = lmx * ntype;
  for (int i = 0; i < nchan; ++i)
    if (lmidx[i] < 0 || lmidx[i] >= nlm) { set_error("qx_set_kb_builder: lmidx out of range"); return QX_ERR_ARG; }
  // the interpolation reads t_{m+2}: the table must reach the largest |G|
  std::vector<double> dk(c->ne);
  CK(cudaMemcpy(dk.data(), c->d_dk, sizeof(double) * c->ne, cudaMemcpyDeviceToHost));
  double g2max = 0.0;
  for (int g = 0; g < nplw1; ++g) g2max = std::max(g2max, dk[2 * g]);
  for (int it = 0; it < ntype; ++it) {
    if (!(dlqlm[it] > 0.0)) { set_error("qx_set_kb_builder: dlqlm must be positive"); return QX_ERR_ARG; }
    const double ag = std::sqrt(g2max);
    const long m = 2 * (long)(ag / (2.0 * dlqlm[it]));
    if (m + 2 > mxqlm) { set_error("qx_set_kb_builder: radial table too short for the largest |G|"); return QX_ERR_ARG; }
  }
  int km[3] = {0, 0, 0};
  for (long i = 0; i < 3L * nplw1; ++i) km[i % 3] = std::max(km[i % 3], std::abs(ngabc[i]));
  double *d_dl = nullptr, *d_tb = nullptr, *d_qlm = nullptr;
  int *d_lmidx = nullptr;
  TRY(dalloc(c, &d_dl, sizeof(double) * ntype));
  TRY(dalloc(c, &d_tb, sizeof(double) * (size_t)(mxqlm + 1) * nchan));
  TRY(dalloc(c, &d_qlm, sizeof(double) * (size_t)nplw1 * nlm));
  TRY(dalloc(c, &d_lmidx, sizeof(int) * nchan));
  TRY(dalloc(c, &c->d_kb_zzz, sizeof(double) * (size_t)nplw1 * nchan));
  TRY(dalloc(c, &c->d_kb_even, sizeof(int) * nchan));
  TRY(dalloc(c, &c->d_kb_vclt, sizeof(double) * nchan));
  TRY(dalloc(c, &c->d_kb_ngabc, sizeof(int) * 3 * (size_t)nplw1));
  CK(cudaMemcpyAsync(d_dl, dlqlm, sizeof(double) * ntype, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(d_tb, tbqlm, sizeof(double) * (size_t)(mxqlm + 1) * nchan, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(d_qlm, qlm, sizeof(double) * (size_t)nplw1 * nlm, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(d_lmidx, lmidx, sizeof(int) * nchan, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_kb_even, even, sizeof(int) * nchan, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_kb_vclt, vclalp, sizeof(double) * nchan, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_kb_ngabc, ngabc, sizeof(int) * 3 * (size_t)nplw1, cudaMemcpyHostToDevice, c->st));
  setqlm(nplw1, nchan, lmx, mxqlm, d_dl, d_tb, d_qlm, d_lmidx, c->d_dk, c->d_kb_zzz, c->st);
  CKL();
  c->kb_ntype = ntype;
  c->kb_lmx = lmx;
  for (int d = 0; d < 3; ++d) c->kb_km[d] = km[d];
  c->kb_ktot = 2 * (km[0] + km[1] + km[2]) + 3;
  c->kb_natom_cap = 0;
  c->have_kb_builder = true;
  return QX_OK;
}

extern "C" int qx_build_kb_g(qx_ctx *c, int natom, const int *ityp, const double *satm) {
  if (!c || natom <= 0 || natom > 65535 || !ityp || !satm) { set_error("qx_build_kb_g: bad arguments"); return QX_ERR_ARG; }
  if (!c->have_kb_builder) { set_error("qx_build_kb_g: qx_set_kb_builder first"); return QX_ERR_STATE; }
  for (int a = 0; a < natom; ++a)
    if (ityp[a] < 0 || ityp[a] >= c->kb_ntype) { set_error("qx_build_kb_g: ityp out of range"); return QX_ERR_ARG; }
  const int lmx = c->kb_lmx, nproj = lmx * natom, ne = c->ne;
  const size_t ts = c->tsize();
  if (!c->have_kbg || c->pl.nproj != nproj) {
    // first build (or a new projector count): the tables of qx_set_kb_g,
    // replacing (and freeing) any earlier ones
    void *kbg = c->have_kbg ? (c->prec == QX_PREC_FP64 ? (void *)c->pl.b64.kbg : (void *)c->pl.b32.kbg) : nullptr;
    void *vcl = c->have_kbg ? (c->prec == QX_PREC_FP64 ? (void *)c->pl.b64.vclalp : (void *)c->pl.b32.vclalp)
                            : nullptr;
    void *proj = c->have_kbg ? c->proj : nullptr;
    TRY(dregrow(c, &kbg, ts * (size_t)nproj * ne));
    TRY(dregrow(c, &vcl, ts * nproj));
    TRY(dregrow(c, &proj, ts * (size_t)nproj * c->nb));
    TRY(dfree(c, c->kbgp));
    c->pl.nproj = nproj;
    drop_scf_graphs(c);
    TRY(tcpad_reserve(c, (long)nproj + c->nb));
    c->kbgp = nullptr;
    c->kbgp_ld = 0;
    if (c->prec == QX_PREC_FP64) { c->pl.b64.kbg = (double *)kbg; c->pl.b64.vclalp = (double *)vcl; }
    else {
      c->pl.b32.kbg = (float *)kbg;
      c->pl.b32.vclalp = (float *)vcl;
      if (ne & 3) {
        c->kbgp_ld = (ne + 3) & ~3L;
        TRY(dalloc(c, &c->kbgp, sizeof(float) * (size_t)nproj * c->kbgp_ld));
      }
    }
    c->proj = proj;
  }
  if (natom > c->kb_natom_cap) {
    TRY(dregrow(c, &c->d_kb_ityp, sizeof(int) * natom));
    TRY(dregrow(c, &c->d_kb_satm, sizeof(double) * 3 * natom));
    TRY(dregrow(c, &c->d_kb_dcq, sizeof(double) * (size_t)natom * c->kb_ktot));
    TRY(dregrow(c, &c->d_kb_dsq, sizeof(double) * (size_t)natom * c->kb_ktot));
    c->kb_natom_cap = natom;
  }
  CK(cudaMemcpyAsync(c->d_kb_ityp, ityp, sizeof(int) * natom, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_kb_satm, satm, sizeof(double) * 3 * natom, cudaMemcpyHostToDevice, c->st));
  const int *km = c->kb_km;
  phase_tables(natom, c->d_kb_satm, km[0], km[1], km[2], c->kb_ktot, c->d_kb_dcq, c->d_kb_dsq, c->st);
  if (c->prec == QX_PREC_FP64)
    setbgq<double>(natom, ne / 2, ne, lmx, c->d_kb_ityp, c->d_kb_ngabc, c->d_kb_dcq, c->d_kb_dsq, km[0], km[1], km[2],
                   c->kb_ktot, c->d_kb_zzz, c->d_kb_even, c->d_kb_vclt, c->pl.b64.kbg, nullptr, 0,
                   c->pl.b64.vclalp, c->st);
  else
    setbgq<float>(natom, ne / 2, ne, lmx, c->d_kb_ityp, c->d_kb_ngabc, c->d_kb_dcq, c->d_kb_dsq, km[0], km[1], km[2],
                  c->kb_ktot, c->d_kb_zzz, c->d_kb_even, c->d_kb_vclt, c->pl.b32.kbg, c->kbgp, c->kbgp_ld,
                  c->pl.b32.vclalp, c->st);
  CKL();
  c->have_kbg = true;
  // force tables of an earlier qx_set_force_tables follow the new geometry:
  // species, phases and the KB derivative tables (the G-vector arrays and
  // form factors do not depend on it)
  if (c->have_ftab && c->f_natom == natom && c->f_nproj == nproj) {
    CK(cudaMemcpyAsync(c->d_ityp, c->d_kb_ityp, sizeof(int) * natom, cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(c->d_satm, c->d_kb_satm, sizeof(double) * 3 * natom, cudaMemcpyDeviceToDevice, c->st));
    phase_tables(natom, c->d_satm, c->f_km[0], c->f_km[1], c->f_km[2], c->f_ktot, c->d_dcq, c->d_dsq, c->st);
    if (c->prec == QX_PREC_FP64)
      dtab_build<double>(nproj, ne / 2 - 1, c->pl.b64.kbg, c->d_gw, (double *)c->dtab, c->st);
    else
      dtab_build<float>(nproj, ne / 2 - 1, c->pl.b32.kbg, c->d_gw, (float *)c->dtab, c->st);
    CKL();
  }
  return QX_OK;
}

template <typename T>
static int get_kb_g(qx_ctx *c, double *eqlmr, double *vclalp) {
  const Bufs<T> &b = c->pl.bufs<T>();
  const long np = c->pl.nproj, ne = c->ne;
  std::vector<T> h((size_t)np * ne), v((size_t)np);
  CK(cudaStreamSynchronize(c->st));
  CK(cudaMemcpy(h.data(), b.kbg, sizeof(T) * h.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(v.data(), b.vclalp, sizeof(T) * v.size(), cudaMemcpyDeviceToHost));
  if (eqlmr)
    for (size_t i = 0; i < h.size(); ++i) eqlmr[i] = (double)h[i];
  if (vclalp)
    for (size_t i = 0; i < v.size(); ++i) vclalp[i] = (double)v[i];
  if (sizeof(T) == sizeof(float) && c->kbgp && eqlmr) {
    // the padded copy must hold the same rows
    std::vector<float> p((size_t)np * c->kbgp_ld);
    CK(cudaMemcpy(p.data(), c->kbgp, sizeof(float) * p.size(), cudaMemcpyDeviceToHost));
    for (long j = 0; j < np; ++j)
      if (std::memcmp(p.data() + j * c->kbgp_ld, (const float *)(const void *)h.data() + j * ne, sizeof(float) * ne)) {
        set_error("qx_get_kb_g: padded copy of projector %ld differs", j);
        return QX_ERR_STATE;
      }
  }
  return QX_OK;
}

extern "C" int qx_get_kb_g(qx_ctx *c, double *eqlmr, double *vclalp) {
  if (!c) { set_error("qx_get_kb_g: null"); return QX_ERR_ARG; }
  if (!c->have_kbg) { set_error("qx_get_kb_g: G-space tables not set"); return QX_ERR_STATE; }
  return c->prec == QX_PREC_FP64 ? get_kb_g<double>(c, eqlmr, vclalp) : get_kb_g<float>(c, eqlmr, vclalp);
}

extern "C" int qx_set_kb_r(qx_ctx *c, int natom, int lmx, const int *off, const int *mesh, const double *vnl,
                           const double *clalp, double rdelv) {
  if (!c || natom <= 0 || lmx < 1 || lmx > QX_KBR_MAX_LMX || !off || !mesh || !vnl || !clalp) {
    set_error("qx_set_kb_r: bad arguments (1 <= lmx <= %d)", QX_KBR_MAX_LMX);
    return QX_ERR_ARG;
  }
  Plan &pl = c->pl;
  const int npts = off[natom];
  for (int a = 0; a < natom; ++a)
    if (off[a + 1] < off[a]) { set_error("qx_set_kb_r: off not ascending"); return QX_ERR_ARG; }
  for (int i = 0; i < npts; ++i)
    if (mesh[i] < 0 || mesh[i] >= pl.n) { set_error("qx_set_kb_r: mesh index out of range"); return QX_ERR_ARG; }
  // line CSR: the projector points that fall on each x line (i3*k2 + i2)
  const long nlines = (long)pl.k2 * pl.k3;
  std::vector<int> loff(nlines + 1, 0);
  for (int i = 0; i < npts; ++i) loff[mesh[i] / pl.k1 + 1]++;
  for (long l = 0; l < nlines; ++l) loff[l + 1] += loff[l];
  std::vector<int4> lent(std::max(npts, 1));
  std::vector<int> fill(loff.begin(), loff.end() - 1);
  for (int a = 0; a < natom; ++a)
    for (int i = off[a]; i < off[a + 1]; ++i) lent[fill[mesh[i] / pl.k1]++] = make_int4(mesh[i] % pl.k1, i, a, 0);
  TRY(dalloc(c, &pl.d_kb_off, sizeof(int) * (natom + 1)));
  TRY(dalloc(c, &pl.d_kb_mesh, sizeof(int) * std::max(npts, 1)));
  TRY(dalloc(c, &pl.d_kb_clalp, sizeof(double) * lmx));
  TRY(dalloc(c, &pl.d_line_off, sizeof(int) * (nlines + 1)));
  TRY(dalloc(c, &pl.d_line_ent, sizeof(int4) * lent.size()));
  CK(cudaMemcpy(pl.d_kb_off, off, sizeof(int) * (natom + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(pl.d_kb_mesh, mesh, sizeof(int) * npts, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(pl.d_kb_clalp, clalp, sizeof(double) * lmx, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(pl.d_line_off, loff.data(), sizeof(int) * (nlines + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(pl.d_line_ent, lent.data(), sizeof(int4) * lent.size(), cudaMemcpyHostToDevice));
  void *v = nullptr;
  TRY(dalloc(c, &v, c->tsize() * (size_t)npts * lmx));
  TRY(up(c, v, vnl, (long)npts * lmx));
  pl.natom = natom;
  pl.npts = npts;
  pl.kb_lmx = lmx;
  pl.rdelv = rdelv;
  drop_scf_graphs(c);
  // real-space line buffer and projection sums, per chunk
  const long ch = pl.chunk;
  if (c->prec == QX_PREC_FP64) {
    pl.b64.kb_vnl = (double *)v;
    TRY(dalloc(c, &pl.b64.bufR, sizeof(double2) * ch * pl.n));
    TRY(dalloc(c, &pl.b64.sumr, sizeof(double2) * ch * natom * lmx));
  } else {
    pl.b32.kb_vnl = (float *)v;
    TRY(dalloc(c, &pl.b32.bufR, sizeof(float2) * ch * pl.n));
    TRY(dalloc(c, &pl.b32.sumr, sizeof(float2) * ch * natom * lmx));
  }
  c->have_kbr = true;
  return QX_OK;
}

extern "C" int qx_set_kb_r_builder(qx_ctx *c, int ntype, int lmx, int mxnl, const double *dltnl, const double *rcut,
                                   const double *tabnl, const double *dtabnl, const int *poly, const double *clalp,
                                   double rdelv, const double *rba) {
  if (!c || ntype <= 0 || lmx < 1 || lmx > QX_KBR_MAX_LMX || mxnl < 2 || !dltnl || !rcut || !tabnl || !poly ||
      !clalp || !rba || !(rdelv > 0.0)) {
    set_error("qx_set_kb_r_builder: bad arguments (1 <= lmx <= %d)", QX_KBR_MAX_LMX);
    return QX_ERR_ARG;
  }
  Plan &pl = c->pl;
  double rmax = 0.0;
  for (int it = 0; it < ntype; ++it) {
    if (!(dltnl[it] > 0.0) || !(rcut[it] > 0.0)) { set_error("qx_set_kb_r_builder: dltnl, rcut must be positive"); return QX_ERR_ARG; }
    if (2 * (long)(rcut[it] / (2.0 * dltnl[it])) + 2 > mxnl) {
      set_error("qx_set_kb_r_builder: radial table too short for the projector radius");
      return QX_ERR_ARG;
    }
    rmax = std::max(rmax, rcut[it]);
  }
  for (int i = 0; i < lmx * ntype; ++i)
    if (poly[i] < 0 || poly[i] > 8) { set_error("qx_set_kb_r_builder: poly out of range"); return QX_ERR_ARG; }
  // inverse lattice (rows b_i: s_i = b_i . r); the sphere must fit in one cell
  const double *a = rba;
  const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                     a[2] * (a[3] * a[7] - a[4] * a[6]);
  if (!(std::fabs(det) > 0.0)) { set_error("qx_set_kb_r_builder: singular lattice"); return QX_ERR_ARG; }
  double b[9];
  b[0] = (a[4] * a[8] - a[5] * a[7]) / det; b[1] = (a[2] * a[7] - a[1] * a[8]) / det; b[2] = (a[1] * a[5] - a[2] * a[4]) / det;
  b[3] = (a[5] * a[6] - a[3] * a[8]) / det; b[4] = (a[0] * a[8] - a[2] * a[6]) / det; b[5] = (a[2] * a[3] - a[0] * a[5]) / det;
  b[6] = (a[3] * a[7] - a[4] * a[6]) / det; b[7] = (a[1] * a[6] - a[0] * a[7]) / det; b[8] = (a[0] * a[4] - a[1] * a[3]) / det;
  KbrGeom G = {};
  const int kk[3] = {pl.k1, pl.k2, pl.k3};
  for (int i = 0; i < 9; ++i) G.rba[i] = a[i];
  for (int i = 0; i < 3; ++i) {
    const double bn = std::sqrt(b[3 * i] * b[3 * i] + b[3 * i + 1] * b[3 * i + 1] + b[3 * i + 2] * b[3 * i + 2]);
    G.k[i] = kk[i];
    G.nd[i] = (int)(rmax * bn * kk[i] + 0.5) + 1;
    if (2.0 * rmax * bn >= 1.0 || 2 * G.nd[i] + 1 > kk[i]) {
      set_error("qx_set_kb_r_builder: projector sphere wider than half the cell");
      return QX_ERR_ARG;
    }
  }
  const int nchan = lmx * ntype;
  TRY(dalloc(c, &c->d_kbr_dl, sizeof(double) * ntype));
  TRY(dalloc(c, &c->d_kbr_rcut, sizeof(double) * ntype));
  TRY(dalloc(c, &c->d_kbr_tab, sizeof(double) * (size_t)(mxnl + 1) * nchan));
  TRY(dalloc(c, &c->d_kbr_poly, sizeof(int) * nchan));
  TRY(dalloc(c, &pl.d_kb_clalp, sizeof(double) * lmx));
  CK(cudaMemcpyAsync(c->d_kbr_dl, dltnl, sizeof(double) * ntype, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_kbr_rcut, rcut, sizeof(double) * ntype, cudaMemcpyHostToDevice, c->st));
  // every channel at the species radius until qx_set_kb_r_channel_radii
  {
    std::vector<double> rcl((size_t)nchan);
    for (int it = 0; it < ntype; ++it)
      for (int l = 0; l < lmx; ++l) rcl[l + lmx * it] = rcut[it];
    TRY(dregrow(c, &c->d_kbr_rcl, sizeof(double) * nchan));
    CK(cudaMemcpyAsync(c->d_kbr_rcl, rcl.data(), sizeof(double) * nchan, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));   // rcl is a host temporary
    c->kbr_rcut_h.assign(rcut, rcut + ntype);
  }
  CK(cudaMemcpyAsync(c->d_kbr_tab, tabnl, sizeof(double) * (size_t)(mxnl + 1) * nchan, cudaMemcpyHostToDevice, c->st));
  c->d_kbr_dtab = nullptr;
  if (dtabnl) {
    TRY(dalloc(c, &c->d_kbr_dtab, sizeof(double) * (size_t)(mxnl + 1) * nchan));
    CK(cudaMemcpyAsync(c->d_kbr_dtab, dtabnl, sizeof(double) * (size_t)(mxnl + 1) * nchan, cudaMemcpyHostToDevice,
                       c->st));
  }
  CK(cudaMemcpyAsync(c->d_kbr_poly, poly, sizeof(int) * nchan, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(pl.d_kb_clalp, clalp, sizeof(double) * lmx, cudaMemcpyHostToDevice, c->st));
  drop_scf_graphs(c);
  c->kbr_geom = G;
  if (lmx != c->kbr_lmx) {   // table buffers sized per projector count: rebuilt at the next build
    c->kbr_cap = 0;
    c->kbr_dvnl_cap = 0;
    c->kbr_natom = 0;
    c->kbr_lmx = lmx;
  }
  c->kbr_ntype = ntype;
  c->kbr_mxnl = mxnl;
  pl.rdelv = rdelv;
  c->have_kbr_builder = true;
  return QX_OK;
}

extern "C" int qx_set_kb_r_channel_radii(qx_ctx *c, const double *rcl) {
  if (!c || !rcl) { set_error("qx_set_kb_r_channel_radii: bad arguments"); return QX_ERR_ARG; }
  if (!c->have_kbr_builder) { set_error("qx_set_kb_r_channel_radii: qx_set_kb_r_builder first"); return QX_ERR_STATE; }
  const int ntype = c->kbr_ntype, lmx = c->kbr_lmx;
  for (int it = 0; it < ntype; ++it)
    for (int l = 0; l < lmx; ++l) {
      const double r = rcl[l + lmx * it];
      if (!(r > 0.0) || r > c->kbr_rcut_h[it]) {
        set_error("qx_set_kb_r_channel_radii: radius %g of projector %d, species %d, outside (0, %g] (the species "
                  "radius of qx_set_kb_r_builder)", r, l, it, c->kbr_rcut_h[it]);
        return QX_ERR_ARG;
      }
    }
  CK(cudaMemcpyAsync(c->d_kbr_rcl, rcl, sizeof(double) * lmx * ntype, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return QX_OK;
}

extern "C" int qx_build_kb_r(qx_ctx *c, int natom, const int *ityp, const double *satm) {
  if (!c || natom <= 0 || natom > 65535 || !ityp || !satm) { set_error("qx_build_kb_r: bad arguments"); return QX_ERR_ARG; }
  if (!c->have_kbr_builder) { set_error("qx_build_kb_r: qx_set_kb_r_builder first"); return QX_ERR_STATE; }
  for (int a = 0; a < natom; ++a)
    if (ityp[a] < 0 || ityp[a] >= c->kbr_ntype) { set_error("qx_build_kb_r: ityp out of range"); return QX_ERR_ARG; }
  Plan &pl = c->pl;
  const size_t ts = c->tsize();
  const long nlines = (long)pl.k2 * pl.k3;
  bool moved = false;   // a table buffer was (re)allocated: captured graphs hold stale pointers
  if (natom != c->kbr_natom) {
    TRY(dregrow(c, &c->d_kbr_ityp, sizeof(int) * natom));
    TRY(dregrow(c, &c->d_kbr_satm, sizeof(double) * 3 * natom));
    TRY(dregrow(c, &c->d_kbr_cnt, sizeof(int) * natom));
    TRY(dregrow(c, &c->d_kbr_off, sizeof(int) * (natom + 1)));
    TRY(dregrow(c, &c->d_kbr_sumr, 2 * ts * (size_t)pl.chunk * natom * c->kbr_lmx));
    c->kbr_natom = natom;
    moved = true;
  }
  if (!c->d_kbr_loff) {
    TRY(dalloc(c, &c->d_kbr_lcnt, sizeof(int) * nlines));
    TRY(dalloc(c, &c->d_kbr_loff, sizeof(int) * (nlines + 1)));
    TRY(dalloc(c, &c->d_kbr_cursor, sizeof(int) * nlines));
    TRY(dalloc(c, &c->d_kbr_bufR, 2 * ts * (size_t)pl.chunk * pl.n));
    moved = true;
  }
  CK(cudaMemcpyAsync(c->d_kbr_ityp, ityp, sizeof(int) * natom, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_kbr_satm, satm, sizeof(double) * 3 * natom, cudaMemcpyHostToDevice, c->st));
  const KbrGeom &G = c->kbr_geom;
  kbr_count(G, natom, c->d_kbr_ityp, c->d_kbr_satm, c->d_kbr_rcut, c->d_kbr_cnt, c->d_kbr_off, c->st);
  int total = 0;
  CK(cudaMemcpyAsync(&total, c->d_kbr_off + natom, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (total > c->kbr_cap) {
    const long cap = (long)(total * 1.25) + 64;
    TRY(dregrow(c, &c->d_kbr_mesh, sizeof(int) * cap));
    TRY(dregrow(c, &c->d_kbr_ptatom, sizeof(int) * cap));
    TRY(dregrow(c, &c->d_kbr_lent, sizeof(int4) * cap));
    TRY(dregrow(c, &c->d_kbr_vnl, ts * c->kbr_lmx * (size_t)cap));
    c->kbr_cap = cap;
    moved = true;
  }
  if (c->d_kbr_dtab && c->kbr_dvnl_cap < c->kbr_cap) {
    TRY(dregrow(c, &c->d_kbr_dvnl, ts * 3 * c->kbr_lmx * (size_t)c->kbr_cap));
    c->kbr_dvnl_cap = c->kbr_cap;
  }
  if (c->prec == QX_PREC_FP64)
    kbr_fill<double>(G, natom, c->kbr_lmx, c->d_kbr_ityp, c->d_kbr_satm, c->d_kbr_rcut, c->d_kbr_rcl, c->d_kbr_dl, c->d_kbr_tab,
                     c->d_kbr_dtab, c->kbr_mxnl, c->d_kbr_poly, c->d_kbr_off, c->kbr_cap, c->d_kbr_mesh,
                     c->d_kbr_ptatom, (double *)c->d_kbr_vnl, (double *)c->d_kbr_dvnl, c->st);
  else
    kbr_fill<float>(G, natom, c->kbr_lmx, c->d_kbr_ityp, c->d_kbr_satm, c->d_kbr_rcut, c->d_kbr_rcl, c->d_kbr_dl, c->d_kbr_tab,
                    c->d_kbr_dtab, c->kbr_mxnl, c->d_kbr_poly, c->d_kbr_off, c->kbr_cap, c->d_kbr_mesh,
                    c->d_kbr_ptatom, (float *)c->d_kbr_vnl, (float *)c->d_kbr_dvnl, c->st);
  if (kbr_lines(c->d_kbr_off, natom, c->d_kbr_mesh, c->d_kbr_ptatom, pl.k1, nlines, c->d_kbr_lcnt, c->d_kbr_loff,
                c->d_kbr_cursor, c->d_kbr_lent, c->st)) {
    set_error("qx_build_kb_r: memset failed");
    return QX_ERR_CUDA;
  }
  CKL();
  if (pl.d_kb_off != c->d_kbr_off || pl.d_kb_mesh != c->d_kbr_mesh || pl.d_line_off != c->d_kbr_loff ||
      pl.d_line_ent != c->d_kbr_lent)
    moved = true;
  pl.d_kb_off = c->d_kbr_off;
  pl.d_kb_mesh = c->d_kbr_mesh;
  pl.d_line_off = c->d_kbr_loff;
  pl.d_line_ent = c->d_kbr_lent;
  if (c->prec == QX_PREC_FP64) {
    moved |= pl.b64.kb_vnl != (double *)c->d_kbr_vnl || pl.b64.sumr != (double2 *)c->d_kbr_sumr;
    pl.b64.kb_vnl = (double *)c->d_kbr_vnl;
    pl.b64.bufR = (double2 *)c->d_kbr_bufR;
    pl.b64.sumr = (double2 *)c->d_kbr_sumr;
  } else {
    moved |= pl.b32.kb_vnl != (float *)c->d_kbr_vnl || pl.b32.sumr != (float2 *)c->d_kbr_sumr;
    pl.b32.kb_vnl = (float *)c->d_kbr_vnl;
    pl.b32.bufR = (float2 *)c->d_kbr_bufR;
    pl.b32.sumr = (float2 *)c->d_kbr_sumr;
  }
  pl.natom = natom;
  pl.npts = total;
  pl.kb_lmx = c->kbr_lmx;
  if (moved) drop_scf_graphs(c);
  c->have_kbr = true;
  return QX_OK;
}

extern "C" int qx_get_kb_r(qx_ctx *c, int *npts, int *off, int *mesh, double *vnl) {
  if (!c || !npts) { set_error("qx_get_kb_r: null"); return QX_ERR_ARG; }
  if (!c->have_kbr) { set_error("qx_get_kb_r: real-space tables not set"); return QX_ERR_STATE; }
  const Plan &pl = c->pl;
  CK(cudaStreamSynchronize(c->st));
  *npts = pl.npts;
  if (off) CK(cudaMemcpy(off, pl.d_kb_off, sizeof(int) * (pl.natom + 1), cudaMemcpyDeviceToHost));
  if (mesh) CK(cudaMemcpy(mesh, pl.d_kb_mesh, sizeof(int) * pl.npts, cudaMemcpyDeviceToHost));
  if (vnl) {
    if (c->prec == QX_PREC_FP64) {
      CK(cudaMemcpy(vnl, pl.b64.kb_vnl, sizeof(double) * pl.kb_lmx * pl.npts, cudaMemcpyDeviceToHost));
    } else {
      std::vector<float> h((size_t)pl.kb_lmx * pl.npts);
      CK(cudaMemcpy(h.data(), pl.b32.kb_vnl, sizeof(float) * h.size(), cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < h.size(); ++i) vnl[i] = h[i];
    }
  }
  return QX_OK;
}

extern "C" int qx_set_nlmode(qx_ctx *c, int mode) {
  if (!c || mode < 0 || mode > 2) { set_error("qx_set_nlmode: bad mode"); return QX_ERR_ARG; }
  if (mode == QX_NL_GSPACE && !c->have_kbg) { set_error("qx_set_nlmode: G-space tables not set"); return QX_ERR_STATE; }
  if (mode == QX_NL_RSPACE && !c->have_kbr) { set_error("qx_set_nlmode: real-space tables not set"); return QX_ERR_STATE; }
  c->nlmode = mode;
  return QX_OK;
}

__global__ void k_wocc(const double *occ, double *w, int n, double rv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) w[i] = occ[i] / rv;
}

extern "C" int qx_set_occ(qx_ctx *c, const double *occ, double rvol) {
  if (!c || !occ || rvol <= 0) { set_error("qx_set_occ: bad arguments"); return QX_ERR_ARG; }
  CK(cudaMemcpyAsync(c->d_occ, occ, sizeof(double) * c->nb, cudaMemcpyHostToDevice, c->st));
  k_wocc<<<(c->nb + 127) / 128, 128, 0, c->st>>>(c->d_occ, c->d_wocc, c->nb, rvol); note_launch();
  CKL();
  c->rvol = rvol;
  c->have_occ = true;
  return QX_OK;
}

extern "C" int qx_put_psi(qx_ctx *c, const double *x) { return c && x ? up(c, c->psi, x, (long)c->nb * c->ne) : QX_ERR_ARG; }
extern "C" int qx_get_psi(qx_ctx *c, double *x) { return c && x ? down(c, x, c->psi, (long)c->nb * c->ne) : QX_ERR_ARG; }
extern "C" int qx_put_hpsi(qx_ctx *c, const double *x) { return c && x ? up(c, c->hpsi, x, (long)c->nb * c->ne) : QX_ERR_ARG; }
extern "C" int qx_get_hpsi(qx_ctx *c, double *x) { return c && x ? down(c, x, c->hpsi, (long)c->nb * c->ne) : QX_ERR_ARG; }
extern "C" int qx_get_eig(qx_ctx *c, double *x) {
  if (!c || !x) return QX_ERR_ARG;
  CK(cudaMemcpyAsync(x, c->d_eig, sizeof(double) * c->nb, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return QX_OK;
}

static int ensure_rho(qx_ctx *c) {
  if (!c->d_rho_out) {
    TRY(dalloc(c, &c->d_rho_out, sizeof(double) * c->pl.n));
    TRY(dalloc(c, &c->d_rho_in, sizeof(double) * c->pl.n));
    CK(cudaMemset(c->d_rho_in, 0, sizeof(double) * c->pl.n));
  }
  return 0;
}
extern "C" int qx_get_rho(qx_ctx *c, double *x) {
  if (!c || !x || !c->d_rho_out) { set_error("qx_get_rho: no density"); return QX_ERR_STATE; }
  CK(cudaMemcpyAsync(x, c->d_rho_out, sizeof(double) * c->pl.n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return QX_OK;
}
extern "C" int qx_put_rho(qx_ctx *c, const double *x) {
  if (!c || !x) return QX_ERR_ARG;
  TRY(ensure_rho(c));
  CK(cudaMemcpyAsync(c->d_rho_in, x, sizeof(double) * c->pl.n, cudaMemcpyHostToDevice, c->st));
  return QX_OK;
}
extern "C" int qx_get_glocal(qx_ctx *c, double *x) {
  if (!c || !x || !c->d_glocal) return QX_ERR_STATE;
  CK(cudaMemcpyAsync(x, c->d_glocal, sizeof(double) * c->pl.n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return QX_OK;
}
extern "C" void *qx_dev_ptr(qx_ctx *c, int which) {
  if (!c) return nullptr;
  switch (which) {
    case 0: return c->psi;
    case 1: return c->hpsi;
    case 2: return c->d_rho_in;
    case 3: return c->d_rho_out;
    case 5: return c->d_vloc;
    case 4: return c->d_eig;
    default: return nullptr;
  }
}
extern "C" int qx_sync(qx_ctx *c) {
  if (!c) return QX_ERR_ARG;
  CK(cudaStreamSynchronize(c->st));
  CKL();
  const int te = tc_error_take();
  if (te) { set_error("qx_sync: tensor-core GEMM wait timed out (code %d)", te); return QX_ERR_CUDA; }
  return QX_OK;
}

// ---------------------------------------------------------------------------
static PipeParams base_params(const qx_ctx *c) {
  const Plan &pl = c->pl;
  PipeParams P;
  P.k1 = pl.k1; P.k2 = pl.k2; P.k3 = pl.k3;
  P.m1 = pl.m1; P.m2 = pl.m2; P.P1 = pl.P1; P.P2 = pl.P2;
  P.nplw = pl.nplw;
  P.L1 = pl.L[0]; P.L2 = pl.L[1]; P.L3 = pl.L[2];
  P.row_lo = pl.d_row_lo; P.row_hi = pl.d_row_hi; P.row_off = pl.d_row_off; P.row_ent = pl.d_row_ent;
  P.col_ja = pl.d_col_ja; P.col_ig = pl.d_col_ig; P.ncol = pl.ncol;
  P.pairs = c->d_allpairs;
  P.npair_dev = nullptr;
  P.npair = c->npair_all;
  P.pair0 = 0;
  P.inv_n = 1.0 / (double)pl.n;
  return P;
}

// The context's second stream and its fork/join events, made on first use.
static int side_stream(qx_ctx *c) {
  if (!c->st2) {
    CK(cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
  }
  return 0;
}

// QX_KB_STREAM=0 keeps the G-space KB contractions behind the FFT pipeline
// on one stream (read at every call).
static bool kb_side_stream_enabled() {
  const char *v = getenv("QX_KB_STREAM");
  return !(v && v[0] == '0');
}

// H|c> for the bands listed in `pairs` (device, 2 per pair).  npair_dev
// (device count) bounds the pairs; npair_max is the host bound.  colmap /
// ncol_dev list the same bands for the G-space KB GEMMs.
template <typename T>
static int hpsi_impl(qx_ctx *c, const T *cin, T *out, const int *pairs, const int *npair_dev, int npair_max,
                     const int *colmap, const int *ncol_dev, int ncol_max, int flags) {
  if (!c->have_glocal) { set_error("hpsi: glocal not set"); return QX_ERR_STATE; }
  const Plan &pl = c->pl;
  PipeParams P = base_params(c);
  P.pairs = pairs;
  P.npair_dev = npair_dev;
  const int nlm = (flags & QX_HPSI_NONLOCAL) ? c->nlmode : 0;
  const double *dk = (flags & QX_HPSI_KINETIC) ? c->d_dk : nullptr;
  const int acc = (flags & QX_HPSI_ACCUMULATE) ? 1 : 0;
  // G-space KB: out = [out +] beta D <beta|c> on the second stream while the
  // FFT pipeline runs here; the pipeline's last kernel then adds the kinetic
  // and local parts to it.  Otherwise the KB GEMMs follow the pipeline on
  // this stream and add onto its result.
  const bool kb = nlm == QX_NL_GSPACE;
  const bool side = kb && kb_side_stream_enabled();
  cudaStream_t kst = c->st;
  if (side) {
    TRY(side_stream(c));
    CK(cudaEventRecord(c->ev_fork, c->st));
    CK(cudaStreamWaitEvent(c->st2, c->ev_fork, 0));
    kst = c->st2;
  }
  auto kb_gemms = [&](T beta_out) -> int {
    Bufs<T> &b = pl.bufs<T>();
    T *proj = (T *)c->proj;
    const int np = pl.nproj;
    // The tensor-core GEMMs take whole columns: with a band list they work on
    // all ncol_max columns, which leaves the columns of bands not in the list
    // holding unused values (the CG reads only active bands).
    const int *cm = colmap, *nd = ncol_dev;
    if (sizeof(T) == sizeof(float) && tc_enabled()) {
      cm = nullptr;
      nd = nullptr;
    }
    // proj = D <beta|c>: the KB energies D (vclalp) scale the rows in the
    // contraction's epilogue
    long kld = 0;
    const T *kb = kbg_operand<T>(c, &kld);
    TRY(gemm<T>(true, false, np, ncol_max, c->ne, (T)1, kb, kld, cin, c->ne, (T)0, proj, np, 2, cm, nd, kst,
                c->gws, c->gws_bytes, (const T *)b.vclalp, c->tcpad, c->tcpad_bytes));
    TRY(gemm<T>(false, false, c->ne, ncol_max, np, (T)1, kb, kld, proj, np, beta_out, out, c->ne, 0, cm, nd,
                kst, c->gws, c->gws_bytes, nullptr, c->tcpad, c->tcpad_bytes));
    CKL();
    return 0;
  };
  if (side) {
    TRY(kb_gemms(acc ? (T)1 : (T)0));
    CK(cudaEventRecord(c->ev_join, c->st2));
  }
  for (int p0 = 0; p0 < npair_max; p0 += pl.chunk) {
    P.pair0 = p0;
    const int npl = std::min(pl.chunk, npair_max - p0);
    P.npair = npair_max;
    TRY(launch_hpsi_chunk<T>(pl, P, npl, cin, c->ne, out, c->ne, dk, side ? 1 : acc, nlm == QX_NL_RSPACE ? 2 : 0,
                             c->st, (side && p0 == 0) ? c->ev_join : nullptr));
    CKL();
  }
  if (kb && !side) TRY(kb_gemms((T)1));
  return 0;
}

template <typename T>
static int hpsi_all(qx_ctx *c, const T *cin, T *out, int nb, int flags) {
  const int npair = (nb + 1) / 2;
  // the all-bands pair list covers nband; fewer bands use its prefix, which
  // is consecutive, except for an odd tail handled by the count bound
  if (nb > c->nb) { set_error("hpsi: nb > nband"); return QX_ERR_ARG; }
  if (nb % 2 && nb != c->nb) {
    std::vector<int> pr(2 * npair);
    for (int p = 0; p < npair; ++p) { pr[2 * p] = 2 * p; pr[2 * p + 1] = (2 * p + 1 < nb) ? 2 * p + 1 : -1; }
    int *dp = (int *)c->cg.pairs;
    CK(cudaMemcpyAsync(dp, pr.data(), sizeof(int) * pr.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return hpsi_impl<T>(c, cin, out, dp, nullptr, npair, nullptr, nullptr, nb, flags);
  }
  return hpsi_impl<T>(c, cin, out, c->d_allpairs, nullptr, npair, nullptr, nullptr, nb, flags);
}

extern "C" int qx_hpsi(qx_ctx *c, const void *cin, void *out, int nb, int flags) {
  if (!c || !cin || !out || nb <= 0) { set_error("qx_hpsi: bad arguments"); return QX_ERR_ARG; }
  if (c->prec == QX_PREC_FP64) return hpsi_all<double>(c, (const double *)cin, (double *)out, nb, flags);
  return hpsi_all<float>(c, (const float *)cin, (float *)out, nb, flags);
}

template <typename T>
static int ekinetic_impl(qx_ctx *c, double *ekin_sum, double *ekib) {
  qx::ekin<T>(c->nb, c->ne, c->ne, (const T *)c->psi, c->d_dk, c->d_ekib, c->st);
  CKL();
  if (ekin_sum || ekib) {
    std::vector<double> e(c->nb), o(c->nb);
    CK(cudaMemcpyAsync(e.data(), c->d_ekib, sizeof(double) * c->nb, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(o.data(), c->d_occ, sizeof(double) * c->nb, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (ekib) memcpy(ekib, e.data(), sizeof(double) * c->nb);
    if (ekin_sum) {
      double s = 0.0;
      for (int b = 0; b < c->nb; ++b) s += (c->have_occ ? o[b] : 0.0) * 0.5 * e[b];
      *ekin_sum = s;
    }
  }
  return 0;
}

extern "C" int qx_ekinetic(qx_ctx *c, double *ekin_out, double *ekib) {
  if (!c) return QX_ERR_ARG;
  return c->prec == QX_PREC_FP64 ? ekinetic_impl<double>(c, ekin_out, ekib) : ekinetic_impl<float>(c, ekin_out, ekib);
}

extern "C" int qx_enonloc(qx_ctx *c) {
  if (!c) return QX_ERR_ARG;
  TRY(qx_ekinetic(c, nullptr, nullptr));
  return qx_hpsi(c, c->psi, c->hpsi, c->nb, QX_HPSI_KINETIC | QX_HPSI_NONLOCAL);
}

template <typename T>
static int hmatrix_impl(qx_ctx *c, double *hsub) {
  const int nb = c->nb;
  T *m = (T *)c->mat_t;
  // m(j, i) = <psi_j | hpsi_i>
  TRY(gemm<T>(true, false, nb, nb, c->ne, (T)1, (const T *)c->psi, c->ne, (const T *)c->hpsi, c->ne, (T)0, m, nb, 1,
              nullptr, nullptr, c->st, c->gws, c->gws_bytes, nullptr, c->tcpad, c->tcpad_bytes));
  symmetrize_lower<T>(m, c->d_hsub, c->d_eig, nb, c->st);
  CKL();
  c->have_hsub = true;
  if (hsub) {
    CK(cudaMemcpyAsync(hsub, c->d_hsub, sizeof(double) * nb * nb, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  return 0;
}
extern "C" int qx_hmatrix(qx_ctx *c, double *hsub) {
  if (!c) return QX_ERR_ARG;
  return c->prec == QX_PREC_FP64 ? hmatrix_impl<double>(c, hsub) : hmatrix_impl<float>(c, hsub);
}

template <typename T>
static int gradres_impl(qx_ctx *c, double *prod, double *zmax, double *zsum) {
  gradres<T>(c->nb, c->ne, c->ne, (const T *)c->psi, (const T *)c->hpsi, c->d_eig, c->d_prod, c->st);
  CKL();
  if (c->defer) {
    gradres_stats(c->d_prod, c->have_occ ? c->d_occ : nullptr, c->nb, c->d_sc + 5, c->st);
    CKL();
    return 0;
  }
  std::vector<double> p(c->nb), o(c->nb, 0.0);
  CK(cudaMemcpyAsync(p.data(), c->d_prod, sizeof(double) * c->nb, cudaMemcpyDeviceToHost, c->st));
  if (c->have_occ) CK(cudaMemcpyAsync(o.data(), c->d_occ, sizeof(double) * c->nb, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double m = 0.0, s = 0.0;
  for (int b = 0; b < c->nb; ++b) { m = std::max(m, p[b]); s += p[b] * o[b]; }
  if (prod) memcpy(prod, p.data(), sizeof(double) * c->nb);
  if (zmax) *zmax = m;
  if (zsum) *zsum = s;
  return 0;
}
extern "C" int qx_gradres(qx_ctx *c, double *prod, double *zmax, double *zsum) {
  if (!c) return QX_ERR_ARG;
  return c->prec == QX_PREC_FP64 ? gradres_impl<double>(c, prod, zmax, zsum) : gradres_impl<float>(c, prod, zmax, zsum);
}

template <typename T>
static int rotate(qx_ctx *c, void *&arr) {
  const int nb = c->nb;
  const T *U = (const T *)c->mat_t;
  TRY(gemm<T>(false, false, c->ne, nb, nb, (T)1, (const T *)arr, c->ne, U, nb, (T)0, (T *)c->tmp, c->ne, 0, nullptr,
              nullptr, c->st, c->gws, c->gws_bytes, nullptr, c->tcpad, c->tcpad_bytes));
  CKL();
  std::swap(arr, c->tmp);
  return 0;
}

template <typename T>
static int untryt_impl(qx_ctx *c, double *ev, int *sweeps) {
  if (!c->have_hsub) { set_error("untryt: call hmatrix first"); return QX_ERR_STATE; }
  const int nb = c->nb;
  CK(cudaMemcpyAsync(c->d_mat, c->d_hsub, sizeof(double) * nb * nb, cudaMemcpyDeviceToDevice, c->st));
  TRY(side_stream(c));
  TRY(syev(c->d_mat, nb, c->d_w, c->d_V, c->d_eigws, c->d_info, c->st, c->st2, c->ev_fork, c->ev_join));
  CKL();
  // U in the working precision for the GEMMs
  convert<double, T>(c->d_V, (T *)c->mat_t, (long)nb * nb, c->st);
  CKL();
  TRY(rotate<T>(c, c->psi));
  c->have_u = true;
  c->have_hsub = false;
  if (c->defer) return 0;   // status read with the iteration's results
  int info = 0;
  CK(cudaMemcpyAsync(&info, c->d_info, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (info <= 0) { set_error("untryt: eigen-decomposition produced no eigenvectors"); return QX_ERR_EIG; }
  if (sweeps) *sweeps = info;
  if (ev) CK(cudaMemcpy(ev, c->d_w, sizeof(double) * nb, cudaMemcpyDeviceToHost));
  return 0;
}
extern "C" int qx_untryt(qx_ctx *c, double *ev) {
  if (!c) return QX_ERR_ARG;
  return c->prec == QX_PREC_FP64 ? untryt_impl<double>(c, ev, nullptr) : untryt_impl<float>(c, ev, nullptr);
}
extern "C" int qx_untryhc(qx_ctx *c) {
  if (!c) return QX_ERR_ARG;
  if (!c->have_u) { set_error("untryhc: call untryt first"); return QX_ERR_STATE; }
  return c->prec == QX_PREC_FP64 ? rotate<double>(c, c->hpsi) : rotate<float>(c, c->hpsi);
}

template <typename T>
static int eigen_impl(qx_ctx *c, const qx_cgparm *p, int *nriter, int *nhpsi_out) {
  const int nb = c->nb, ne = c->ne;
  CgParm pm{p->itermx, p->iteremx, p->noband, p->tolera, p->roughfzan, p->roughfeig, p->threinn, p->wdinner};
  T *x = (T *)c->psi, *hx = (T *)c->hpsi, *g = (T *)c->g, *h = (T *)c->h, *gh = (T *)c->gh, *snap = (T *)c->snap;
  T *pm_t = (T *)c->mat_t;
  const CgState &s = c->cg;
  // lower-band snapshot (real*4 when requested in FP64 contexts)
  if (sizeof(T) == sizeof(double) && p->ccreal4) {
    convert<double, float>((const double *)x, (float *)c->tmp, (long)nb * ne, c->st);
    convert<float, double>((const float *)c->tmp, (double *)snap, (long)nb * ne, c->st);
  } else {
    CK(cudaMemcpyAsync(snap, x, sizeof(T) * (size_t)nb * ne, cudaMemcpyDeviceToDevice, c->st));
  }
  cg_init<T>(nb, ne, ne, x, hx, g, s, c->st);
  CKL();
  const int maxit = std::max(p->itermx, p->iteremx);
  int nh = 0;
  for (int it = 0; it < maxit; ++it) {
    cg_prec<T>(nb, ne, ne, g, h, c->d_dk, s, c->st);
    // subgs3: Pm = snap^T h ; Pm masked to j < i, active i ; h -= snap * Pm
    TRY(gemm<T>(true, false, nb, nb, ne, (T)1, snap, ne, h, ne, (T)0, pm_t, nb, 1, nullptr, nullptr, c->st, c->gws, c->gws_bytes, nullptr, c->tcpad, c->tcpad_bytes));
    cg_mask<T>(nb, pm_t, s, c->st);
    TRY(gemm<T>(false, false, ne, nb, nb, (T)-1, snap, ne, pm_t, nb, (T)1, h, ne, 0, nullptr, nullptr, c->st, nullptr, 0, nullptr, c->tcpad, c->tcpad_bytes));
    cg_orth<T>(nb, ne, ne, x, hx, h, s, c->st);
    cg_list(nb, s, c->st);
    CKL();
    TRY(hpsi_impl<T>(c, h, gh, s.pairs, s.npair, c->npair_all, s.list, s.nact, nb,
                     QX_HPSI_KINETIC | QX_HPSI_NONLOCAL));
    cg_update<T>(nb, ne, ne, x, hx, g, h, gh, s, pm, c->st);
    CKL();
  }
  // eig and iteration counts
  CK(cudaMemcpyAsync(c->d_eig, s.eig, sizeof(double) * nb, cudaMemcpyDeviceToDevice, c->st));
  c->have_hsub = false;
  if (c->defer) {
    iter_sum(s.iter, nb, c->d_info + 2, c->st);
    CKL();
    return 0;
  }
  std::vector<int> iters(nb);
  CK(cudaMemcpyAsync(iters.data(), s.iter, sizeof(int) * nb, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  for (int b = 0; b < nb; ++b) nh += iters[b];
  if (nriter) memcpy(nriter, iters.data(), sizeof(int) * nb);
  if (nhpsi_out) *nhpsi_out = nh;
  c->have_hsub = false;
  return 0;
}
// One CG step of band *cur (the body of the sequential loop): preconditioned
// direction, subgs3 against the snapshot of the bands below (already final),
// subgs4, H|h> of this one band, BKL update and, once the band stops, the
// move to the next band.
template <typename T>
static int seq_body(qx_ctx *c, const CgParm &pm, const SeqArgs &q) {
  const int nb = c->nb, ne = c->ne;
  T *x = (T *)c->psi, *hx = (T *)c->hpsi, *g = (T *)c->g, *h = (T *)c->h, *gh = (T *)c->gh;
  const T *snap = (const T *)c->snap;
  const CgState &s = c->cg;
  cg_prec<T>(nb, ne, ne, g, h, c->d_dk, s, c->st, q.cur);
  seq_dots<T>(nb, q.cur, ne, snap, ne, h, ne, q.cur, 1, nullptr, c->d_seqw, c->st);
  seq_axpy<T>(nb, q.cur, ne, snap, ne, c->d_seqw, -1.0, h, ne, q.cur, c->st);
  cg_orth<T>(nb, ne, ne, x, hx, h, s, c->st, q.cur);
  CKL();
  const int fl = QX_HPSI_KINETIC | (c->nlmode == QX_NL_RSPACE ? QX_HPSI_NONLOCAL : 0);
  TRY(hpsi_impl<T>(c, h, gh, q.pairs, nullptr, 1, nullptr, nullptr, 1, fl));
  if (c->nlmode == QX_NL_GSPACE) {
    const Bufs<T> &b = c->pl.bufs<T>();
    const int np = c->pl.nproj;
    seq_dots<T>(np, nullptr, ne, b.kbg, ne, h, ne, q.cur, 2, b.vclalp, c->d_seqw, c->st);
    seq_axpy<T>(np, nullptr, ne, b.kbg, ne, c->d_seqw, 1.0, gh, ne, q.cur, c->st);
  }
  cg_update_seq<T>(ne, ne, x, hx, g, h, gh, s, pm, q, c->st);
  CKL();
  return 0;
}

// The sequential loop as one graph: a while node whose body is seq_body,
// captured once per set of buffers and parameters.  The body's last kernel
// clears the loop condition after the last band, so a whole CG sweep is one
// graph launch with no host round trip per band or step.
template <typename T>
static int seq_graph(qx_ctx *c, const qx_cgparm *p, const CgParm &pm) {
  const Bufs<T> &b = c->pl.bufs<T>();
  const void *keyp[] = {c->psi, c->hpsi, c->snap, b.kbg, b.vclalp};
  std::vector<char> key(sizeof(keyp) + sizeof(qx_cgparm) + 2 * sizeof(int));
  memcpy(key.data(), keyp, sizeof(keyp));
  memcpy(key.data() + sizeof(keyp), p, sizeof(qx_cgparm));
  const int extra[2] = {c->nlmode, c->pl.nproj};
  memcpy(key.data() + sizeof(keyp) + sizeof(qx_cgparm), extra, sizeof(extra));
  if (c->seq_exec && key == c->seq_key) return 0;
  if (c->seq_exec) { cudaGraphExecDestroy(c->seq_exec); c->seq_exec = nullptr; }
  if (c->seq_graph) { cudaGraphDestroy(c->seq_graph); c->seq_graph = nullptr; }
  if (!c->cap_st) CK(cudaStreamCreateWithFlags(&c->cap_st, cudaStreamNonBlocking));
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  c->seq_graph = g;
  cudaGraphConditionalHandle hd;
  CK(cudaGraphConditionalHandleCreate(&hd, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = hd;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, g, nullptr, 0, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  SeqArgs q{c->d_seqi, c->d_seqi + 1, c->d_seqi + 3, c->snap, c->nb,
            (sizeof(T) == sizeof(double) && p->ccreal4) ? 1 : 0, hd};
  CK(cudaStreamBeginCaptureToGraph(c->cap_st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  cudaStream_t user = c->st;
  c->st = c->cap_st;
  const long l0 = g_launches.load();
  const int r = seq_body<T>(c, pm, q);
  c->seq_body_launches = g_launches.load() - l0;
  g_launches.fetch_sub(c->seq_body_launches);
  c->st = user;
  cudaGraph_t captured = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(c->cap_st, &captured);
  if (r) return r;
  CK(ec);
  CK(cudaGraphInstantiate(&c->seq_exec, g, 0));
  c->seq_key = key;
  return 0;
}

// eigen_BKL on one rank: bands one after another, band ib projected against
// the final vectors of bands < ib (the reference's own order within a rank).
template <typename T>
static int eigen_seq_impl(qx_ctx *c, const qx_cgparm *p, int *nriter, int *nhpsi_out) {
  const int nb = c->nb, ne = c->ne;
  CgParm pm{p->itermx, p->iteremx, p->noband, p->tolera, p->roughfzan, p->roughfeig, p->threinn, p->wdinner};
  T *x = (T *)c->psi, *hx = (T *)c->hpsi, *g = (T *)c->g;
  const int need = std::max(nb, c->pl.nproj);
  if (c->seqw_len < need) {
    TRY(dalloc(c, &c->d_seqw, sizeof(double) * need));
    c->seqw_len = need;
  }
  if (!c->d_seqi) TRY(dalloc(c, &c->d_seqi, sizeof(int) * 4));
  // No entry snapshot: band ib reads the columns of bands < ib only, and each
  // of those is written with its final vector before band ib starts.
  cg_init<T>(nb, ne, ne, x, hx, g, c->cg, c->st);
  CKL();
  TRY(seq_graph<T>(c, p, pm));
  SeqArgs q{c->d_seqi, c->d_seqi + 1, c->d_seqi + 3, c->snap, nb, 0, 0};
  seq_reset(q, c->st);
  CKL();
  CK(cudaGraphLaunch(c->seq_exec, c->st));
  CK(cudaMemcpyAsync(c->d_eig, c->cg.eig, sizeof(double) * nb, cudaMemcpyDeviceToDevice, c->st));
  if (c->defer) iter_sum(c->cg.iter, nb, c->d_info + 2, c->st);
  std::vector<int> iters(nb);
  CK(cudaMemcpyAsync(iters.data(), c->cg.iter, sizeof(int) * nb, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  int nh = 0;
  for (int b = 0; b < nb; ++b) nh += iters[b];
  g_launches.fetch_add(c->seq_body_launches * nh);
  if (nriter) memcpy(nriter, iters.data(), sizeof(int) * nb);
  if (nhpsi_out) *nhpsi_out = nh;
  c->have_hsub = false;
  return 0;
}

extern "C" int qx_eigen(qx_ctx *c, const qx_cgparm *p, int *nriter, int *nhpsi) {
  if (!c || !p) return QX_ERR_ARG;
  if (p->sequential)
    return c->prec == QX_PREC_FP64 ? eigen_seq_impl<double>(c, p, nriter, nhpsi)
                                   : eigen_seq_impl<float>(c, p, nriter, nhpsi);
  return c->prec == QX_PREC_FP64 ? eigen_impl<double>(c, p, nriter, nhpsi) : eigen_impl<float>(c, p, nriter, nhpsi);
}

template <typename T>
static int schmidt_impl(qx_ctx *c) {
  const int nb = c->nb, ne = c->ne;
  T *m = (T *)c->mat_t;
  TRY(gemm<T>(true, false, nb, nb, ne, (T)1, (const T *)c->psi, ne, (const T *)c->psi, ne, (T)0, m, nb, 1, nullptr,
              nullptr, c->st, c->gws, c->gws_bytes, nullptr, c->tcpad, c->tcpad_bytes));
  convert<T, double>(m, c->d_mat, (long)nb * nb, c->st);
  TRY(cholinv(c->d_mat, nb, c->d_eigws, c->d_info + 1, c->st));
  CKL();
  if (!c->defer) {   // deferred: the status is read with the iteration's results
    int info = 0;
    CK(cudaMemcpyAsync(&info, c->d_info + 1, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (info < 0) { set_error("schmidt: a grid barrier of the Cholesky kernel timed out"); return QX_ERR_CUDA; }
    if (info) { set_error("schmidt: <psi|psi> not positive definite at band %d", info - 1); return QX_ERR_NOTPD; }
  }
  convert<double, T>(c->d_mat, m, (long)nb * nb, c->st);
  // psi <- psi * Linv^T
  TRY(gemm<T>(false, true, ne, nb, nb, (T)1, (const T *)c->psi, ne, m, nb, (T)0, (T *)c->tmp, ne, 0, nullptr, nullptr,
              c->st, nullptr, 0, nullptr, c->tcpad, c->tcpad_bytes));
  CKL();
  std::swap(c->psi, c->tmp);
  return 0;
}
extern "C" int qx_schmidt(qx_ctx *c) {
  if (!c) return QX_ERR_ARG;
  return c->prec == QX_PREC_FP64 ? schmidt_impl<double>(c) : schmidt_impl<float>(c);
}

template <typename T>
static int softchg_impl(qx_ctx *c) {
  if (!c->have_occ) { set_error("softchg: occupations not set"); return QX_ERR_STATE; }
  TRY(ensure_rho(c));
  const Plan &pl = c->pl;
  PipeParams P = base_params(c);
  for (int p0 = 0; p0 < c->npair_all; p0 += pl.chunk) {
    // pairs p0 .. p0+npl-1: the kernels bound pairs by npair and k_xrho
    // loops over npair - pair0 of them
    P.pair0 = p0;
    const int npl = std::min(pl.chunk, c->npair_all - p0);
    P.npair = p0 + npl;
    TRY(launch_rho_chunk<T>(pl, P, npl, (const T *)c->psi, c->ne, c->d_wocc, c->d_rho_out, p0 > 0, c->st));
    CKL();
  }
  return 0;
}
extern "C" int qx_softchg(qx_ctx *c) {
  if (!c) return QX_ERR_ARG;
  return c->prec == QX_PREC_FP64 ? softchg_impl<double>(c) : softchg_impl<float>(c);
}

// ---------------------------------------------------------------------------
// SCF iteration
extern "C" int qx_scf_init(qx_ctx *c, const double *vloc, const double *cross, double ecutdens, double eion,
                           double mixbeta, double q0) {
  if (!c || !vloc || !cross) return QX_ERR_ARG;
  TRY(ensure_rho(c));
  const long n = c->pl.n;
  if (!c->d_vloc) {
    TRY(dalloc(c, &c->d_vloc, sizeof(double) * n));
    TRY(dalloc(c, &c->d_g2, sizeof(double) * n));
    TRY(dalloc(c, &c->d_zg, sizeof(double2) * n));
    TRY(dalloc(c, &c->d_part, sizeof(double) * 2 * SCF_NBLK));
    TRY(dalloc(c, &c->d_sc, sizeof(double) * 16));
    if (!c->d_glocal) TRY(dalloc(c, &c->d_glocal, sizeof(double) * n));
  }
  CK(cudaMemcpyAsync(c->d_vloc, vloc, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  grid_g2(c->pl.k1, c->pl.k2, c->pl.k3, cross, ecutdens, c->d_g2, c->st);
  CKL();
  c->eion = eion;
  c->mixbeta = mixbeta;
  c->q02 = q0 * q0;
  // smallest and largest nonzero |G|^2 of the density sphere (the metric of
  // the Pulay residual, reclat.f90:205 and chgdns.f90:661-668)
  {
    const int k1 = c->pl.k1, k2 = c->pl.k2, k3 = c->pl.k3;
    double mn = 0.0, mx = 0.0;
    for (int i3 = 0; i3 < k3; ++i3)
      for (int i2 = 0; i2 < k2; ++i2)
        for (int i1 = 0; i1 < k1; ++i1) {
          const double d1 = i1 <= k1 / 2 ? i1 : i1 - k1, d2 = i2 <= k2 / 2 ? i2 : i2 - k2,
                       d3 = i3 <= k3 / 2 ? i3 : i3 - k3;
          const double gx = cross[0] * d1 + cross[3] * d2 + cross[6] * d3;
          const double gy = cross[1] * d1 + cross[4] * d2 + cross[7] * d3;
          const double gz = cross[2] * d1 + cross[5] * d2 + cross[8] * d3;
          const double q = gx * gx + gy * gy + gz * gz;
          if (q > 0.0 && q <= ecutdens) {
            if (mn == 0.0 || q < mn) mn = q;
            if (q > mx) mx = q;
          }
        }
    c->g2min = mn;
    c->g2max = mx;
  }
  c->scf_ready = true;
  return QX_OK;
}

extern "C" int qx_scf_mixing(qx_ctx *c, int itratn, double cmetric) {
  if (!c || itratn < 0 || itratn > PULAY_MAX) {
    set_error("qx_scf_mixing: itratn must be in [0, %d]", PULAY_MAX);
    return QX_ERR_ARG;
  }
  if (!c->scf_ready) { set_error("qx_scf_mixing: call qx_scf_init first"); return QX_ERR_STATE; }
  const long n = c->pl.n;
  if (itratn > 1 && !c->d_pulay) {
    TRY(dalloc(c, &c->d_pulay, sizeof(PulayDev)));
    TRY(dalloc(c, &c->d_pu, sizeof(double2) * n * PULAY_MAX));
    TRY(dalloc(c, &c->d_pd, sizeof(double2) * n * PULAY_MAX));
    TRY(dalloc(c, &c->d_ppart, sizeof(double) * SCF_NBLK * PULAY_MAX));
    TRY(dalloc(c, &c->d_adot, sizeof(double) * PULAY_MAX));
    CK(cudaMemsetAsync(c->d_pulay, 0, sizeof(PulayDev), c->st));
  }
  c->itratn = itratn;
  c->cmetric = cmetric;
  c->pulay_reset = true;
  return QX_OK;
}

extern "C" int qx_scf_rho_from_psi(qx_ctx *c) {
  if (!c) return QX_ERR_ARG;
  c->pulay_reset = true;
  TRY(qx_softchg(c));
  CK(cudaMemcpyAsync(c->d_rho_in, c->d_rho_out, sizeof(double) * c->pl.n, cudaMemcpyDeviceToDevice, c->st));
  return QX_OK;
}

// glocal = V_loc + V_H[rho_in] + V_xc[rho_in]; sc[0] = E_H, sc[1..2] = E_xc, int V_xc rho.
static int scf_potential(qx_ctx *c) {
  const long n = c->pl.n;
  real_to_cplx(c->d_rho_in, nullptr, c->d_zg, n, c->st);
  TRY(launch_full_fft<double>(c->pl, c->d_zg, -1, 1.0 / (double)n, c->st));
  hartree_g(c->d_zg, c->d_g2, n, 0.5 * c->rvol, c->d_part, c->d_sc + 0, c->st);
  TRY(launch_full_fft<double>(c->pl, c->d_zg, +1, 1.0, c->st));
  const double rdelv = c->rvol / (double)n;
  if (c->prec == QX_PREC_FP64)
    xc_glocal<double>(c->d_rho_in, c->d_vloc, c->d_zg, n, rdelv, c->d_glocal, c->pl.b64.vloc, c->d_part, c->d_sc + 1,
                      c->st);
  else
    xc_glocal<float>(c->d_rho_in, c->d_vloc, c->d_zg, n, rdelv, c->d_glocal, c->pl.b32.vloc, c->d_part, c->d_sc + 1,
                     c->st);
  CKL();
  c->have_glocal = true;
  return 0;
}

// mxchgg_pulay (chgdns.f90:954-1120): both densities through one complex
// transform, history, coefficients and the new density on the device.
static int scf_mix_pulay(qx_ctx *c) {
  const long n = c->pl.n;
  const double bbb = c->g2max - c->cmetric * c->g2min;
  const double q1 = bbb > 1.0e-5 ? (c->cmetric - 1.0) * c->g2max * c->g2min / bbb : 0.0;
  PulayState p{c->d_pulay, c->d_pu, c->d_pd, c->itratn, q1};
  pulay_push(p, c->pulay_reset ? 1 : 0, c->st);
  c->pulay_reset = false;
  pack2(c->d_rho_in, c->d_rho_out, c->d_zg, n, c->st);
  TRY(launch_full_fft<double>(c->pl, c->d_zg, -1, 1.0 / (double)n, c->st));
  pulay_store(c->d_zg, c->d_g2, c->pl.k1, c->pl.k2, c->pl.k3, p, c->st);
  pulay_coef(c->d_g2, n, p, c->rvol, c->d_ppart, c->d_adot, c->st);
  pulay_new(c->d_g2, n, p, c->mixbeta, c->q02, c->d_zg, c->st);
  TRY(launch_full_fft<double>(c->pl, c->d_zg, +1, 1.0, c->st));
  take_real(c->d_rho_in, c->d_rho_out, c->d_zg, n, c->rvol / (double)n, c->d_part, c->d_sc + 3, c->st);
  CKL();
  return 0;
}

static int scf_mix(qx_ctx *c) {
  if (c->itratn > 1) return scf_mix_pulay(c);
  const long n = c->pl.n;
  real_to_cplx(c->d_rho_out, c->d_rho_in, c->d_zg, n, c->st);
  TRY(launch_full_fft<double>(c->pl, c->d_zg, -1, 1.0 / (double)n, c->st));
  kerker(c->d_zg, c->d_g2, n, c->q02, c->st);
  TRY(launch_full_fft<double>(c->pl, c->d_zg, +1, 1.0, c->st));
  mix(c->d_rho_in, c->d_rho_out, c->d_zg, n, c->mixbeta, c->rvol / (double)n, c->d_part, c->d_sc + 3, c->st);
  CKL();
  return 0;
}

// Records ev on the iteration's stream; under capture as an event-record
// node of the graph, so that each launch of the graph records it.
static int mark_final(qx_ctx *c, cudaEvent_t ev) {
  if (!ev || !c->host_io) return 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(c->st, &cs));
  if (cs == cudaStreamCaptureStatusActive)
    CK(cudaEventRecordWithFlags(ev, c->st, cudaEventRecordExternal));
  else
    CK(cudaEventRecord(ev, c->st));
  return 0;
}

// One SCF iteration in pwlda_md order with every status and summary left on
// the device (c->defer): no host round trip between the first kernel and the
// final read.
// Makes the iteration's stream wait for ev (under capture an event-wait node
// of the graph, so that each launch waits for the event's latest record).
static int wait_mark(qx_ctx *c, cudaEvent_t ev) {
  if (!ev || !c->host_io) return 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(c->st, &cs));
  if (cs == cudaStreamCaptureStatusActive)
    CK(cudaStreamWaitEvent(c->st, ev, cudaEventWaitExternal));
  else
    CK(cudaStreamWaitEvent(c->st, ev, 0));
  return 0;
}

template <typename T>
static int scf_body(qx_ctx *c, const qx_cgparm *p) {
  TRY(scf_potential(c));
  TRY(wait_mark(c, c->ev_psi_in));   // psi from the host, when qx_scf_iteration_host sent one
  TRY(qx_enonloc(c));
  TRY(qx_hmatrix(c, nullptr));
  TRY(gradres_impl<T>(c, nullptr, nullptr, nullptr));
  TRY(untryt_impl<T>(c, nullptr, nullptr));
  TRY(qx_untryhc(c));
  band_energy(c->d_w, c->d_occ, c->nb, c->d_sc + 4, c->st);
  CKL();
  TRY(qx_eigen(c, p, nullptr, nullptr));
  TRY(qx_schmidt(c));
  TRY(mark_final(c, c->ev_psi_final));   // psi final: the read-back may start
  TRY(qx_softchg(c));
  TRY(mark_final(c, c->ev_rho_final));   // rho_out final
  TRY(scf_mix(c));
  return 0;
}

// QX_GRAPH=0 runs the same sync-free iteration as plain stream launches.
static bool scf_graphs_enabled() {
  const char *e = getenv("QX_GRAPH");
  return !(e && e[0] == '0');
}

// The iteration as a CUDA graph: captured once per arrangement of the
// rotating psi/hpsi/tmp buffers (two alternate), mixing restart flag and CG
// parameters, then replayed.  The one-rank CG order launches its own graph
// and runs outside this one.
template <typename T>
static int scf_graph_launch(qx_ctx *c, const qx_cgparm *p) {
  const void *keyp[] = {c->psi, c->hpsi, c->tmp};
  const int keyi[] = {c->pulay_reset ? 1 : 0, c->itratn, c->nlmode, c->host_io ? 1 : 0};
  std::vector<char> key(sizeof(keyp) + sizeof(keyi) + sizeof(qx_cgparm));
  memcpy(key.data(), keyp, sizeof(keyp));
  memcpy(key.data() + sizeof(keyp), keyi, sizeof(keyi));
  memcpy(key.data() + sizeof(keyp) + sizeof(keyi), p, sizeof(qx_cgparm));
  qx_ctx::ScfGraph *g = nullptr;
  for (auto &e : c->scf_graphs)
    if (e.key == key) g = &e;
  if (!g) {
    if (c->scf_graphs.size() >= 4) {
      for (auto &e : c->scf_graphs) cudaGraphExecDestroy(e.exec);
      c->scf_graphs.clear();
    }
    if (!c->cap_st) CK(cudaStreamCreateWithFlags(&c->cap_st, cudaStreamNonBlocking));
    // the capture runs the host side of the iteration (pointer rotation,
    // flags) without executing anything; the graph then does the work
    void *psi0 = c->psi, *hpsi0 = c->hpsi, *tmp0 = c->tmp;
    const bool reset0 = c->pulay_reset;
    CK(cudaStreamBeginCapture(c->cap_st, cudaStreamCaptureModeThreadLocal));
    cudaStream_t user = c->st;
    c->st = c->cap_st;
    const long l0 = g_launches.load(), f0 = fp32_gemm_fallbacks();
    const int r = scf_body<T>(c, p);
    const long nl = g_launches.load() - l0, nf = fp32_gemm_fallbacks() - f0;
    g_launches.fetch_sub(nl);
    fp32_gemm_fallbacks_add(-nf);
    c->st = user;
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c->cap_st, &graph);
    if (r || ec != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      c->psi = psi0; c->hpsi = hpsi0; c->tmp = tmp0; c->pulay_reset = reset0;
      if (!r) set_error("qx_scf_iteration: graph capture failed: %s", cudaGetErrorString(ec));
      return r ? r : QX_ERR_CUDA;
    }
    qx_ctx::ScfGraph e;
    e.key = key;
    e.psi = c->psi; e.hpsi = c->hpsi; e.tmp = c->tmp;
    e.launches = nl;
    e.fallbacks = nf;
    const cudaError_t ei = cudaGraphInstantiate(&e.exec, graph, 0);
    cudaGraphDestroy(graph);
    c->psi = psi0; c->hpsi = hpsi0; c->tmp = tmp0;
    if (ei != cudaSuccess) {
      c->pulay_reset = reset0;
      set_error("qx_scf_iteration: graph instantiation failed: %s", cudaGetErrorString(ei));
      return QX_ERR_CUDA;
    }
    c->scf_graphs.push_back(e);
    g = &c->scf_graphs.back();
  }
  CK(cudaGraphLaunch(g->exec, c->st));
  g_launches.fetch_add(g->launches);
  fp32_gemm_fallbacks_add(g->fallbacks);
  c->psi = g->psi; c->hpsi = g->hpsi; c->tmp = g->tmp;
  c->pulay_reset = false;
  c->have_glocal = true;
  c->have_u = true;
  c->have_hsub = false;
  return 0;
}

extern "C" int qx_scf_launch(qx_ctx *c, const qx_cgparm *p) {
  if (!c || !p) return QX_ERR_ARG;
  if (!c->scf_ready || !c->have_occ) { set_error("qx_scf_iteration: call qx_scf_init and qx_set_occ first"); return QX_ERR_STATE; }
  c->defer = true;
  int r;
  if (scf_graphs_enabled() && !p->sequential)
    r = c->prec == QX_PREC_FP64 ? scf_graph_launch<double>(c, p) : scf_graph_launch<float>(c, p);
  else
    r = c->prec == QX_PREC_FP64 ? scf_body<double>(c, p) : scf_body<float>(c, p);
  c->defer = false;
  return r;
}

extern "C" int qx_scf_result(qx_ctx *c, qx_scf_out *out) {
  if (!c) return QX_ERR_ARG;
  double sc[7];
  int info[3];
  CK(cudaMemcpyAsync(sc, c->d_sc, sizeof(double) * 7, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(info, c->d_info, sizeof(int) * 3, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (info[0] <= 0) { set_error("untryt: eigen-decomposition produced no eigenvectors"); return QX_ERR_EIG; }
  if (info[1] < 0) { set_error("schmidt: a grid barrier of the Cholesky kernel timed out"); return QX_ERR_CUDA; }
  if (info[1]) { set_error("schmidt: <psi|psi> not positive definite at band %d", info[1] - 1); return QX_ERR_NOTPD; }
  if (out) {
    out->ehartree = sc[0];
    out->exc = sc[1];
    out->evxc = sc[2];
    out->resid = sc[3];
    out->eband = sc[4];
    out->etot = sc[4] - sc[0] + sc[1] - sc[2] + c->eion;
    out->zmax = sc[5];
    out->ncg_hpsi = info[2];
    out->eig_clusters = info[0];
  }
  return QX_OK;
}

extern "C" int qx_scf_iteration(qx_ctx *c, const qx_cgparm *p, qx_scf_out *out) {
  TRY(qx_scf_launch(c, p));
  return qx_scf_result(c, out);
}

extern "C" int qx_scf_iteration_host(qx_ctx *c, const qx_cgparm *p, qx_scf_out *out, const double *psi_in,
                                     double *psi_out, double *rho_out, double *eig_out) {
  if (!c || !p) return QX_ERR_ARG;
  c->host_io = true;   // the iteration records and waits for the I/O events from now on
  const long n = (long)c->nb * c->ne;
  if ((psi_out || psi_in) && c->prec != QX_PREC_FP64 && c->io_len < n) {   // sized before the launch
    TRY(dregrow(c, &c->d_io, sizeof(double) * n));
    c->io_len = n;
  }
  if (rho_out && !c->d_rho_out) { set_error("qx_scf_iteration_host: no density (qx_scf_init)"); return QX_ERR_STATE; }
  if (psi_in) {
    // upload on io_st while the iteration builds the potential, which does
    // not read psi; the iteration waits for ev_psi_in before H|psi>.  io_st
    // first waits for everything already on the context's stream (psi's
    // previous readers).
    CK(cudaEventRecord(c->ev_psi_in, c->st));
    CK(cudaStreamWaitEvent(c->io_st, c->ev_psi_in, 0));
    if (c->prec == QX_PREC_FP64) {
      CK(cudaMemcpyAsync(c->psi, psi_in, sizeof(double) * n, cudaMemcpyHostToDevice, c->io_st));
    } else {
      CK(cudaMemcpyAsync(c->d_io, psi_in, sizeof(double) * n, cudaMemcpyHostToDevice, c->io_st));
      convert<double, float>(c->d_io, (float *)c->psi, n, c->io_st);
      CKL();
    }
    CK(cudaEventRecord(c->ev_psi_in, c->io_st));
  }
  TRY(qx_scf_launch(c, p));
  if (psi_out) {
    CK(cudaStreamWaitEvent(c->io_st, c->ev_psi_final, 0));
    if (c->prec == QX_PREC_FP64) {
      CK(cudaMemcpyAsync(psi_out, c->psi, sizeof(double) * n, cudaMemcpyDeviceToHost, c->io_st));
    } else {
      convert<float, double>((const float *)c->psi, c->d_io, n, c->io_st);
      CKL();
      CK(cudaMemcpyAsync(psi_out, c->d_io, sizeof(double) * n, cudaMemcpyDeviceToHost, c->io_st));
    }
  }
  if (rho_out) {
    CK(cudaStreamWaitEvent(c->io_st, c->ev_rho_final, 0));
    CK(cudaMemcpyAsync(rho_out, c->d_rho_out, sizeof(double) * c->pl.n, cudaMemcpyDeviceToHost, c->io_st));
  }
  if (eig_out) CK(cudaMemcpyAsync(eig_out, c->d_eig, sizeof(double) * c->nb, cudaMemcpyDeviceToHost, c->st));
  const int r = qx_scf_result(c, out);
  const cudaError_t e = cudaStreamSynchronize(c->io_st);
  if (r) return r;
  if (e != cudaSuccess) { set_error("qx_scf_iteration_host: read-back: %s", cudaGetErrorString(e)); return QX_ERR_CUDA; }
  return QX_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: times the candidates of this context's launch choices on its own
// buffers (outputs into scratch) and keeps the fastest:
//  * the K-split factor of each tensor-core contraction shape (process-wide);
//  * the fused plane kernels against the generic y/x passes of the FP32 FFT
//    pipeline (per context).
// Reads psi/hpsi and overwrites only scratch (tmp, mat_t, proj); previously
// captured SCF graphs are dropped so the next iteration is captured with the
// new choices.
static int time_ms(cudaStream_t st, const std::function<int()> &f, int reps, float *ms) {
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  TRY(f());   // warm-up
  CK(cudaEventRecord(e0, st));
  for (int r = 0; r < reps; ++r) TRY(f());
  CK(cudaEventRecord(e1, st));
  CK(cudaEventSynchronize(e1));
  CK(cudaEventElapsedTime(ms, e0, e1));
  *ms /= reps;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return 0;
}

// Applies the radix plans L[0..2] of the three grid lengths and rebuilds what
// depends on them: the table offsets, the stage output bases and the
// twiddles of every precision the context holds (the old tables are freed
// and captured graphs dropped).  QX_ERR_ARG, with nothing changed, when the
// plans' shared-memory tiles would exceed 227 KB.
static int replan_fft(qx_ctx *c, const FftLen L[3]) {
  Plan &pl = c->pl;
  Plan trial = pl;
  for (int d = 0; d < 3; ++d) trial.L[d] = L[d];
  const size_t need64 = fft_smem_need<double>(trial), need32 = fft_smem_need<float>(trial);
  if (need64 > 227 * 1024 || (c->prec == QX_PREC_MIXED && need32 > 227 * 1024)) return QX_ERR_ARG;
  CK(cudaStreamSynchronize(c->st));
  if (c->st2) CK(cudaStreamSynchronize(c->st2));
  for (int d = 0; d < 3; ++d) pl.L[d] = L[d];
  pl.stw_off[0] = 0; pl.stw_off[1] = pl.L[0].nst; pl.stw_off[2] = pl.L[0].nst + pl.L[1].nst;
  pl.sob_off[0] = 0; pl.sob_off[1] = pl.L[0].nob; pl.sob_off[2] = pl.L[0].nob + pl.L[1].nob;
  std::vector<int> sob;
  for (int d = 0; d < 3; ++d) stage_bases(pl.L[d], sob);
  TRY(dregrow(c, &pl.d_sob, sizeof(int) * std::max<size_t>(sob.size(), 1)));
  if (!sob.empty()) CK(cudaMemcpy(pl.d_sob, sob.data(), sizeof(int) * sob.size(), cudaMemcpyHostToDevice));
  if (c->prec == QX_PREC_MIXED) {
    TRY(upload_tw<float>(c));
    set_fft_smem_limits<float>(need32);
  }
  TRY(upload_tw<double>(c));
  set_fft_smem_limits<double>(need64);
  drop_scf_graphs(c);
  if (c->seq_exec) { cudaGraphExecDestroy(c->seq_exec); c->seq_exec = nullptr; }
  if (c->seq_graph) { cudaGraphDestroy(c->seq_graph); c->seq_graph = nullptr; }
  CKL();
  return QX_OK;
}

static std::string plan_str(const FftLen &L) {
  std::string s;
  for (int i = 0; i < L.nstage; ++i) s += (i ? "x" : "") + std::to_string(L.radix[i]);
  return s;
}

extern "C" int qx_autotune(qx_ctx *c, char *report, int report_len) {
  if (!c) return QX_ERR_ARG;
  std::string rep;
  char buf[256];
  const int nb = c->nb, ne = c->ne, np = c->pl.nproj;
  // FFT radix plans of the shared-memory stage kernels: for each distinct
  // grid length, every ordered factorisation into radices 2..9 of at most
  // four stages (fewest stages first, at most 16), timed on one H|psi> pass
  // of this context plus an FP64 full-grid transform pair (the density side),
  // the other lengths held at their current plans
  if (c->have_glocal) {
    auto measure = [&](float *ms) -> int {
      float m1 = 0.f, m2 = 0.f;
      TRY(time_ms(c->st, [&]() { return qx_hpsi(c, c->psi, c->tmp, nb, QX_HPSI_KINETIC); }, 3, &m1));
      if (c->d_zg)
        TRY(time_ms(c->st, [&]() {
          TRY(launch_full_fft<double>(c->pl, c->d_zg, -1, 1.0, c->st));
          return launch_full_fft<double>(c->pl, c->d_zg, +1, 1.0, c->st);
        }, 3, &m2));
      *ms = m1 + m2;
      return 0;
    };
    const int lens[3] = {c->pl.k1, c->pl.k2, c->pl.k3};
    bool done_len[3] = {false, false, false};
    for (int d = 0; d < 3; ++d) {
      if (done_len[d]) continue;
      const int n = lens[d];
      std::vector<std::vector<int>> cands;
      std::vector<int> cur;
      radix_plans(n, 4, cands, cur);
      std::stable_sort(cands.begin(), cands.end(),
                       [](const std::vector<int> &x, const std::vector<int> &y) { return x.size() < y.size(); });
      if (cands.size() > 16) cands.resize(16);
      FftLen best[3] = {c->pl.L[0], c->pl.L[1], c->pl.L[2]};
      float tbest = 0.f;
      TRY(measure(&tbest));
      const float tdef = tbest;
      for (const auto &cd : cands) {
        FftLen L[3] = {c->pl.L[0], c->pl.L[1], c->pl.L[2]};
        bool ok = true;
        for (int e = 0; e < 3; ++e)
          if (lens[e] == n) ok = ok && plan_len(n, cd.data(), (int)cd.size(), L[e]);
        if (!ok || replan_fft(c, L) != QX_OK) continue;
        float t = 0.f;
        TRY(measure(&t));
        if (t < tbest) {
          tbest = t;
          for (int e = 0; e < 3; ++e) best[e] = L[e];
        }
      }
      TRY(replan_fft(c, best));
      for (int e = 0; e < 3; ++e)
        if (lens[e] == n) done_len[e] = true;
      snprintf(buf, sizeof(buf), "FFT length %d: %zu plans, %s (%.1f us; default %.1f us); ", n, cands.size() + 1,
               plan_str(best[d]).c_str(), tbest * 1e3, tdef * 1e3);
      rep += buf;
    }
  }
  if (c->prec == QX_PREC_MIXED && tc_enabled()) {
    struct Shape { bool ta, tb; int M, N, K, gamma; const void *A; long lda; const void *B; long ldb; float beta; long ldc; const char *what; };
    std::vector<Shape> shapes = {
        {true, false, nb, nb, ne, 1, c->psi, ne, c->hpsi, ne, 0.f, nb, "C^T X"},
        {false, false, ne, nb, nb, 0, c->psi, ne, c->mat_t, nb, 0.f, ne, "C U"},
    };
    if (c->have_kbg && np > 0) {
      shapes.push_back({true, false, np, nb, ne, 2, c->pl.b32.kbg, ne, c->psi, ne, 0.f, np, "K^T C"});
      shapes.push_back({false, false, ne, nb, np, 0, c->pl.b32.kbg, ne, c->proj, np, 1.f, ne, "K P"});
    }
    // tile width x K split per contraction shape
    const int cand[] = {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48};
    const int tiles[] = {64, 80, 96, 128};
    for (const Shape &sh : shapes) {
      const int nkb = (sh.K + 31) / 32;
      float best = 1e30f;
      int bests = 1, bestt = 0;
      for (int bn : tiles) {
        if (!tc_tile_valid(sh.tb, bn)) continue;
        for (int ns : cand) {
          if (ns > nkb || (size_t)ns * sh.M * sh.N * sizeof(float) > c->gws_bytes) continue;
          float ms = 0.f;
          tc_split_force = ns;
          tc_tile_force = bn;
          const int r = time_ms(c->st, [&]() {
            return gemm<float>(sh.ta, sh.tb, sh.M, sh.N, sh.K, 1.f, (const float *)sh.A, sh.lda, (const float *)sh.B,
                               sh.ldb, sh.beta, (float *)c->tmp, sh.ldc, sh.gamma, nullptr, nullptr, c->st, c->gws,
                               c->gws_bytes, nullptr, c->tcpad, c->tcpad_bytes);
          }, 3, &ms);
          tc_split_force = 0;
          tc_tile_force = 0;
          TRY(r);
          if (ms < best) { best = ms; bests = ns; bestt = bn; }
        }
      }
      tc_split_store(sh.ta, sh.tb, sh.M, sh.N, sh.K, sh.gamma, bests, bestt);
      snprintf(buf, sizeof(buf), "%s %dx%dx%d: tile %d, K split %d (%.1f us); ", sh.what, sh.M, sh.N, sh.K, bestt,
               bests, best * 1e3);
      rep += buf;
    }
  }
  if (c->prec == QX_PREC_MIXED && c->have_glocal && plane_length_supported(c->pl.k1, c->pl.k2)) {
    float ms[2] = {0.f, 0.f};
    for (int v = 0; v < 2; ++v) {
      c->pl.use_plane = (v == 0);
      TRY(time_ms(c->st, [&]() { return qx_hpsi(c, c->psi, c->tmp, nb, QX_HPSI_KINETIC); }, 3, &ms[v]));
    }
    c->pl.use_plane = ms[0] <= ms[1];
    snprintf(buf, sizeof(buf), "H|psi> pass: fused planes %.1f us, y/x passes %.1f us -> %s", ms[0] * 1e3,
             ms[1] * 1e3, c->pl.use_plane ? "fused planes" : "y/x passes");
    rep += buf;
  }
  for (auto &g : c->scf_graphs) cudaGraphExecDestroy(g.exec);
  c->scf_graphs.clear();
  if (report && report_len > 0) {
    strncpy(report, rep.c_str(), report_len - 1);
    report[report_len - 1] = 0;
  }
  return QX_OK;
}

// ---------------------------------------------------------------------------
// FP64 refinement sweep: an FP64 context of the same cell takes over the
// converged state of a mixed-precision one on the device (psi widened to
// FP64, rho_out as the next input density, the Pulay history restarted); the
// caller then runs a few FP64 SCF iterations on it.
extern "C" int qx_refine_from(qx_ctx *dst, qx_ctx *src) {
  if (!dst || !src) return QX_ERR_ARG;
  if (dst->prec != QX_PREC_FP64 || src->nb != dst->nb || src->ne != dst->ne || src->pl.n != dst->pl.n) {
    set_error("qx_refine_from: needs an FP64 context of the same cell (bands, sphere, grid)");
    return QX_ERR_ARG;
  }
  if (!dst->scf_ready || !src->d_rho_out) { set_error("qx_refine_from: call qx_scf_init on both contexts first"); return QX_ERR_STATE; }
  TRY(ensure_rho(dst));
  // src's work must be complete before dst's stream reads its buffers
  CK(cudaStreamSynchronize(src->st));
  const long n = (long)dst->nb * dst->ne;
  if (src->prec == QX_PREC_FP64)
    CK(cudaMemcpyAsync(dst->psi, src->psi, sizeof(double) * n, cudaMemcpyDeviceToDevice, dst->st));
  else
    convert<float, double>((const float *)src->psi, (double *)dst->psi, n, dst->st);
  CK(cudaMemcpyAsync(dst->d_rho_in, src->d_rho_out, sizeof(double) * dst->pl.n, cudaMemcpyDeviceToDevice, dst->st));
  CKL();
  dst->pulay_reset = true;
  dst->have_u = false;
  dst->have_hsub = false;
  return QX_OK;
}

// ---------------------------------------------------------------------------
// TDDFT-FSSH overlaps (tddft_fssh_cal_matrix, tddft_fssh.f90:1344-1414)
extern "C" int qx_tddft_store(qx_ctx *c) {
  if (!c) return QX_ERR_ARG;
  const size_t bytes = c->tsize() * (size_t)c->nb * c->ne;
  if (!c->prev) TRY(dalloc(c, &c->prev, bytes));
  CK(cudaMemcpyAsync(c->prev, c->psi, bytes, cudaMemcpyDeviceToDevice, c->st));
  c->have_prev = true;
  return QX_OK;
}

template <typename T>
static int tddft_overlap_impl(qx_ctx *c, double *aij) {
  const int nb = c->nb;
  T *m = (T *)c->mat_t;
  // m(i, j) = <prev_i | psi_j> (column-major), Gamma metric: aijr(i, j) of the reference
  TRY(gemm<T>(true, false, nb, nb, c->ne, (T)1, (const T *)c->prev, c->ne, (const T *)c->psi, c->ne, (T)0, m, nb, 1,
              nullptr, nullptr, c->st, c->gws, c->gws_bytes, nullptr, c->tcpad, c->tcpad_bytes));
  convert<T, double>(m, c->d_mat, (long)nb * nb, c->st);
  CKL();
  if (aij) {
    CK(cudaMemcpyAsync(aij, c->d_mat, sizeof(double) * nb * nb, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  return 0;
}

extern "C" int qx_tddft_overlap(qx_ctx *c, double *aij) {
  if (!c) return QX_ERR_ARG;
  if (!c->have_prev) { set_error("qx_tddft_overlap: call qx_tddft_store at the previous step first"); return QX_ERR_STATE; }
  return c->prec == QX_PREC_FP64 ? tddft_overlap_impl<double>(c, aij) : tddft_overlap_impl<float>(c, aij);
}

// ---------------------------------------------------------------------------
// Local pseudopotential of the current geometry (vlocal_g, nlkbpp.f90:862-1036)
extern "C" int qx_build_vloc(qx_ctx *c) {
  if (!c) return QX_ERR_ARG;
  if (!c->have_ftab || !c->scf_ready || !c->have_occ) {
    set_error("qx_build_vloc: call qx_set_occ, qx_scf_init and qx_set_force_tables first");
    return QX_ERR_STATE;
  }
  const long n = c->pl.n;
  CK(cudaMemsetAsync(c->d_zg, 0, sizeof(double2) * n, c->st));
  vloc_g(c->f_n5, c->f_natom, c->d_ijk5, c->d_ngabc, c->d_svco, c->d_ityp, c->d_dcq, c->d_dsq, c->f_km[0],
         c->f_km[1], c->f_km[2], c->f_ktot, c->rvol, c->pl.k1, c->pl.k2, c->pl.k3, c->d_zg, c->st);
  CKL();
  TRY(launch_full_fft<double>(c->pl, c->d_zg, +1, 1.0, c->st));
  real_part(c->d_zg, c->d_vloc, n, c->st);
  CKL();
  return QX_OK;
}

// ---------------------------------------------------------------------------
// TDDFT-FSSH surface hopping (tddft_fssh_dm, tddft_fssh.f90:1989-2402)
namespace qx {
void fssh_init(int nst, double *dnr, double *dni, double *accum, cudaStream_t st);
void fssh_step(int nst, const double *A, const double *eig, double dtmd, double dttddft, int boltz, double treq,
               int hop, double *dnr, double *dni, const double *occ_store, double *occ_rec, double *probinteg,
               double *accum, double *rndx, double *bkl, int *trans, cudaStream_t st);
}  // namespace qx

extern "C" int qx_fssh_init(qx_ctx *c, const qx_fssh_parm *p, const double *occ) {
  if (!c || !p || !occ) { set_error("qx_fssh_init: bad arguments"); return QX_ERR_ARG; }
  const int nst = p->nstate;
  if (nst < 2 || nst > QX_FSSH_MAX_STATES || p->b0 < 0 || p->b0 + nst > c->nb) {
    set_error("qx_fssh_init: window b0 = %d, nstate = %d outside 2..%d states within %d bands", p->b0, nst,
              QX_FSSH_MAX_STATES, c->nb);
    return QX_ERR_ARG;
  }
  if (!(p->dtmd > 0.0) || !(p->dttddft > 0.0) || p->dtmd / p->dttddft > 1.0e7 ||
      (p->boltzmann && !(p->treq > 0.0)) || !(p->seed > 0.0) || !(p->seed < 2147483647.0)) {
    set_error("qx_fssh_init: need dtmd, dttddft > 0 with dtmd/dttddft <= 1e7, treq > 0 with the Boltzmann factor, "
              "0 < seed < 2147483647");
    return QX_ERR_ARG;
  }
  if (nst > c->fs_cap) {
    TRY(dregrow(c, &c->d_fs_dnr, sizeof(double) * 49 * (size_t)nst));
    TRY(dregrow(c, &c->d_fs_dni, sizeof(double) * 49 * (size_t)nst));
    TRY(dregrow(c, &c->d_fs_pint, sizeof(double) * 7 * (size_t)nst));
    TRY(dregrow(c, &c->d_fs_bkl, sizeof(double) * 7 * (size_t)nst));
    TRY(dregrow(c, &c->d_fs_accum, sizeof(double) * (size_t)nst * nst));
    TRY(dregrow(c, &c->d_fs_occ, sizeof(double) * (size_t)nst));
    TRY(dregrow(c, &c->d_fs_occ0, sizeof(double) * (size_t)nst));
    TRY(dregrow(c, &c->d_fs_A, sizeof(double) * (size_t)nst * nst));
    TRY(dregrow(c, &c->d_fs_eig, sizeof(double) * (size_t)nst));
    if (!c->d_fs_rndx) TRY(dalloc(c, &c->d_fs_rndx, sizeof(double)));
    if (!c->d_fs_trans) TRY(dalloc(c, &c->d_fs_trans, sizeof(int)));
    c->fs_cap = nst;
  }
  c->fs = *p;
  fssh_init(nst, c->d_fs_dnr, c->d_fs_dni, c->d_fs_accum, c->st);
  CKL();
  CK(cudaMemcpyAsync(c->d_fs_occ, occ, sizeof(double) * nst, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_fs_rndx, &p->seed, sizeof(double), cudaMemcpyHostToDevice, c->st));
  TRY(qx_tddft_store(c));
  CK(cudaStreamSynchronize(c->st));
  c->have_fssh = true;
  return QX_OK;
}

template <typename T>
static int fssh_overlap(qx_ctx *c) {
  const int nst = c->fs.nstate, b0 = c->fs.b0;
  T *m = (T *)c->mat_t;
  // A(k, j) = <prev_(b0+k)|psi_(b0+j)> with the Gamma metric (tddft_fssh_cal_matrix)
  const T *pv = (const T *)c->prev + (size_t)b0 * c->ne, *ps = (const T *)c->psi + (size_t)b0 * c->ne;
  TRY(gemm<T>(true, false, nst, nst, c->ne, (T)1, pv, c->ne, ps, c->ne, (T)0, m, nst, 1, nullptr, nullptr, c->st,
              c->gws, c->gws_bytes, nullptr, c->tcpad, c->tcpad_bytes));
  convert<T, double>(m, c->d_fs_A, (long)nst * nst, c->st);
  CKL();
  return 0;
}

extern "C" int qx_fssh_step(qx_ctx *c, const double *phis, const double *eig, double *occ, int *transition,
                            double *bkl) {
  if (!c) return QX_ERR_ARG;
  if (!c->have_fssh) { set_error("qx_fssh_step: qx_fssh_init first"); return QX_ERR_STATE; }
  const qx_fssh_parm &p = c->fs;
  const int nst = p.nstate;
  if (phis) {
    CK(cudaMemcpyAsync(c->d_fs_A, phis, sizeof(double) * (size_t)nst * nst, cudaMemcpyHostToDevice, c->st));
  } else {
    TRY(c->prec == QX_PREC_FP64 ? fssh_overlap<double>(c) : fssh_overlap<float>(c));
    TRY(qx_tddft_store(c));   // psi(t + dt) becomes the previous step's
  }
  if (eig) CK(cudaMemcpyAsync(c->d_fs_eig, eig, sizeof(double) * nst, cudaMemcpyHostToDevice, c->st));
  else CK(cudaMemcpyAsync(c->d_fs_eig, c->d_eig + p.b0, sizeof(double) * nst, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_fs_occ0, c->d_fs_occ, sizeof(double) * nst, cudaMemcpyDeviceToDevice, c->st));
  fssh_step(nst, c->d_fs_A, c->d_fs_eig, p.dtmd, p.dttddft, p.boltzmann, p.treq, p.hop, c->d_fs_dnr, c->d_fs_dni,
            c->d_fs_occ0, c->d_fs_occ, c->d_fs_pint, c->d_fs_accum, c->d_fs_rndx, c->d_fs_bkl, c->d_fs_trans, c->st);
  CKL();
  if (occ) CK(cudaMemcpyAsync(occ, c->d_fs_occ, sizeof(double) * nst, cudaMemcpyDeviceToHost, c->st));
  if (transition) CK(cudaMemcpyAsync(transition, c->d_fs_trans, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  if (bkl) CK(cudaMemcpyAsync(bkl, c->d_fs_bkl, sizeof(double) * 7 * (size_t)nst, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return QX_OK;
}

extern "C" int qx_fssh_state(qx_ctx *c, double *dnr, double *dni, double *accum, double *rndx) {
  if (!c) return QX_ERR_ARG;
  if (!c->have_fssh) { set_error("qx_fssh_state: qx_fssh_init first"); return QX_ERR_STATE; }
  const size_t nst = c->fs.nstate;
  if (dnr) CK(cudaMemcpyAsync(dnr, c->d_fs_dnr, sizeof(double) * 49 * nst, cudaMemcpyDeviceToHost, c->st));
  if (dni) CK(cudaMemcpyAsync(dni, c->d_fs_dni, sizeof(double) * 49 * nst, cudaMemcpyDeviceToHost, c->st));
  if (accum) CK(cudaMemcpyAsync(accum, c->d_fs_accum, sizeof(double) * nst * nst, cudaMemcpyDeviceToHost, c->st));
  if (rndx) CK(cudaMemcpyAsync(rndx, c->d_fs_rndx, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return QX_OK;
}

// ---------------------------------------------------------------------------
// Hellmann-Feynman forces
extern "C" int qx_set_force_tables(qx_ctx *c, int natom, int ntype, const int *ityp, const double *satm, int n5,
                                   const int *ijk5, const int *ngabc, const double *gvec5, const double *svco,
                                   const double *gw) {
  if (!c || natom <= 0 || ntype <= 0 || n5 <= 1 || !ityp || !satm || !ijk5 || !ngabc || !gvec5 || !svco || !gw) {
    set_error("qx_set_force_tables: bad arguments");
    return QX_ERR_ARG;
  }
  if (!c->have_kbg || c->pl.nproj % natom) {
    set_error("qx_set_force_tables: G-space KB tables (qx_set_kb_g) with nproj a multiple of natom are needed");
    return QX_ERR_STATE;
  }
  for (int a = 0; a < natom; ++a)
    if (ityp[a] < 0 || ityp[a] >= ntype) { set_error("qx_set_force_tables: ityp out of range"); return QX_ERR_ARG; }
  for (long i = 0; i < n5; ++i)
    if (ijk5[i] < 0 || ijk5[i] >= c->pl.n) { set_error("qx_set_force_tables: ijk5 out of range"); return QX_ERR_ARG; }
  int km[3] = {0, 0, 0};
  for (long i = 0; i < 3L * n5; ++i) km[i % 3] = std::max(km[i % 3], std::abs(ngabc[i]));
  const int ktot = 2 * (km[0] + km[1] + km[2]) + 3;
  const int np = c->pl.nproj, ne = c->ne, nb = c->nb;
  const size_t ts = c->tsize();
  if (c->f_natom != natom || c->f_n5 != n5 || c->f_ntype != ntype || c->f_ktot != ktot || !c->d_force) {
    TRY(dalloc(c, &c->d_ityp, sizeof(int) * natom));
    TRY(dalloc(c, &c->d_satm, sizeof(double) * 3 * natom));
    TRY(dalloc(c, &c->d_ijk5, sizeof(int) * n5));
    TRY(dalloc(c, &c->d_ngabc, sizeof(int) * 3 * (size_t)n5));
    TRY(dalloc(c, &c->d_gvec5, sizeof(double) * 3 * (size_t)n5));
    TRY(dalloc(c, &c->d_svco, sizeof(double) * (size_t)n5 * ntype));
    TRY(dalloc(c, &c->d_dcq, sizeof(double) * (size_t)natom * ktot));
    TRY(dalloc(c, &c->d_dsq, sizeof(double) * (size_t)natom * ktot));
    TRY(dalloc(c, &c->d_force, sizeof(double) * 6 * natom));
  }
  if (!c->d_gw) TRY(dalloc(c, &c->d_gw, sizeof(double) * 3 * (size_t)(ne / 2)));
  if (!c->dtab) {
    TRY(dalloc(c, &c->dtab, ts * 3 * (size_t)np * ne));
    TRY(dalloc(c, &c->dproj, ts * 3 * (size_t)np * nb));
  }
  if (!c->d_zg) TRY(dalloc(c, &c->d_zg, sizeof(double2) * c->pl.n));
  TRY(ensure_rho(c));
  CK(cudaMemcpyAsync(c->d_ityp, ityp, sizeof(int) * natom, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_satm, satm, sizeof(double) * 3 * natom, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_ijk5, ijk5, sizeof(int) * n5, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_ngabc, ngabc, sizeof(int) * 3 * (size_t)n5, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_gvec5, gvec5, sizeof(double) * 3 * (size_t)n5, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_svco, svco, sizeof(double) * (size_t)n5 * ntype, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_gw, gw, sizeof(double) * 3 * (size_t)(ne / 2), cudaMemcpyHostToDevice, c->st));
  // the host arrays may go away when this returns
  CK(cudaStreamSynchronize(c->st));
  c->f_natom = natom;
  c->f_ntype = ntype;
  c->f_n5 = n5;
  c->f_ktot = ktot;
  c->f_nproj = np;
  for (int d = 0; d < 3; ++d) c->f_km[d] = km[d];
  phase_tables(natom, c->d_satm, km[0], km[1], km[2], ktot, c->d_dcq, c->d_dsq, c->st);
  if (c->prec == QX_PREC_FP64)
    dtab_build<double>(np, ne / 2 - 1, c->pl.b64.kbg, c->d_gw, (double *)c->dtab, c->st);
  else
    dtab_build<float>(np, ne / 2 - 1, c->pl.b32.kbg, c->d_gw, (float *)c->dtab, c->st);
  CKL();
  c->have_ftab = true;
  return QX_OK;
}

template <typename T>
static int forces_impl(qx_ctx *c, double *floc, double *fnl) {
  const int natom = c->f_natom, np = c->pl.nproj, ne = c->ne, nb = c->nb;
  const long n = c->pl.n;
  TRY(qx_softchg(c));   // rho of the current psi
  real_to_cplx(c->d_rho_out, nullptr, c->d_zg, n, c->st);
  TRY(launch_full_fft<double>(c->pl, c->d_zg, -1, 1.0 / (double)n, c->st));
  floc_g(natom, c->f_n5, c->d_ijk5, c->d_ngabc, c->d_gvec5, c->d_svco, c->d_ityp, c->d_zg, c->d_dcq, c->d_dsq,
         c->f_km[0], c->f_km[1], c->f_km[2], c->f_ktot, c->d_force, c->st);
  CKL();
  const Bufs<T> &b = c->pl.bufs<T>();
  T *P = (T *)c->proj, *D = (T *)c->dproj;
  long kld = 0;
  const T *kb = kbg_operand<T>(c, &kld);
  TRY(gemm<T>(true, false, np, nb, ne, (T)1, kb, kld, (const T *)c->psi, ne, (T)0, P, np, 2, nullptr, nullptr,
              c->st, c->gws, c->gws_bytes, nullptr, c->tcpad, c->tcpad_bytes));
  TRY(gemm<T>(true, false, 3 * np, nb, ne, (T)1, (const T *)c->dtab, ne, (const T *)c->psi, ne, (T)0, D, 3 * np, 0,
              nullptr, nullptr, c->st, c->gws, c->gws_bytes, nullptr, c->tcpad, c->tcpad_bytes));
  fnl_reduce<T>(natom, np / natom, np, nb, P, D, b.vclalp, c->d_occ, c->d_force + 3 * natom, c->st);
  CKL();
  std::vector<double> f(6 * (size_t)natom);
  CK(cudaMemcpyAsync(f.data(), c->d_force, sizeof(double) * 6 * natom, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (floc) memcpy(floc, f.data(), sizeof(double) * 3 * natom);
  if (fnl) memcpy(fnl, f.data() + 3 * natom, sizeof(double) * 3 * natom);
  return 0;
}

extern "C" int qx_forces(qx_ctx *c, double *floc, double *fnl) {
  if (!c) return QX_ERR_ARG;
  if (!c->have_ftab || !c->have_occ) { set_error("qx_forces: call qx_set_force_tables and qx_set_occ first"); return QX_ERR_STATE; }
  return c->prec == QX_PREC_FP64 ? forces_impl<double>(c, floc, fnl) : forces_impl<float>(c, floc, fnl);
}

// Real-space KB forces of the current psi (fnnlcl2, nlkbppr.f90:2024-3120),
// from the tables of qx_build_kb_r with the gradient table given.
template <typename T>
static int fnl_r_impl(qx_ctx *c, double *fnl) {
  const Plan &pl = c->pl;
  const int natom = pl.natom;
  const long need = (long)c->npair_all * natom * 3;
  if (need > c->kbr_fpart_n) {
    TRY(dregrow(c, &c->d_kbr_fpart, sizeof(double) * need));
    TRY(dregrow(c, &c->d_kbr_fout, sizeof(double) * 3 * (size_t)natom));
    c->kbr_fpart_n = need;
  }
  PipeParams P = base_params(c);
  for (int p0 = 0; p0 < c->npair_all; p0 += pl.chunk) {
    P.pair0 = p0;
    const int npl = std::min(pl.chunk, c->npair_all - p0);
    P.npair = p0 + npl;
    TRY(launch_fnl_r_chunk<T>(pl, P, npl, (const T *)c->psi, c->ne, (const T *)c->d_kbr_dvnl, c->d_wocc,
                              c->d_kbr_fpart, c->st));
    CKL();
  }
  fnl_r_sum(c->d_kbr_fpart, c->npair_all, natom, c->d_kbr_fout, c->st);
  CKL();
  CK(cudaMemcpyAsync(fnl, c->d_kbr_fout, sizeof(double) * 3 * natom, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

extern "C" int qx_forces_nl_r(qx_ctx *c, double *fnl) {
  if (!c || !fnl) { set_error("qx_forces_nl_r: null"); return QX_ERR_ARG; }
  if (!c->have_occ) { set_error("qx_forces_nl_r: occupations not set"); return QX_ERR_STATE; }
  if (!c->have_kbr || !c->d_kbr_dvnl || c->pl.d_kb_mesh != c->d_kbr_mesh) {
    set_error("qx_forces_nl_r: real-space tables with gradients (qx_set_kb_r_builder with dtabnl, qx_build_kb_r) needed");
    return QX_ERR_STATE;
  }
  return c->prec == QX_PREC_FP64 ? fnl_r_impl<double>(c, fnl) : fnl_r_impl<float>(c, fnl);
}

extern "C" int qxgpu_fnnlcl2(qx_ctx *c, const double *cgjr, double *fnlc) {
  if (!c || !cgjr || !fnlc) return QX_ERR_ARG;
  TRY(qx_put_psi(c, cgjr));
  std::vector<double> f(3 * (size_t)std::max(c->pl.natom, 1));
  TRY(qx_forces_nl_r(c, f.data()));
  for (int i = 0; i < 3 * c->pl.natom; ++i) fnlc[i] += f[i];
  return QX_OK;
}

extern "C" int qxgpu_kbnlpp_frc2(qx_ctx *c, const double *cgjr, double *fnlc) {
  if (!c || !cgjr || !fnlc) return QX_ERR_ARG;
  if (!c->have_ftab || !c->have_occ) { set_error("qxgpu_kbnlpp_frc2: call qx_set_force_tables and qx_set_occ first"); return QX_ERR_STATE; }
  TRY(qx_put_psi(c, cgjr));
  std::vector<double> fnl(3 * (size_t)c->f_natom);
  TRY(c->prec == QX_PREC_FP64 ? forces_impl<double>(c, nullptr, fnl.data()) : forces_impl<float>(c, nullptr, fnl.data()));
  for (size_t i = 0; i < fnl.size(); ++i) fnlc[i] += fnl[i];
  return QX_OK;
}

// ---------------------------------------------------------------------------
// Drop-in shims on host arrays.
extern "C" int qxgpu_hcnonloc(qx_ctx *c, const double *cgjr, double *rhcr, int nb) {
  if (!c || nb > c->nb) return QX_ERR_ARG;
  TRY(up(c, c->g, cgjr, (long)nb * c->ne));
  TRY(up(c, c->gh, rhcr, (long)nb * c->ne));
  const int save = c->nlmode;
  if (c->nlmode == QX_NL_GSPACE) c->nlmode = QX_NL_NONE;
  int r = qx_hpsi(c, c->g, c->gh, nb, QX_HPSI_ACCUMULATE | QX_HPSI_NONLOCAL);
  c->nlmode = save;
  TRY(r);
  return down(c, rhcr, c->gh, (long)nb * c->ne);
}

template <typename T>
static int kbg_only(qx_ctx *c, const T *cin, T *out, int nb) {
  const Plan &pl = c->pl;
  Bufs<T> &b = pl.bufs<T>();
  const int np = pl.nproj;
  T *proj = (T *)c->proj;
  long kld = 0;
  const T *kb = kbg_operand<T>(c, &kld);
  TRY(gemm<T>(true, false, np, nb, c->ne, (T)1, kb, kld, cin, c->ne, (T)0, proj, np, 2, nullptr, nullptr, c->st, c->gws, c->gws_bytes, nullptr, c->tcpad, c->tcpad_bytes));
  scale_rows<T>(np, nb, proj, np, b.vclalp, nullptr, nullptr, c->st);
  TRY(gemm<T>(false, false, c->ne, nb, np, (T)1, kb, kld, proj, np, (T)1, out, c->ne, 0, nullptr, nullptr, c->st, nullptr, 0, nullptr, c->tcpad, c->tcpad_bytes));
  CKL();
  return 0;
}
extern "C" int qxgpu_hckbpp_g(qx_ctx *c, const double *cgjr, double *rhcr, int nb) {
  if (!c || nb > c->nb || !c->have_kbg) return QX_ERR_ARG;
  TRY(up(c, c->g, cgjr, (long)nb * c->ne));
  TRY(up(c, c->gh, rhcr, (long)nb * c->ne));
  TRY(c->prec == QX_PREC_FP64 ? kbg_only<double>(c, (double *)c->g, (double *)c->gh, nb)
                              : kbg_only<float>(c, (float *)c->g, (float *)c->gh, nb));
  return down(c, rhcr, c->gh, (long)nb * c->ne);
}

extern "C" int qxgpu_enonloc(qx_ctx *c, const double *cgjr, double *rhcr, double *ekib) {
  if (!c) return QX_ERR_ARG;
  TRY(qx_put_psi(c, cgjr));
  TRY(qx_enonloc(c));
  if (ekib) TRY(qx_ekinetic(c, nullptr, ekib));
  return qx_get_hpsi(c, rhcr);
}

extern "C" int qxgpu_eigen(qx_ctx *c, double *gdcr, double *rhcr, const double *ekib, double *eig, const qx_cgparm *p) {
  if (!c || !p) return QX_ERR_ARG;
  TRY(qx_put_psi(c, gdcr));
  TRY(qx_put_hpsi(c, rhcr));
  if (ekib) CK(cudaMemcpyAsync(c->d_ekib, ekib, sizeof(double) * c->nb, cudaMemcpyHostToDevice, c->st));
  else TRY(qx_ekinetic(c, nullptr, nullptr));
  TRY(qx_eigen(c, p, nullptr, nullptr));
  TRY(qx_get_psi(c, gdcr));
  TRY(qx_get_hpsi(c, rhcr));
  if (eig) TRY(qx_get_eig(c, eig));
  return QX_OK;
}

extern "C" int qxgpu_schmidt(qx_ctx *c, double *cgjr) {
  if (!c) return QX_ERR_ARG;
  TRY(qx_put_psi(c, cgjr));
  TRY(qx_schmidt(c));
  return qx_get_psi(c, cgjr);
}

extern "C" int qxgpu_hmatrix(qx_ctx *c, const double *cgjr, const double *rhcr, double *dmtrxr, double *eig) {
  if (!c) return QX_ERR_ARG;
  TRY(qx_put_psi(c, cgjr));
  TRY(qx_put_hpsi(c, rhcr));
  TRY(qx_hmatrix(c, dmtrxr));
  if (eig) TRY(qx_get_eig(c, eig));
  return QX_OK;
}

extern "C" int qxgpu_untryt(qx_ctx *c, double *gdcr, double *rhcr, double *ev) {
  if (!c) return QX_ERR_ARG;
  TRY(qx_put_psi(c, gdcr));
  TRY(qx_put_hpsi(c, rhcr));
  TRY(qx_untryt(c, ev));
  TRY(qx_untryhc(c));
  TRY(qx_get_psi(c, gdcr));
  return qx_get_hpsi(c, rhcr);
}

extern "C" int qxgpu_softchg(qx_ctx *c, const double *cgjr, double *rho) {
  if (!c) return QX_ERR_ARG;
  TRY(qx_put_psi(c, cgjr));
  TRY(qx_softchg(c));
  return qx_get_rho(c, rho);
}

__global__ void k_split(const double2 *z, double *x, double *y, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    x[i] = z[i].x;
    if (y) y[i] = z[i].y;
  }
}
__global__ void k_join(const double *x, const double *y, double2 *z, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    z[i] = make_double2(x[i], y ? y[i] : 0.0);
}

extern "C" int qxgpu_rfft3(qx_ctx *c, int key, double *fft3x, double *fft3y) {
  if (!c || !fft3x || !fft3y) return QX_ERR_ARG;
  const long n = c->pl.n;
  double2 *z = nullptr;
  double *x = nullptr, *y = nullptr;
  CK(cudaMallocAsync((void **)&z, sizeof(double2) * n, c->st));
  CK(cudaMallocAsync((void **)&x, sizeof(double) * n, c->st));
  CK(cudaMallocAsync((void **)&y, sizeof(double) * n, c->st));
  CK(cudaMemcpyAsync(x, fft3x, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  if (key == 1) {
    k_join<<<148 * 4, 256, 0, c->st>>>(x, nullptr, z, n); note_launch();
    TRY(launch_full_fft<double>(c->pl, z, -1, 1.0 / (double)n, c->st));
  } else {
    CK(cudaMemcpyAsync(y, fft3y, sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
    k_join<<<148 * 4, 256, 0, c->st>>>(x, y, z, n); note_launch();
    TRY(launch_full_fft<double>(c->pl, z, +1, 1.0, c->st));
  }
  k_split<<<148 * 4, 256, 0, c->st>>>(z, x, key == 1 ? y : nullptr, n); note_launch();
  CKL();
  CK(cudaMemcpyAsync(fft3x, x, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  if (key == 1) CK(cudaMemcpyAsync(fft3y, y, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaFreeAsync(z, c->st));
  CK(cudaFreeAsync(x, c->st));
  CK(cudaFreeAsync(y, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (key != 1) memset(fft3y, 0, sizeof(double) * n);
  return QX_OK;
}
