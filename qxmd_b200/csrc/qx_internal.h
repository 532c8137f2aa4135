// Internal structures shared by the kernel files and the C-ABI layer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "qx_common.cuh"

// Parameters of one launch of the FFT pipeline (passed by value).
struct PipeParams {
  int k1, k2, k3;
  int m1, m2, P1, P2;
  int nplw;
  FftLen L1, L2, L3;
  const int *row_lo, *row_hi, *row_off;
  const int4 *row_ent;      // {line = a - lo, i3, ig, sign(+1 : +G, -1 : -G)}
  // sphere z-columns (j2, a): col_ja[q] = j2 * P1 + a; col_ig[i3 * ncol + q] =
  // ig + 1 for the +G entry at (a, j2, i3), -(ig + 1) for the -G entry, 0 none
  const int *col_ja;
  const int *col_ig;
  int ncol;
  const int *pairs;         // band indices, 2 per pair, -1 = empty slot
  const int *npair_dev;     // number of valid pairs (device), or null
  int npair;                // pair bound when npair_dev is null
  int pair0;                // first pair of this launch
  double inv_n;             // 1 / kfft0
};

namespace qx {

void set_error(const char *fmt, ...);
// Count of kernels launched by this library (qx_launch_count()).
void note_launch();

// Per-precision device buffers of the FFT pipeline.
template <typename T>
struct Bufs {
  typedef typename c2t<T>::type C;
  C *tw = nullptr;         // base twiddles of the three lengths
  C *stw = nullptr;        // stage twiddles of the three lengths
  C *bufA = nullptr;       // [chunk][k3][P2][P1]
  C *bufB = nullptr;       // [chunk][k3][k2][P1]
  C *bufR = nullptr;       // [chunk][k3][k2][k1] (real-space KB mode)
  C *zsph = nullptr;       // [chunk][nplw+1][2]
  C *sumr = nullptr;       // [chunk][natom][4]
  T *vloc = nullptr;       // glocal(kfft0)
  T *kb_vnl = nullptr;     // real-space projector values [npts][4]
  T *kbg = nullptr;        // G-space projectors [nproj][nplwex]
  T *vclalp = nullptr;     // [nproj]
  double *rho_part = nullptr;   // RHO_GROUPS partial density planes (plane-kernel grids)
};

struct Plan {
  int k1 = 0, k2 = 0, k3 = 0;
  long n = 0;
  int m1 = 0, m2 = 0, m3 = 0, P1 = 0, P2 = 0;
  int nplw = 0, nplwex = 0;
  FftLen L[3];
  int tw_off[3], stw_off[3], sob_off[3];
  int *d_sob = nullptr;    // stage output bases of the three lengths
  int chunk = 0;           // pairs per pipeline launch
  int rholines = 8;
  int xl32 = 32, xl64 = 16; // lines per CTA of the x pass
  // sphere rows
  int *d_row_lo = nullptr, *d_row_hi = nullptr, *d_row_off = nullptr;
  int4 *d_row_ent = nullptr;
  // sphere z-columns (see PipeParams)
  int *d_col_ja = nullptr, *d_col_ig = nullptr;
  int ncol = 0;
  // real-space KB (kb_lmx projectors per point, at most 9: s, p, d)
  int natom = 0, npts = 0, kb_lmx = 4;
  int *d_kb_off = nullptr, *d_kb_mesh = nullptr;
  double *d_kb_clalp = nullptr;
  double rdelv = 0.0;
  int *d_line_off = nullptr;
  int4 *d_line_ent = nullptr;
  // G-space KB
  int nproj = 0;
  bool use_plane = true;   // FP32 fused plane kernels where supported (the autotuner may turn them off)
  mutable Bufs<float> b32;
  mutable Bufs<double> b64;
  template <typename T> Bufs<T> &bufs() const;
  template <typename T> int xlines() const;
};

template <> inline Bufs<float> &Plan::bufs<float>() const { return b32; }
template <> inline Bufs<double> &Plan::bufs<double>() const { return b64; }
template <> inline int Plan::xlines<float>() const { return xl32; }
template <> inline int Plan::xlines<double>() const { return xl64; }

// qx_fft.cu
template <typename T>
int launch_hpsi_chunk(const Plan &pl, const PipeParams &P, int npl, const T *cin, long ldc, T *out, long ldo,
                      const double *dk, int accumulate, int nlmode, cudaStream_t st,
                      cudaEvent_t before_unpack = nullptr);
template <typename T>
int launch_rho_chunk(const Plan &pl, const PipeParams &P, int npl, const T *cin, long ldc, const double *wocc,
                     double *rho, int accumulate, cudaStream_t st);
// real-space KB force partials of a chunk of band pairs (fpart: npair x natom x 3)
template <typename T>
int launch_fnl_r_chunk(const Plan &pl, const PipeParams &P, int npl, const T *cin, long ldc, const T *dvnl,
                       const double *wocc, double *fpart, cudaStream_t st);
void fnl_r_sum(const double *fpart, int npair, int natom, double *fnl, cudaStream_t st);
template <typename T>
int launch_full_fft(const Plan &pl, typename c2t<T>::type *g, int sign, double scale, cudaStream_t st);
// qx_fftfull.cu: one z (axis 2), y (axis 1) or x (axis 0, times scale) pass
// of the FP64 full-grid transform with the lines in registers; -1 when the
// length has no kernel.
int launch_full_lines_f64(double2 *g, int k1, int k2, int k3, int axis, int sign, double scale, cudaStream_t st);
template <typename T> void set_fft_smem_limits(size_t bytes);
// qx_fftplane.cu: fused y-x-y pass (FP32, k1 x k2 planes of a specialised
// shape, QX_PLANE_GRIDS); returns -1 when the grid is not covered.
int launch_plane_f32(const PipeParams &P, int npl, float2 *bufA, const float *vloc, cudaStream_t st);
// Density through the plane kernel: groups of pairs per z plane, partial
// planes in part (RHO_GROUPS * kfft0 doubles) summed in a fixed order.
constexpr int RHO_GROUPS = 16;
int launch_rho_plane_f32(const PipeParams &P, int npl, const float2 *bufA, const double *wocc, double *part,
                         double *rho, int accumulate, cudaStream_t st);
bool plane_length_supported(int k1, int k2);
// Column-wise z transforms (one sphere z-column per thread, FP32, register
// FFTs of length k3); -1 when k3 has no specialised length.
int launch_zcols_inv_f32(const PipeParams &P, int npl, const float *cin, long ldc, float2 *bufA, cudaStream_t st);
int launch_zcols_fwd_f32(const PipeParams &P, int npl, const float2 *bufA, float2 *zsph, cudaStream_t st);
template <typename T> size_t fft_smem_need(const Plan &pl);
int init_fft_roots();

// The split-K workspace of gemm() opens with GEMM_COUNTER_BYTES of per-tile
// arrival counters (zeroed when the workspace is allocated; each split
// launch leaves them zero again); the partial sums follow.
constexpr size_t GEMM_COUNTER_BYTES = 16384;
constexpr long GEMM_TILE_COUNTERS = GEMM_COUNTER_BYTES / sizeof(int);
// qx_gemm.cu: C(m,n) = alpha * op(A)(m,:) . op(B)(:,n) + beta * C(m,n), column-major.
// TA: A stored K x M (A[m*lda + k]); TB: B stored N x K (B[k*ldb + n]).
// gamma: 0 plain; 1 Gamma-point metric 2*sum - a0*b0; 2 KB projection
// metric 2*sum - a0*b0 - 2*a1*b1.  colmap (device, optional) maps output
// column n to stored column colmap[n] of B and C; ncol_dev (device,
// optional) bounds the number of columns.
// ws/ws_bytes: optional split-K workspace (null: no split).
template <typename T>
int gemm(bool ta, bool tb, int M, int N, int K, T alpha, const T *A, long lda, const T *B, long ldb, T beta, T *C,
         long ldc, int gamma, const int *colmap, const int *ncol_dev, cudaStream_t st, void *ws = nullptr,
         size_t ws_bytes = 0, const T *rowscale = nullptr, void *pad = nullptr, size_t pad_bytes = 0);

void gemm_reduce_f32(bool ta, bool tb, int M, int N, int nsplit, float alpha, const float *A, long lda, const float *B,
                     long ldb, float beta, float *C, long ldc, int gamma, const float *W, cudaStream_t st,
                     const float *rowscale = nullptr);

// qx_tcgemm.cu: tcgen05 3xTF32 GEMM with gemm<float>'s semantics (no column
// map).  Returns 0 launched, -1 operands unsuitable (use the CUDA-core
// kernel), > 0 launch error.
int tc_gemm(bool ta, bool tb, int M, int N, int K, float alpha, const float *A, long lda, const float *B, long ldb,
            float beta, float *C, long ldc, int gamma, cudaStream_t st, void *ws, size_t ws_bytes, const float *rowscale = nullptr, void *pad = nullptr,
            size_t pad_bytes = 0);
bool tc_enabled();
// Copies `rows` rows of `inner` floats from stride ld to stride ldp (the
// tensor maps' 16-byte row-stride rule wants ldp a multiple of four).
void pad_rows_f32(const float *src, long ld, long inner, long rows, float *dst, long ldp, cudaStream_t st);
// Error code left by a tensor-core GEMM whose bounded wait ran out (0: none); clears it.
int tc_error_take();
// FP32 contractions that ran on the CUDA-core kernel (qx_gemm.cu)
long fp32_gemm_fallbacks();
void fp32_gemm_fallbacks_add(long n);   // graph capture and replay accounting
// autotuner hooks of the tensor-core GEMM: a per-shape K-split table and a
// per-thread override used while timing candidates
extern thread_local int tc_split_force, tc_tile_force;
int tc_split_lookup(bool ta, bool tb, int M, int N, int K, int gamma);
int tc_tile_lookup(bool ta, bool tb, int M, int N, int K, int gamma);
void tc_split_store(bool ta, bool tb, int M, int N, int K, int gamma, int nsplit, int tile);
bool tc_tile_valid(bool tb, int bn);

// qx_dense.cu (FP64, nb x nb)
// work: >= 32*33 + n doubles, used when S does not fit shared memory.
int cholinv(double *S, int n, double *work, int *d_info, cudaStream_t st);
// Symmetric eigen-decomposition; work >= 8*n*n + 1024*n doubles.
int syev(double *A, int n, double *w, double *V, double *work, int *d_info, cudaStream_t st,
         cudaStream_t side = nullptr, cudaEvent_t evf = nullptr, cudaEvent_t evj = nullptr);
template <typename Tin, typename Tout>
void convert(const Tin *in, Tout *out, long n, cudaStream_t st);
template <typename T>
void symmetrize_lower(const T *in, double *out, double *diag, int n, cudaStream_t st);

// qx_force.cu (Hellmann-Feynman forces)
void phase_tables(int natom, const double *satm, int km1, int km2, int km3, int ktot, double *dcq, double *dsq,
                  cudaStream_t st);
void floc_g(int natom, int n5, const int *ijk5, const int *ngabc, const double *gvec5, const double *svco,
            const int *ityp, const double2 *rhog, const double *dcq, const double *dsq, int km1, int km2, int km3,
            int ktot, double *floc, cudaStream_t st);
void real_part(const double2 *z, double *out, long n, cudaStream_t st);
void vloc_g(int n5, int natom, const int *ijk5, const int *ngabc, const double *svco, const int *ityp,
            const double *dcq, const double *dsq, int km1, int km2, int km3, int ktot, double rvol, int k1, int k2,
            int k3, double2 *zg, cudaStream_t st);
template <typename T>
void dtab_build(int nproj, int nplw, const T *kbg, const double *gw, T *dtab, cudaStream_t st);
template <typename T>
void fnl_reduce(int natom, int lmx, int nproj, int nb, const T *P, const T *D, const T *vclalp, const double *occ,
                double *fnl, cudaStream_t st);

// qx_tables.cu (G-space KB projector tables: setqlm once per cell, setbgq once per geometry)
void setqlm(int nplw1, int nchan, int lmx, int mxqlm, const double *dlqlm, const double *tbqlm, const double *qlm,
            const int *lmidx, const double *dk, double *zzz, cudaStream_t st);
template <typename T>
void setbgq(int natom, int nplw1, int ne, int lmx, const int *ityp, const int *ngabc, const double *dcq,
            const double *dsq, int km1, int km2, int km3, int ktot, const double *zzz, const int *even,
            const double *vcl_type, T *kbg, float *kbgp, long ldp, T *vcl, cudaStream_t st);
// real-space tables (setnlc): geometry of the point search
struct KbrGeom {
  double rba[9];   // lattice vectors as columns, row-major (x row, y row, z row)
  int k[3];        // FFT grid
  int nd[3];       // box half-widths in grid points
};
void kbr_count(const KbrGeom &G, int natom, const int *ityp, const double *satm, const double *rcut, int *cnt,
               int *off, cudaStream_t st);
template <typename T>
void kbr_fill(const KbrGeom &G, int natom, int lmx, const int *ityp, const double *satm, const double *rcut,
              const double *rcl, const double *dltnl, const double *tabnl, const double *dtabnl, int mxnl,
              const int *poly, const int *off, long cap, int *mesh, int *ptatom, T *vnl, T *dvnl, cudaStream_t st);
int kbr_lines(const int *off, int natom, const int *mesh, const int *ptatom, int k1, long nlines, int *lcnt,
              int *loff, int *cursor, int4 *lent, cudaStream_t st);

}  // namespace qx
