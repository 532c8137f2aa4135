// Device state and launchers of the batched CG band update and small
// per-band reductions.
#pragma once
#include <cuda_runtime.h>

namespace qx {

// Per-band CG state (device arrays of length nb) plus the active list.
struct CgState {
  double *eig, *zansa, *zansab, *z000re, *x000re, *eigb, *betk, *dinnerx, *ekib, *cai;
  int *iter, *izcnt, *lreset, *active;
  int *list;    // active band indices (nb)
  int *pairs;   // band pairs of the FFT pipeline (2 * ceil(nb/2))
  int *nact;    // number of active bands
  int *npair;   // number of pairs
};

// Convergence parameters of eigen_BKL (modules.f90:171-182 defaults).
struct CgParm {
  int itermx, iteremx, noband;
  double tolera, roughfzan, roughfeig, threinn, wdinner;
};

// Sequential (one-rank) CG: bands are updated one after another; *cur is the
// band being updated, pairs = {cur, -1} and list = {cur} drive the H|psi>
// pipeline, and the update kernel advances cur, refreshes the band's snapshot
// column and clears the while-loop condition of the enclosing graph after the
// last band.
struct SeqArgs {
  int *cur, *pairs, *list;
  void *snap;
  int nb;
  int ccreal4;
  cudaGraphConditionalHandle handle;
};

template <typename T> void cg_init(int nb, int ne, long ldx, const T *x, const T *hx, T *g, const CgState &s, cudaStream_t st);
// cur != nullptr: one CTA updates band *cur (< nb) instead of one CTA per band.
template <typename T> void cg_prec(int nb, int ne, long ldx, T *g, T *h, const double *dk, const CgState &s, cudaStream_t st,
                                   const int *cur = nullptr);
template <typename T> void cg_mask(int nb, T *Pm, const CgState &s, cudaStream_t st);
template <typename T> void cg_orth(int nb, int ne, long ldx, const T *x, const T *hx, T *h, const CgState &s, cudaStream_t st,
                                   const int *cur = nullptr);
template <typename T> void cg_update_seq(int ne, long ldx, T *x, T *hx, T *g, const T *h, const T *gh, const CgState &s,
                                         const CgParm &pm, const SeqArgs &q, cudaStream_t st);
void seq_reset(const SeqArgs &q, cudaStream_t st);
// out[j] = <V_j | Y_cur> (Gamma metric; gamma 2 adds the -2 a1 b1 term of the
// KB projection) times scale[j] (nullable), for j < n (n = *n_dev if given).
template <typename T> void seq_dots(int nmax, const int *n_dev, int ne, const T *V, long ldv, const T *Y, long ldy,
                                    const int *cur, int gamma, const T *scale, double *out, cudaStream_t st);
// Y_cur += sign * sum_{j<n} coef[j] V_j.
template <typename T> void seq_axpy(int nmax, const int *n_dev, int ne, const T *V, long ldv, const double *coef,
                                    double sign, T *Y, long ldy, const int *cur, cudaStream_t st);
void cg_list(int nb, const CgState &s, cudaStream_t st);
void gradres_stats(const double *prod, const double *occ, int nb, double *out, cudaStream_t st);
void iter_sum(const int *iter, int nb, int *out, cudaStream_t st);
template <typename T> void cg_update(int nb, int ne, long ldx, T *x, T *hx, T *g, const T *h, const T *gh,
                                     const CgState &s, const CgParm &pm, cudaStream_t st);
template <typename T> void ekin(int nb, int ne, long ldx, const T *x, const double *dk, double *ekib, cudaStream_t st);
template <typename T> void gradres(int nb, int ne, long ldx, const T *x, const T *hx, const double *eig, double *prod,
                                   cudaStream_t st);
template <typename T> void scale_rows(int nproj, int ncol, T *P, long ldp, const T *v, const int *colmap,
                                      const int *ncol_dev, cudaStream_t st);

}  // namespace qx
