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

template <typename T> void cg_init(int nb, int ne, long ldx, const T *x, const T *hx, T *g, const CgState &s, cudaStream_t st);
template <typename T> void cg_prec(int nb, int ne, long ldx, T *g, T *h, const double *dk, const CgState &s, cudaStream_t st);
template <typename T> void cg_mask(int nb, T *Pm, const CgState &s, cudaStream_t st);
template <typename T> void cg_orth(int nb, int ne, long ldx, const T *x, const T *hx, T *h, const CgState &s, cudaStream_t st);
void cg_list(int nb, const CgState &s, cudaStream_t st);
template <typename T> void cg_update(int nb, int ne, long ldx, T *x, T *hx, T *g, const T *h, const T *gh,
                                     const CgState &s, const CgParm &pm, cudaStream_t st);
template <typename T> void ekin(int nb, int ne, long ldx, const T *x, const double *dk, double *ekib, cudaStream_t st);
template <typename T> void gradres(int nb, int ne, long ldx, const T *x, const T *hx, const double *eig, double *prod,
                                   cudaStream_t st);
template <typename T> void scale_rows(int nproj, int ncol, T *P, long ldp, const T *v, const int *colmap,
                                      const int *ncol_dev, cudaStream_t st);

}  // namespace qx
