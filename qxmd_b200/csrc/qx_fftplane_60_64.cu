// Fused FFT plane launchers for k1 x k2 planes 60x60, 64x64 and z lengths 60, 64.
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_GRID(60, 60)
QX_PLANE_GRID(64, 64)
QX_ZCOLS_LENGTH(60)
QX_ZCOLS_LENGTH(64)
}  // namespace qx
