// Fused FFT plane launchers for k1 x k2 planes 54x54, 54x24, 54x25, 54x27 and z lengths 54.
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_GRID(54, 54)
QX_PLANE_GRID(54, 24)
QX_PLANE_GRID(54, 25)
QX_PLANE_GRID(54, 27)
QX_ZCOLS_LENGTH(54)
}  // namespace qx
