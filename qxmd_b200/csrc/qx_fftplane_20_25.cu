// Fused FFT plane launchers for k1 x k2 planes 20x20, 21x21, 24x24, 25x25, 24x25, 25x24, 25x27
// and z lengths 20, 21, 24, 25.
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_GRID(20, 20)
QX_PLANE_GRID(21, 21)
QX_PLANE_GRID(24, 24)
QX_PLANE_GRID(25, 25)
QX_PLANE_GRID(24, 25)
QX_PLANE_GRID(25, 24)
QX_PLANE_GRID(25, 27)
QX_ZCOLS_LENGTH(20)
QX_ZCOLS_LENGTH(21)
QX_ZCOLS_LENGTH(24)
QX_ZCOLS_LENGTH(25)
}  // namespace qx
