// Fused FFT plane launchers for k1 x k2 planes 27x27, 27x25, 30x30, 32x32, 36x36 and z lengths
// 27, 30, 32, 36.
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_GRID(27, 27)
QX_PLANE_GRID(27, 25)
QX_PLANE_GRID(30, 30)
QX_PLANE_GRID(32, 32)
QX_PLANE_GRID(36, 36)
QX_ZCOLS_LENGTH(27)
QX_ZCOLS_LENGTH(30)
QX_ZCOLS_LENGTH(32)
QX_ZCOLS_LENGTH(36)
}  // namespace qx
