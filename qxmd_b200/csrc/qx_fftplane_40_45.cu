// Fused FFT plane launchers for k1 x k2 planes 40x40, 42x42, 42x21, 45x45, 45x24, 45x42 and z
// lengths 40, 42, 45.
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_GRID(40, 40)
QX_PLANE_GRID(42, 42)
QX_PLANE_GRID(42, 21)
QX_PLANE_GRID(45, 45)
QX_PLANE_GRID(45, 24)
QX_PLANE_GRID(45, 42)
QX_ZCOLS_LENGTH(40)
QX_ZCOLS_LENGTH(42)
QX_ZCOLS_LENGTH(45)
}  // namespace qx
