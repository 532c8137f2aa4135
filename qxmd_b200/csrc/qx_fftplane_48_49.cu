// Fused FFT plane launchers for k1 x k2 planes 48x48, 48x45, 49x49, 49x25 and z lengths 48, 49.
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_GRID(48, 48)
QX_PLANE_GRID(48, 45)
QX_PLANE_GRID(49, 49)
QX_PLANE_GRID(49, 25)
QX_ZCOLS_LENGTH(48)
QX_ZCOLS_LENGTH(49)
}  // namespace qx
