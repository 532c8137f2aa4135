// Fused FFT plane launchers for grid lengths 27, 30, 32, 36.
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_LENGTH(27)
QX_PLANE_LENGTH(30)
QX_PLANE_LENGTH(32)
QX_PLANE_LENGTH(36)
}  // namespace qx
