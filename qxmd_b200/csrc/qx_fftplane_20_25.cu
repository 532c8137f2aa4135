// Fused FFT plane launchers for grid lengths 20, 21, 24, 25.
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_LENGTH(20)
QX_PLANE_LENGTH(21)
QX_PLANE_LENGTH(24)
QX_PLANE_LENGTH(25)
}  // namespace qx
