// Fused FFT plane launchers for grid lengths 40, 42, 45.
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_LENGTH(40)
QX_PLANE_LENGTH(42)
QX_PLANE_LENGTH(45)
}  // namespace qx
