// Fused FFT plane launchers for grid lengths 60, 64.
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_LENGTH(60)
QX_PLANE_LENGTH(64)
}  // namespace qx
