// Fused FFT plane launchers for grid lengths 48, 49, 54.
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_LENGTH(48)
QX_PLANE_LENGTH(49)
QX_PLANE_LENGTH(54)
}  // namespace qx
