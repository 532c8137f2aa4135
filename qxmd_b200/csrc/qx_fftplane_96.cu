// Fused FFT plane launchers for grid length 96 (two lanes a line).
#include "qx_fftplane_kern.cuh"

namespace qx {
QX_PLANE_LENGTH2(96)
}  // namespace qx
