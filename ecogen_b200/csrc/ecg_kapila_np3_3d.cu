// Explicit instantiations of the Kapila step kernels: 3 phases 3D.
#include "ecg_kapila_launch.cuh"

namespace ecg {
ECG_KAPILA_INSTANTIATE(3, 3, false)
}  // namespace ecg
