// Explicit instantiations of the Kapila step kernels: 2 phases 3D.
#include "ecg_kapila_launch.cuh"

namespace ecg {
ECG_KAPILA_INSTANTIATE(2, 3, false)
}  // namespace ecg
