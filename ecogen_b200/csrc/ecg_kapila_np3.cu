// Explicit instantiations of the Kapila step kernels: 3 phases 1D, 3 phases 2D, 3 phases 3D.
#include "ecg_kapila_launch.cuh"

namespace ecg {
ECG_KAPILA_INSTANTIATE(3, 1, false)
ECG_KAPILA_INSTANTIATE(3, 2, false)
ECG_KAPILA_INSTANTIATE(3, 3, false)
}  // namespace ecg
