// Explicit instantiations of the Kapila step kernels: 2 phases 2D, 2 phases 2D p-T-mu.
#include "ecg_kapila_launch.cuh"

namespace ecg {
ECG_KAPILA_INSTANTIATE(2, 2, false)
ECG_KAPILA_INSTANTIATE(2, 2, true)
}  // namespace ecg
