// Explicit instantiations of the Kapila step kernels: 2 phases 1D, 2 phases 1D p-T-mu.
#include "ecg_kapila_launch.cuh"

namespace ecg {
ECG_KAPILA_INSTANTIATE(2, 1, false)
ECG_KAPILA_INSTANTIATE(2, 1, true)
}  // namespace ecg
