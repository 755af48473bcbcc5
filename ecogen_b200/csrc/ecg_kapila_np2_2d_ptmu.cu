// Explicit instantiations of the Kapila step kernels: 2 phases 2D with p-T-mu relaxation.
#include "ecg_kapila_launch.cuh"

namespace ecg {
ECG_KAPILA_INSTANTIATE(2, 2, true)
}  // namespace ecg
