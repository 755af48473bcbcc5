// Explicit instantiations of the Kapila step kernels: 3 phases 1D.
#include "ecg_kapila_launch.cuh"

namespace ecg {
ECG_KAPILA_INSTANTIATE(3, 1, false)
}  // namespace ecg
