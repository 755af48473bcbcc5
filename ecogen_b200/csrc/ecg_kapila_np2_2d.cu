// Explicit instantiations of the Kapila step kernels: 2 phases 2D.
#include "ecg_kapila_launch.cuh"

namespace ecg {
ECG_KAPILA_INSTANTIATE(2, 2, false)
}  // namespace ecg
