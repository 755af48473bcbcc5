// Explicit instantiations of the Kapila step kernels: 3 phases 2D.
#include "ecg_kapila_launch.cuh"

namespace ecg {
ECG_KAPILA_INSTANTIATE(3, 2, false)
}  // namespace ecg
