// Euler (single-phase) step kernels.
#include <cuda_runtime.h>

#include "ecg_step.cuh"

namespace ecg {

cudaError_t euler_launch(int dim, int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                         cudaStream_t s, bool prepare) {
  (void)dim; (void)pass; (void)P; (void)G; (void)eos; (void)eps; (void)s; (void)prepare;
  return cudaErrorNotSupported;
}

}  // namespace ecg
