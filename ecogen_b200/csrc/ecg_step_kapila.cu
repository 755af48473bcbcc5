// Dispatch of the Kapila step kernels over (phases, dimension, p-T-mu) variants.
#include "ecg_step.cuh"

namespace ecg {

template <int NP, int DIM, bool PTMU>
cudaError_t launch_pass(int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                        cudaStream_t s, bool prepare);

// Launches (or, with prepare, configures) one pass of the Kapila step for a case shape.
cudaError_t kapila_launch(int np, int dim, bool ptmu, int pass, const StepParams& P, const Geometry& G,
                          const ecg_eos* eos, double eps, cudaStream_t s, bool prepare) {
  if (np == 2) {
    if (ptmu) {
      if (dim == 1) return launch_pass<2, 1, true>(pass, P, G, eos, eps, s, prepare);
      if (dim == 2) return launch_pass<2, 2, true>(pass, P, G, eos, eps, s, prepare);
      return cudaErrorNotSupported;
    }
    if (dim == 1) return launch_pass<2, 1, false>(pass, P, G, eos, eps, s, prepare);
    if (dim == 2) return launch_pass<2, 2, false>(pass, P, G, eos, eps, s, prepare);
    return launch_pass<2, 3, false>(pass, P, G, eos, eps, s, prepare);
  }
  if (np == 3 && !ptmu) {
    if (dim == 1) return launch_pass<3, 1, false>(pass, P, G, eos, eps, s, prepare);
    if (dim == 2) return launch_pass<3, 2, false>(pass, P, G, eos, eps, s, prepare);
    return launch_pass<3, 3, false>(pass, P, G, eos, eps, s, prepare);
  }
  return cudaErrorNotSupported;
}

}  // namespace ecg
