// Kapila step kernels with passive transports, 3 phases (1D, 2D, 3D), and the transport dispatcher.
#include "ecg_kapila_launch.cuh"

namespace ecg {

cudaError_t kapila_launch_tr_np2(int dim, bool ptmu, int pass, const StepParams& P, const Geometry& G,
                                 const ecg_eos* eos, double eps, cudaStream_t s, bool prepare);

cudaError_t kapila_launch_tr(int np, int dim, bool ptmu, int pass, const StepParams& P, const Geometry& G,
                             const ecg_eos* eos, double eps, cudaStream_t s, bool prepare) {
  if (P.ntr > KAPILA_MAX_TRANSPORTS) return cudaErrorNotSupported;
  if (np == 2) return kapila_launch_tr_np2(dim, ptmu, pass, P, G, eos, eps, s, prepare);
  if (np != 3 || ptmu) return cudaErrorNotSupported;
  constexpr int NT = KAPILA_MAX_TRANSPORTS;
  if (dim == 1) return launch_pass_seed<3, 1, false, false, EOS_DYNAMIC, NT>(pass, P, G, eos, eps, s, prepare);
  if (dim == 2) return launch_pass_seed<3, 2, false, false, EOS_DYNAMIC, NT>(pass, P, G, eos, eps, s, prepare);
  return launch_pass_seed<3, 3, false, false, EOS_DYNAMIC, NT>(pass, P, G, eos, eps, s, prepare);
}

}  // namespace ecg
