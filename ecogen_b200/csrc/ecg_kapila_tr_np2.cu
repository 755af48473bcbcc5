// Kapila step kernels with passive transports, 2 phases (1D, 2D, 3D; with and without p-T-mu).
#include "ecg_kapila_launch.cuh"

namespace ecg {

cudaError_t kapila_launch_tr_np2(int dim, bool ptmu, int pass, const StepParams& P, const Geometry& G,
                                 const ecg_eos* eos, double eps, cudaStream_t s, bool prepare) {
  constexpr int NT = KAPILA_MAX_TRANSPORTS;
  if (dim == 1) return ptmu ? launch_pass_seed<2, 1, true, false, EOS_DYNAMIC, NT>(pass, P, G, eos, eps, s, prepare)
                            : launch_pass_seed<2, 1, false, false, EOS_DYNAMIC, NT>(pass, P, G, eos, eps, s, prepare);
  if (dim == 2) return ptmu ? launch_pass_seed<2, 2, true, false, EOS_DYNAMIC, NT>(pass, P, G, eos, eps, s, prepare)
                            : launch_pass_seed<2, 2, false, false, EOS_DYNAMIC, NT>(pass, P, G, eos, eps, s, prepare);
  if (ptmu) return cudaErrorNotSupported;  // p-T-mu is not built for 3D meshes
  return launch_pass_seed<2, 3, false, false, EOS_DYNAMIC, NT>(pass, P, G, eos, eps, s, prepare);
}

}  // namespace ecg
