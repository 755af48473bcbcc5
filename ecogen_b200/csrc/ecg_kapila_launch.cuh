// Launch templates of the Kapila step kernels; explicit instantiations live in ecg_kapila_*.cu so
// that the (large) kernel variants compile in parallel.
#pragma once
#include "ecg_kapila_kernel.cuh"

namespace ecg {

template <int NP, int DIM, int PASS, bool PTMU, bool SEED>
cudaError_t launch_one(const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps, cudaStream_t s,
                              bool prepare) {
  using K = KapilaStep<NP, DIM, PASS>;
  using TS = TileShape<DIM>;
  auto kern = k_kapila_step<NP, DIM, PASS, PTMU, SEED>;
  const size_t sm = K::smem_bytes();
  if (prepare) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  }
  Model<NP> M;
  for (int k = 0; k < NP; k++) M.eos[k] = make_eos_params(eos[k]);
  M.eps = eps;
  dim3 grid((G.n[0] + TS::X - 1) / TS::X, (G.n[1] + TS::Y - 1) / TS::Y, (G.n[2] + TS::Z - 1) / TS::Z);
  kern<<<grid, K::NTH, sm, s>>>(P, G, M);
  return cudaGetLastError();
}

template <int NP, int DIM, bool PTMU, bool SEED>
cudaError_t launch_pass_seed(int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                             cudaStream_t s, bool prepare) {
  switch (pass) {
    case PASS_O1: return launch_one<NP, DIM, PASS_O1, PTMU, SEED && !PTMU>(P, G, eos, eps, s, prepare);
    case PASS_PRED: return launch_one<NP, DIM, PASS_PRED, PTMU, SEED && !PTMU>(P, G, eos, eps, s, prepare);
    default: return launch_one<NP, DIM, PASS_CORR, PTMU, SEED && !PTMU>(P, G, eos, eps, s, prepare);
  }
}

template <int NP, int DIM, bool PTMU>
cudaError_t launch_pass(int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                               cudaStream_t s, bool prepare) {
  // kernels with the learned seed are separate variants, so that the plain kernels carry none of
  // its registers; with prepare both are configured
  if (prepare) {
    cudaError_t e = launch_pass_seed<NP, DIM, PTMU, false>(pass, P, G, eos, eps, s, true);
    if (e != cudaSuccess || PTMU) return e;
    return launch_pass_seed<NP, DIM, PTMU, true>(pass, P, G, eos, eps, s, true);
  }
  if (P.mlp != nullptr) {
    if (PTMU) return cudaErrorNotSupported;
    return launch_pass_seed<NP, DIM, PTMU, true>(pass, P, G, eos, eps, s, false);
  }
  return launch_pass_seed<NP, DIM, PTMU, false>(pass, P, G, eos, eps, s, false);
}


#define ECG_KAPILA_INSTANTIATE(NP, DIM, PTMU)                                                                 \
  template cudaError_t launch_pass<NP, DIM, PTMU>(int, const StepParams&, const Geometry&, const ecg_eos*, double, \
                                                  cudaStream_t, bool);

}  // namespace ecg
