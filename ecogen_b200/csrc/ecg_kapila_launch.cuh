// Launch templates of the Kapila step kernels; explicit instantiations live in ecg_kapila_*.cu so
// that the (large) kernel variants compile in parallel.
#pragma once
#include "ecg_kapila_split.cuh"

namespace ecg {

template <int NP, int DIM, int PASS, bool PTMU, bool SEED, int TYPES = EOS_DYNAMIC, int NTM = 0>
cudaError_t launch_one(const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps, cudaStream_t s,
                              bool prepare) {
  using K = KapilaStep<NP, DIM, PASS, NTM>;
  using TS = TileShape<DIM>;
  auto kern = k_kapila_step<NP, DIM, PASS, PTMU, SEED, TYPES, NTM>;
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

// One pass of one kernel variant: the split form (face kernels + cell kernel) for 2D and 3D cases whose
// context holds face arrays, the fused kernel otherwise (1D, passive transports, the allocation-free
// entry point).  With prepare both forms are configured.
template <int NP, int DIM, int PASS, bool PTMU, bool SEED, int TYPES, int NTM>
cudaError_t launch_form(const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps, cudaStream_t s,
                        bool prepare) {
  constexpr bool kSplit = DIM >= 2 && NTM == 0;
  if (prepare) {
    cudaError_t e = launch_one<NP, DIM, PASS, PTMU, SEED, TYPES, NTM>(P, G, eos, eps, s, true);
    if (kSplit && e == cudaSuccess) e = launch_split<NP, DIM, PASS, PTMU, SEED, TYPES>(P, G, eos, eps, s, true);
    return e;
  }
  if (kSplit && P.flux[0] != nullptr) return launch_split<NP, DIM, PASS, PTMU, SEED, TYPES>(P, G, eos, eps, s, false);
  return launch_one<NP, DIM, PASS, PTMU, SEED, TYPES, NTM>(P, G, eos, eps, s, false);
}

template <int NP, int DIM, bool PTMU, bool SEED, int TYPES = EOS_DYNAMIC, int NTM = 0>
cudaError_t launch_pass_seed(int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                             cudaStream_t s, bool prepare) {
  switch (pass) {
    case PASS_O1: return launch_form<NP, DIM, PASS_O1, PTMU, SEED, TYPES, NTM>(P, G, eos, eps, s, prepare);
    case PASS_PRED: return launch_form<NP, DIM, PASS_PRED, PTMU, SEED, TYPES, NTM>(P, G, eos, eps, s, prepare);
    default: return launch_form<NP, DIM, PASS_CORR, PTMU, SEED, TYPES, NTM>(P, G, eos, eps, s, prepare);
  }
}

// Kernels with passive transports (up to two, generic EOS, no seed) live in their own translation
// units (ecg_kapila_tr_np2.cu, ecg_kapila_tr_np3.cu).
cudaError_t kapila_launch_tr(int np, int dim, bool ptmu, int pass, const StepParams& P, const Geometry& G,
                             const ecg_eos* eos, double eps, cudaStream_t s, bool prepare);
constexpr int KAPILA_MAX_TRANSPORTS = 2;

// The EOS combination of the shipped workloads (SG liquid first, ideal gases after; two stiffened
// gases with p-T-mu relaxation) has kernels (plain and seeded) with the types compiled in and no
// THINC or PT-relaxation code; every other case (other EOS, THINC, PT relaxation, passive
// transports) runs the generic kernels.
template <int NP>
constexpr int eos_fast_types() {
  return NP == 2 ? eos_types_code<2>(ECG_EOS_SG, ECG_EOS_IG) : eos_types_code<3>(ECG_EOS_SG, ECG_EOS_IG, ECG_EOS_IG);
}
// ... and the limiter of the shipped workloads (van Leer in the two-phase cases, minmod in the
// three-phase one), compiled into a further variant when all four limiter slots use it
template <int NP>
constexpr int eos_fast_limiter() {
  return NP == 2 ? ECG_LIM_VANLEER : ECG_LIM_MINMOD;
}
// With p-T-mu relaxation the shipped workload has a stiffened-gas liquid and a stiffened-gas vapour.
template <int NP, bool PTMU>
constexpr int workload_types() {
  return PTMU ? eos_types_code<NP>(ECG_EOS_SG, ECG_EOS_SG) : eos_fast_types<NP>();
}
template <int NP, bool PTMU = false>
inline bool eos_is_fast(const ecg_eos* eos) {
  int t[3] = {eos[0].type, eos[1].type, NP > 2 ? eos[2].type : 0};
  return eos_types_code<NP>(t[0], t[1], t[2]) == workload_types<NP, PTMU>();
}

template <int NP, int DIM, bool PTMU>
cudaError_t launch_pass(int pass, const StepParams& P, const Geometry& G, const ecg_eos* eos, double eps,
                               cudaStream_t s, bool prepare) {
  // kernels with the learned seed are separate variants, so that the plain kernels carry none of
  // its registers; with prepare both are configured
#ifndef ECG_NO_EOS_SPECIALIZATION
  constexpr bool kFast = true;
#else
  constexpr bool kFast = false;
#endif
  if (P.ntr > 0) {
    if (P.mlp != nullptr) return cudaErrorNotSupported;
    return kapila_launch_tr(NP, DIM, PTMU, pass, P, G, eos, eps, s, prepare);
  }
  // EOS types compiled in (limiters at run time), and EOS types plus the workload's limiter
  constexpr int kEos = kFast ? fast_code(workload_types<NP, PTMU>(), -1) : EOS_DYNAMIC;
  constexpr int kEosLim = kFast ? fast_code(workload_types<NP, PTMU>(), eos_fast_limiter<NP>()) : EOS_DYNAMIC;
  if (prepare) {
    cudaError_t e = launch_pass_seed<NP, DIM, PTMU, false>(pass, P, G, eos, eps, s, true);
    if (e == cudaSuccess && kFast) e = launch_pass_seed<NP, DIM, PTMU, false, kEos>(pass, P, G, eos, eps, s, true);
    if (e == cudaSuccess && kFast) e = launch_pass_seed<NP, DIM, PTMU, false, kEosLim>(pass, P, G, eos, eps, s, true);
    if (e != cudaSuccess) return e;
    e = launch_pass_seed<NP, DIM, PTMU, true>(pass, P, G, eos, eps, s, true);
    if (e == cudaSuccess && kFast) e = launch_pass_seed<NP, DIM, PTMU, true, kEos>(pass, P, G, eos, eps, s, true);
    if (e == cudaSuccess && kFast) e = launch_pass_seed<NP, DIM, PTMU, true, kEosLim>(pass, P, G, eos, eps, s, true);
    return e;
  }
  const bool fast_eos = kFast && !P.thinc && !P.pt && eos_is_fast<NP, PTMU>(eos);
  const int L = eos_fast_limiter<NP>();
  const bool fast_lim = P.lim[0] == L && P.lim[1] == L && P.lim[2] == L && P.lim[3] == L;
  if (P.mlp != nullptr) {  // the seeded kernels get the same compile-time configurations as the plain ones
    if (fast_eos && fast_lim) return launch_pass_seed<NP, DIM, PTMU, true, kEosLim>(pass, P, G, eos, eps, s, false);
    if (fast_eos) return launch_pass_seed<NP, DIM, PTMU, true, kEos>(pass, P, G, eos, eps, s, false);
    return launch_pass_seed<NP, DIM, PTMU, true>(pass, P, G, eos, eps, s, false);
  }
  if (fast_eos) {
    if (fast_lim) return launch_pass_seed<NP, DIM, PTMU, false, kEosLim>(pass, P, G, eos, eps, s, false);
    return launch_pass_seed<NP, DIM, PTMU, false, kEos>(pass, P, G, eos, eps, s, false);
  }
  return launch_pass_seed<NP, DIM, PTMU, false>(pass, P, G, eos, eps, s, false);
}


#define ECG_KAPILA_INSTANTIATE(NP, DIM, PTMU)                                                                 \
  template cudaError_t launch_pass<NP, DIM, PTMU>(int, const StepParams&, const Geometry&, const ecg_eos*, double, \
                                                  cudaStream_t, bool);

}  // namespace ecg
