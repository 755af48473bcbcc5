// Learned initial guess for the pressure-relaxation Newton iteration.
//
// Features of one relaxation (per phase k < NP, as rebuilt by buildPrim before relaxing):
//   alpha_k, log(rho_k), asinh(p_k / 1e5)
// Target: where the relaxed pressure falls inside the bracket of the phase pressures,
//   t = (p* - min_k p_k) / (max_k p_k - min_k p_k)        (0.5 when the bracket is empty),
// so that a seed p_min + clamp(t,0,1)*(p_max - p_min) always lies in the bracket that contains p*.
//
// Packed parameter block (floats), H = ECG_MLP_HIDDEN, I = number of inputs:
//   w1[H*I] b1[H] w2[H*H] b2[H] w3[H] b3 in_shift[I] in_scale[I] out_shift out_scale
#pragma once
#include "ecg_device.cuh"

namespace ecg {

constexpr int MLP_H = ECG_MLP_HIDDEN;

__host__ __device__ constexpr int mlp_packed_size(int nin) { return MLP_H * nin + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1 + 2 * nin + 2; }

template <int NP>
__device__ __forceinline__ void mlp_features(const double a[NP], const double r[NP], const double p[NP], float* x) {
#pragma unroll
  for (int k = 0; k < NP; k++) {
    x[3 * k + 0] = (float)a[k];
    x[3 * k + 1] = (float)log(r[k] > 1e-300 ? r[k] : 1e-300);
    x[3 * k + 2] = (float)asinh(p[k] * 1.e-5);
  }
}

__device__ __forceinline__ float gelu_f(float x) {
  const float c = 0.7978845608028654f;  // sqrt(2/pi)
  return 0.5f * x * (1.f + tanhf(c * (x + 0.044715f * x * x * x)));
}

// Per-thread FP32 evaluation of the MLP (weights read through the read-only cache).
template <int NP>
__device__ __forceinline__ double mlp_seed(const float* __restrict__ W, int nin, const double a[NP], const double r[NP],
                                           const double p[NP]) {
  constexpr int NI = 3 * NP;
  float x[NI];
  mlp_features<NP>(a, r, p, x);
  const float* w1 = W;
  const float* b1 = w1 + MLP_H * nin;
  const float* w2 = b1 + MLP_H;
  const float* b2 = w2 + MLP_H * MLP_H;
  const float* w3 = b2 + MLP_H;
  const float* b3 = w3 + MLP_H;
  const float* ish = b3 + 1;
  const float* isc = ish + nin;
  const float osh = isc[nin], osc = isc[nin + 1];
#pragma unroll
  for (int i = 0; i < NI; i++) x[i] = (x[i] - __ldg(ish + i)) * __ldg(isc + i);
  float h1[MLP_H];
#pragma unroll 4
  for (int j = 0; j < MLP_H; j++) {
    float acc = __ldg(b1 + j);
#pragma unroll
    for (int i = 0; i < NI; i++) acc += __ldg(w1 + j * nin + i) * x[i];
    h1[j] = gelu_f(acc);
  }
  float y = __ldg(b3);
#pragma unroll 2
  for (int j = 0; j < MLP_H; j++) {
    float acc = __ldg(b2 + j);
#pragma unroll 16
    for (int i = 0; i < MLP_H; i++) acc += __ldg(w2 + j * MLP_H + i) * h1[i];
    y += __ldg(w3 + j) * gelu_f(acc);
  }
  double t = (double)(y * osc + osh);
  double lo = p[0], hi = p[0];
#pragma unroll
  for (int k = 1; k < NP; k++) {
    lo = dmin(lo, p[k]);
    hi = dmax(hi, p[k]);
  }
  t = t < 0. ? 0. : (t > 1. ? 1. : t);
  return lo + t * (hi - lo);
}

// Appends one (features, target) pair of a converged relaxation to the recording buffer.
template <int NP>
__device__ __forceinline__ void record_pair(float* rx, float* ry, unsigned long long* count, unsigned long long maxn,
                                            const double a[NP], const double r[NP], const double p[NP], double pstar) {
  unsigned long long i = atomicAdd(count, 1ull);
  if (i >= maxn) return;
  float x[3 * NP];
  mlp_features<NP>(a, r, p, x);
#pragma unroll
  for (int j = 0; j < 3 * NP; j++) rx[i * (3 * NP) + j] = x[j];
  double lo = p[0], hi = p[0];
#pragma unroll
  for (int k = 1; k < NP; k++) {
    lo = dmin(lo, p[k]);
    hi = dmax(hi, p[k]);
  }
  ry[i] = (hi > lo) ? (float)((pstar - lo) / (hi - lo)) : 0.5f;
}

}  // namespace ecg
