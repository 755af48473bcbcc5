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
// and for a two-output network (the p-T-mu seed, further down) w3b[H] b3b out_shift_1 out_scale_1.
#pragma once
#include <cuda_bf16.h>

#include "ecg_device.cuh"

namespace ecg {

constexpr int MLP_H = ECG_MLP_HIDDEN;

__host__ __device__ constexpr int mlp_packed_size(int nin) { return MLP_H * nin + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1 + 2 * nin + 2; }

template <int NP>
__device__ __forceinline__ void mlp_features(const double a[NP], const double r[NP], const double p[NP], float* x) {
#pragma unroll
  for (int k = 0; k < NP; k++) {
    x[3 * k + 0] = (float)a[k];
    x[3 * k + 1] = logf(fmaxf((float)r[k], 1e-30f));  // single precision: the features enter as BF16
    x[3 * k + 2] = asinhf((float)(p[k] * 1.e-5));
  }
}

// GELU (tanh form) of the inference path with the SFU's tanh (tanh.approx.f32, relative error about
// 2^-11): its result is rounded to BF16 for the next layer, 2^-8 relative, so the approximation is below
// the network's own precision.  Training evaluates the same formula with tanhf.
__device__ __forceinline__ float tanh_sfu(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_f(float x) {
  const float c = 0.7978845608028654f;  // sqrt(2/pi)
  return 0.5f * x * (1.f + tanh_sfu(c * (x + 0.044715f * x * x * x)));
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

// ----------------------------------------------------------------------------------------------
// Warp-level evaluation with BF16 tensor-core MMA (mma.sync m16n8k16, FP32 accumulation).  The 32
// lanes of a warp form a 32 x 16 feature matrix (inputs padded to 16), gathered into A fragments by
// warp shuffles; layer 1 is 2 x 8 MMAs, layer 2 is 2 x 8 x 4 MMAs, the 64 -> 1 output is a dot
// product over the accumulator fragments reduced across each lane quad.  The accumulator fragment
// of an m16n8 tile is, register for register, the A fragment of the next layer's k16 slice, so
// layer outputs never leave registers.  The weights are read as ready-made BF16 B fragments from
// an installed model (MlpDev, about 11 KB, L1-resident), so the kernels keep no shared memory for
// them.  Every lane of the warp must call mlp_seed_warp.

// Device form of an installed seed model, built once by mlp_install (ecg_api.cu) from the packed
// FP32 parameters: w1[n-tile][lane] and w2[n-tile][k-chunk][lane] are the two 32-bit words of each
// lane's B fragment (bf16 pairs of a weight row, rounded to nearest even).
struct MlpDev {
  uint2 w1[8][32];
  uint2 w2[8][4][32];
  float b1[MLP_H], b2[MLP_H], w3[MLP_H];
  float ish[16], isc[16];
  float b3, osh, osc, pad;
  // second output of a two-output network (the p-T-mu seed's T_sat head)
  float w3b[MLP_H];
  float b3b, osh2, osc2, pad2;
};

__device__ __forceinline__ unsigned int pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned int*>(&v);
}

__device__ __forceinline__ void mma_bf16(float d[4], const unsigned int a[4], unsigned int b0, unsigned int b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// The network's NO raw outputs (before de-normalisation, bias included) for this lane's cell, from its
// NI normalised inputs (zeros on lanes without a cell).  Every lane of the warp must call it.
template <int NI, int NO>
__device__ __forceinline__ void mlp_warp_raw(const MlpDev* __restrict__ W, const float xn[NI], float y[NO]) {
  static_assert(NI <= 16, "inputs padded to one k16 slice");
  static_assert(NO == 1 || NO == 2, "one or two outputs");
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  float out[NO][4];  // row sums: tile 0 rows g, g+8; tile 1 rows g, g+8 (complete on lanes with t == 0)
#pragma unroll
  for (int m = 0; m < 2; m++) {
    // A fragment of rows (16m + g, 16m + g + 8), columns (2t, 2t+1) and (2t+8, 2t+9)
    float v[2][4];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int src = 16 * m + g + 8 * h;
#pragma unroll
      for (int q = 0; q < 4; q++) v[h][q] = 0.f;
#pragma unroll
      for (int i = 0; i < NI; i++) {
        const float xi = __shfl_sync(FULL, xn[i], src);
        if (i == 2 * t) v[h][0] = xi;
        if (i == 2 * t + 1) v[h][1] = xi;
        if (i == 2 * t + 8) v[h][2] = xi;
        if (i == 2 * t + 9) v[h][3] = xi;
      }
    }
    unsigned int A1[4] = {pack_bf16(v[0][0], v[0][1]), pack_bf16(v[1][0], v[1][1]), pack_bf16(v[0][2], v[0][3]),
                          pack_bf16(v[1][2], v[1][3])};
    unsigned int A2[4][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      const uint2 b = __ldg(&W->w1[nt][lane]);
      mma_bf16(c, A1, b.x, b.y);
      const int col = 8 * nt + 2 * t;
      const float2 bb = __ldg(reinterpret_cast<const float2*>(&W->b1[col]));
      unsigned int lo = pack_bf16(gelu_f(c[0] + bb.x), gelu_f(c[1] + bb.y));
      unsigned int hi = pack_bf16(gelu_f(c[2] + bb.x), gelu_f(c[3] + bb.y));
      const int kc = nt >> 1;
      if ((nt & 1) == 0) {
        A2[kc][0] = lo;
        A2[kc][1] = hi;
      } else {
        A2[kc][2] = lo;
        A2[kc][3] = hi;
      }
    }
    float sum_lo[NO], sum_hi[NO];
#pragma unroll
    for (int o = 0; o < NO; o++) sum_lo[o] = sum_hi[o] = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int kc = 0; kc < 4; kc++) {
        const uint2 b = __ldg(&W->w2[nt][kc][lane]);
        mma_bf16(c, A2[kc], b.x, b.y);
      }
      const int col = 8 * nt + 2 * t;
      const float2 b2 = __ldg(reinterpret_cast<const float2*>(&W->b2[col]));
      const float h0 = gelu_f(c[0] + b2.x), h1 = gelu_f(c[1] + b2.y), h2 = gelu_f(c[2] + b2.x),
                  h3 = gelu_f(c[3] + b2.y);
#pragma unroll
      for (int o = 0; o < NO; o++) {
        const float2 w3 = __ldg(reinterpret_cast<const float2*>(o == 0 ? &W->w3[col] : &W->w3b[col]));
        sum_lo[o] += w3.x * h0 + w3.y * h1;
        sum_hi[o] += w3.x * h2 + w3.y * h3;
      }
    }
#pragma unroll
    for (int o = 0; o < NO; o++) {
#pragma unroll
      for (int q = 1; q < 4; q <<= 1) {
        sum_lo[o] += __shfl_xor_sync(FULL, sum_lo[o], q);
        sum_hi[o] += __shfl_xor_sync(FULL, sum_hi[o], q);
      }
      out[o][2 * m] = sum_lo[o];
      out[o][2 * m + 1] = sum_hi[o];
    }
  }
  // row `lane` of the 32 x NO output: tile lane / 16, row lane % 16 held by lane 4 * (lane % 8)
  const int src = 4 * (lane & 7), sel = lane >> 3;
#pragma unroll
  for (int o = 0; o < NO; o++) {
    float yo = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const float v = __shfl_sync(FULL, out[o][q], src);
      if (q == sel) yo = v;
    }
    y[o] = yo + __ldg(o == 0 ? &W->b3 : &W->b3b);
  }
}

// Returns the seed for this lane's cell (lanes with `valid`), NaN for the other lanes.
template <int NP>
__device__ __forceinline__ double mlp_seed_warp(const MlpDev* __restrict__ W, bool valid, const double a[NP],
                                                const double r[NP], const double p[NP]) {
  constexpr int NI = 3 * NP;
  float xn[NI];
  if (valid) {
    float x[NI];
    mlp_features<NP>(a, r, p, x);
#pragma unroll
    for (int i = 0; i < NI; i++) xn[i] = (x[i] - __ldg(&W->ish[i])) * __ldg(&W->isc[i]);
  } else {
#pragma unroll
    for (int i = 0; i < NI; i++) xn[i] = 0.f;
  }
  float y[1];
  mlp_warp_raw<NI, 1>(W, xn, y);
  if (!valid) return __longlong_as_double(0x7ff8000000000000LL);
  double tt = (double)(y[0] * __ldg(&W->osc) + __ldg(&W->osh));
  double lo = p[0], hi = p[0];
#pragma unroll
  for (int k = 1; k < NP; k++) {
    lo = dmin(lo, p[k]);
    hi = dmax(hi, p[k]);
  }
  tt = tt < 0. ? 0. : (tt > 1. ? 1. : tt);
  return lo + tt * (hi - lo);
}

// ----------------------------------------------------------------------------------------------
// Learned (p*, T) seed of the p-T-mu relaxation (RelaxationPTMu::relaxation
// src/Relaxations/RelaxationPTMu.cpp:73-200).  The saturation solve's answer depends on the mixture
// density and internal energy the cell holds after buildPrim, so the features come from that state:
//   ln rho, asinh(e / 1e5), alpha_liq, ln rho_liq, ln rho_vap, asinh(sum_k alpha_k p_k / 1e5) (the
//   plain start), asinh(p_vap(rho, e) / 1e5), asinh(p_liq(rho, e) / 1e5) (the pure-phase pressures)
// and the targets are ln p* and T_sat(p*) of the converged solve.
constexpr int PTMU_NIN = 8;

template <int NP>
__device__ __forceinline__ void ptmu_features(const Model<NP>& M, int liq, int vap, const double a[NP],
                                              const double r[NP], const double p[NP], double rhomix, double emix,
                                              float x[PTMU_NIN]) {
  double ps = 0.;
#pragma unroll
  for (int k = 0; k < NP; k++) ps += a[k] * p[k];
  const double pv = eos_p(M.eos[vap], M.eps, rhomix, emix), pl = eos_p(M.eos[liq], M.eps, rhomix, emix);
  // single precision: the features enter the network as BF16
  x[0] = logf(fmaxf((float)rhomix, 1e-30f));
  x[1] = asinhf((float)(emix * 1.e-5));
  x[2] = (float)a[liq];
  x[3] = logf(fmaxf((float)r[liq], 1e-30f));
  x[4] = logf(fmaxf((float)r[vap], 1e-30f));
  x[5] = asinhf((float)(ps * 1.e-5));
  x[6] = asinhf((float)(pv * 1.e-5));
  x[7] = asinhf((float)(pl * 1.e-5));
}

// Appends one (features, ln p*, T_sat) record of a converged saturation solve.
__device__ __forceinline__ void record_ptmu_pair(float* rx, float* ry, unsigned long long* count,
                                                 unsigned long long maxn, const float x[PTMU_NIN], double pstar,
                                                 double tsat) {
  unsigned long long i = atomicAdd(count, 1ull);
  if (i >= maxn) return;
#pragma unroll
  for (int j = 0; j < PTMU_NIN; j++) rx[i * PTMU_NIN + j] = x[j];
  ry[2 * i] = (float)log(pstar);
  ry[2 * i + 1] = (float)tsat;
}

// (p*, T) seed for this lane's cell from its features (lanes with `valid`); every lane of the warp must
// call it.  p_seed / T_seed are -1 on lanes without a cell.
__device__ __forceinline__ void mlp_ptmu_seed_warp(const MlpDev* __restrict__ W, bool valid, const float x[PTMU_NIN],
                                                   double& p_seed, double& T_seed) {
  float xn[PTMU_NIN];
#pragma unroll
  for (int i = 0; i < PTMU_NIN; i++) xn[i] = valid ? (x[i] - __ldg(&W->ish[i])) * __ldg(&W->isc[i]) : 0.f;
  float y[2];
  mlp_warp_raw<PTMU_NIN, 2>(W, xn, y);
  p_seed = T_seed = -1.;
  if (!valid) return;
  p_seed = exp((double)(y[0] * __ldg(&W->osc) + __ldg(&W->osh)));
  T_seed = (double)(y[1] * __ldg(&W->osc2) + __ldg(&W->osh2));
}

// Builds the device form of a model from the packed FP32 parameters (see the top of this file).
cudaError_t mlp_install(const float* d_params, int nin, int nout, MlpDev* d_out, cudaStream_t stream);
// Checks, packs and installs an ABI model into *dev (allocated on first use); synchronous.  The pressure
// relaxation's model has 3 np inputs and one output, the p-T-mu relaxation's (ptmu) 8 inputs and two.
ecg_status mlp_upload(const ecg_mlp* m, int np, bool ptmu, MlpDev** dev, cudaStream_t stream);

}  // namespace ecg
