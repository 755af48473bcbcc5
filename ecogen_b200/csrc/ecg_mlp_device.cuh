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
    x[3 * k + 1] = (float)log(r[k] > 1e-300 ? r[k] : 1e-300);
    x[3 * k + 2] = (float)asinh(p[k] * 1.e-5);
  }
}

__device__ __forceinline__ float gelu_f(float x) {
  const float c = 0.7978845608028654f;  // sqrt(2/pi)
  return 0.5f * x * (1.f + tanhf(c * (x + 0.044715f * x * x * x)));
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
// Warp-level evaluation with BF16 tensor-core MMA (mma.sync m16n8k16, FP32 accumulation) and the
// weights held in shared memory as BF16.  The 32 lanes of a warp form a 32 x 16 feature matrix
// (inputs padded to 16); layer 1 is 2 x 8 MMAs, layer 2 is 2 x 8 x 4 MMAs, the 64 -> 1 output is
// a dot product over the accumulator fragments reduced across each lane quad.  The accumulator
// fragment of an m16n8 tile is, register for register, the A fragment of the next layer's k16
// slice, so layer outputs never leave registers.  Every lane of the warp must call it.

constexpr int MLP_WARPS = 8;  // warps per block that may call mlp_seed_warp (blocks of <= 256 threads)

struct MlpSmem {
  __nv_bfloat16 w1[MLP_H][16];
  __nv_bfloat16 w2[MLP_H][MLP_H];
  float b1[MLP_H], b2[MLP_H], w3[MLP_H];
  float b3, osh, osc, pad;
  float ish[16], isc[16];
  __nv_bfloat16 xs[MLP_WARPS][32][16];
  float ys[MLP_WARPS][32];
};

// Cooperative load of the packed FP32 parameters into shared memory (all threads of the block).
__device__ __forceinline__ void mlp_load(MlpSmem* S, const float* __restrict__ W, int nin) {
  const float* w1 = W;
  const float* b1 = w1 + MLP_H * nin;
  const float* w2 = b1 + MLP_H;
  const float* b2 = w2 + MLP_H * MLP_H;
  const float* w3 = b2 + MLP_H;
  const float* b3 = w3 + MLP_H;
  const float* ish = b3 + 1;
  const float* isc = ish + nin;
  for (int i = threadIdx.x; i < MLP_H * 16; i += blockDim.x) {
    int o = i / 16, k = i % 16;
    S->w1[o][k] = __float2bfloat16_rn(k < nin ? w1[o * nin + k] : 0.f);
  }
  for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) S->w2[i / MLP_H][i % MLP_H] = __float2bfloat16_rn(w2[i]);
  for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
    S->b1[i] = b1[i];
    S->b2[i] = b2[i];
    S->w3[i] = w3[i];
  }
  for (int i = threadIdx.x; i < 16; i += blockDim.x) {
    S->ish[i] = i < nin ? ish[i] : 0.f;
    S->isc[i] = i < nin ? isc[i] : 0.f;
  }
  if (threadIdx.x == 0) {
    S->b3 = b3[0];
    S->osh = isc[nin];
    S->osc = isc[nin + 1];
  }
}

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

// Returns the seed for this lane's cell (valid lanes), NaN for lanes without a cell.
template <int NP>
__device__ __forceinline__ double mlp_seed_warp(MlpSmem* S, bool valid, const double a[NP], const double r[NP],
                                                const double p[NP]) {
  constexpr int NI = 3 * NP;
  const int lane = threadIdx.x & 31, warp = (threadIdx.x >> 5) % MLP_WARPS;
  const int g = lane >> 2, t = lane & 3;
  float x[NI];
  if (valid) mlp_features<NP>(a, r, p, x);
#pragma unroll
  for (int i = 0; i < 16; i++) {
    float v = (valid && i < NI) ? (x[i < NI ? i : 0] - S->ish[i]) * S->isc[i] : 0.f;
    S->xs[warp][lane][i] = __float2bfloat16_rn(v);
  }
  __syncwarp();
  const unsigned int* xw = reinterpret_cast<const unsigned int*>(&S->xs[warp][0][0]);  // 8 words per row
  const unsigned int* w1w = reinterpret_cast<const unsigned int*>(&S->w1[0][0]);      // 8 words per row
  const unsigned int* w2w = reinterpret_cast<const unsigned int*>(&S->w2[0][0]);      // 32 words per row
  float out_lo[2], out_hi[2];
#pragma unroll
  for (int m = 0; m < 2; m++) {
    const int r0 = 16 * m + g, r1 = r0 + 8;
    unsigned int A1[4] = {xw[r0 * 8 + t], xw[r1 * 8 + t], xw[r0 * 8 + t + 4], xw[r1 * 8 + t + 4]};
    unsigned int A2[4][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      const int n = 8 * nt + g;
      mma_bf16(c, A1, w1w[n * 8 + t], w1w[n * 8 + t + 4]);
      const int col = 8 * nt + 2 * t;
      unsigned int lo = pack_bf16(gelu_f(c[0] + S->b1[col]), gelu_f(c[1] + S->b1[col + 1]));
      unsigned int hi = pack_bf16(gelu_f(c[2] + S->b1[col]), gelu_f(c[3] + S->b1[col + 1]));
      const int kc = nt >> 1;
      if ((nt & 1) == 0) {
        A2[kc][0] = lo;
        A2[kc][1] = hi;
      } else {
        A2[kc][2] = lo;
        A2[kc][3] = hi;
      }
    }
    float sum_lo = 0.f, sum_hi = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      const int n = 8 * nt + g;
#pragma unroll
      for (int kc = 0; kc < 4; kc++) mma_bf16(c, A2[kc], w2w[n * 32 + kc * 8 + t], w2w[n * 32 + kc * 8 + t + 4]);
      const int col = 8 * nt + 2 * t;
      sum_lo += S->w3[col] * gelu_f(c[0] + S->b2[col]) + S->w3[col + 1] * gelu_f(c[1] + S->b2[col + 1]);
      sum_hi += S->w3[col] * gelu_f(c[2] + S->b2[col]) + S->w3[col + 1] * gelu_f(c[3] + S->b2[col + 1]);
    }
#pragma unroll
    for (int o = 1; o < 4; o <<= 1) {
      sum_lo += __shfl_xor_sync(0xffffffffu, sum_lo, o);
      sum_hi += __shfl_xor_sync(0xffffffffu, sum_hi, o);
    }
    out_lo[m] = sum_lo;
    out_hi[m] = sum_hi;
  }
  if (t == 0) {
    S->ys[warp][g] = out_lo[0];
    S->ys[warp][g + 8] = out_hi[0];
    S->ys[warp][16 + g] = out_lo[1];
    S->ys[warp][24 + g] = out_hi[1];
  }
  __syncwarp();
  float y = S->ys[warp][lane] + S->b3;
  __syncwarp();
  if (!valid) return __longlong_as_double(0x7ff8000000000000LL);
  double tt = (double)(y * S->osc + S->osh);
  double lo = p[0], hi = p[0];
#pragma unroll
  for (int k = 1; k < NP; k++) {
    lo = dmin(lo, p[k]);
    hi = dmax(hi, p[k]);
  }
  tt = tt < 0. ? 0. : (tt > 1. ? 1. : tt);
  return lo + tt * (hi - lo);
}

}  // namespace ecg
