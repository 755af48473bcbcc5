// Training of the relaxation-seed MLP (nin -> 64 -> 64 -> 1, GELU) on the GPU: forward, backward
// and AdamW kernels written for this library.
//
// Work split: a block of 64 threads owns hidden unit j = threadIdx.x of both hidden layers and a
// tile of rows at a time.  Activations of the tile live in shared memory; each thread accumulates
// the gradient rows it owns (row j of W1 and W2, entry j of b1, b2, w3) in shared memory across
// the tiles of its slice of the batch, and adds them to the global gradient once per block.
// Everything is FP32; the loss is the mean squared error of the normalised target.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "ecg_internal.h"

namespace ecg {

constexpr int TH = ECG_MLP_HIDDEN;  // hidden width
constexpr int TROWS = 32;           // rows per tile

struct MlpDev {
  float *w1, *b1, *w2, *b2, *w3, *b3;  // parameters
};

__device__ __forceinline__ float t_gelu(float z, float* d) {
  const float c = 0.7978845608028654f;
  float u = c * (z + 0.044715f * z * z * z);
  float th = tanhf(u);
  if (d) {
    float du = c * (1.f + 3.f * 0.044715f * z * z);
    *d = 0.5f * (1.f + th) + 0.5f * z * (1.f - th * th) * du;
  }
  return 0.5f * z * (1.f + th);
}

// Forward (and, with grads != nullptr, backward) of rows [r0, r1) of the batch, NOUT outputs per row
// (y and yhat are n x NOUT).  Gradients are added into g (same layout as the parameters) scaled by
// 1/n_total; loss_sum receives the sum of squared errors over rows and outputs.
template <int NOUT>
__global__ void __launch_bounds__(TH) k_mlp_fwd_bwd(MlpDev P, int nin, const float* __restrict__ x,
                                                    const float* __restrict__ y, int n, float* yhat, MlpDev G,
                                                    float* loss_sum, float inv_n) {
  extern __shared__ float sm[];
  float* sW1 = sm;                     // [TH][nin]
  float* sW2 = sW1 + TH * nin;         // [TH][TH]
  float* sx = sW2 + TH * TH;           // [TROWS][nin]
  float* sh1 = sx + TROWS * nin;       // [TROWS][TH]
  float* sz1 = sh1 + TROWS * TH;       // [TROWS][TH]  (gelu' of layer 1)
  float* sdz2 = sz1 + TROWS * TH;      // [TROWS][TH]
  float* sy = sdz2 + TROWS * TH;       // [TROWS][NOUT], room for two outputs
  float* gW1 = sy + 2 * TROWS;         // [TH][nin] gradient accumulators (row j owned by thread j)
  float* gW2 = gW1 + TH * nin;         // [TH][TH]
  const int j = threadIdx.x;
  const bool train = (G.w1 != nullptr);
  for (int i = j; i < TH * nin; i += TH) {
    sW1[i] = P.w1[i];
    gW1[i] = 0.f;
  }
  for (int i = j; i < TH * TH; i += TH) {
    sW2[i] = P.w2[i];
    gW2[i] = 0.f;
  }
  const float b1j = P.b1[j], b2j = P.b2[j];
  float w3j[NOUT], b3[NOUT], gw3[NOUT], gb3[NOUT];
#pragma unroll
  for (int o = 0; o < NOUT; o++) {
    w3j[o] = P.w3[o * TH + j];
    b3[o] = P.b3[o];
    gw3[o] = gb3[o] = 0.f;
  }
  float gb1 = 0.f, gb2 = 0.f, lsum = 0.f;
  __syncthreads();
  const int ntiles = (n + TROWS - 1) / TROWS;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = tile * TROWS;
    const int nr = min(TROWS, n - r0);
    for (int i = j; i < nr * nin; i += TH) sx[i] = x[(size_t)r0 * nin + i];
    __syncthreads();
    // layer 1 (unit j)
    float h2[TROWS], d2[TROWS];
    for (int r = 0; r < nr; r++) {
      float z = b1j;
      for (int i = 0; i < nin; i++) z += sW1[j * nin + i] * sx[r * nin + i];
      float d;
      sh1[r * TH + j] = t_gelu(z, &d);
      sz1[r * TH + j] = d;
    }
    __syncthreads();
    // layer 2 (unit j) and the output partial sums
    for (int r = 0; r < nr; r++) {
      float z = b2j;
      for (int i = 0; i < TH; i++) z += sW2[j * TH + i] * sh1[r * TH + i];
      h2[r] = t_gelu(z, &d2[r]);
    }
    for (int r = 0; r < nr; r++) {
#pragma unroll
      for (int o = 0; o < NOUT; o++) {
        float v = w3j[o] * h2[r];
        for (int q = 16; q > 0; q >>= 1) v += __shfl_xor_sync(0xffffffffu, v, q);
        if ((j & 31) == 0) sdz2[r * TH + j + o] = v;  // scratch: warp partials at columns o and 32 + o
      }
    }
    __syncthreads();
    if (j < nr) {
#pragma unroll
      for (int o = 0; o < NOUT; o++) {
        float out = sdz2[j * TH + o] + sdz2[j * TH + 32 + o] + b3[o];
        sy[j * NOUT + o] = out;
        if (yhat) yhat[(size_t)(r0 + j) * NOUT + o] = out;
      }
    }
    __syncthreads();
    if (train) {
      // backward: dL/dy_o = 2 (yhat_o - y_o) / n
      for (int r = 0; r < nr; r++) {
        float dsum = 0.f;
#pragma unroll
        for (int o = 0; o < NOUT; o++) {
          float e = sy[r * NOUT + o] - y[(size_t)(r0 + r) * NOUT + o];
          float dy = 2.f * e * inv_n;
          if (j == 0) {
            gb3[o] += dy;
            lsum += e * e;
          }
          gw3[o] += dy * h2[r];
          dsum += dy * w3j[o];
        }
        float dz2 = dsum * d2[r];
        sdz2[r * TH + j] = dz2;
        gb2 += dz2;
        for (int i = 0; i < TH; i++) gW2[j * TH + i] += dz2 * sh1[r * TH + i];
      }
      __syncthreads();
      // dh1[r][j] = sum_m W2[m][j] dz2[r][m]
      for (int r = 0; r < nr; r++) {
        float dh = 0.f;
        for (int m = 0; m < TH; m++) dh += sW2[m * TH + j] * sdz2[r * TH + m];
        float dz1 = dh * sz1[r * TH + j];
        gb1 += dz1;
        for (int i = 0; i < nin; i++) gW1[j * nin + i] += dz1 * sx[r * nin + i];
      }
    }
    __syncthreads();
  }
  if (train) {
    for (int i = 0; i < nin; i++) atomicAdd(&G.w1[j * nin + i], gW1[j * nin + i]);
    for (int i = 0; i < TH; i++) atomicAdd(&G.w2[j * TH + i], gW2[j * TH + i]);
    atomicAdd(&G.b1[j], gb1);
    atomicAdd(&G.b2[j], gb2);
#pragma unroll
    for (int o = 0; o < NOUT; o++) atomicAdd(&G.w3[o * TH + j], gw3[o]);
    if (j == 0) {
#pragma unroll
      for (int o = 0; o < NOUT; o++) atomicAdd(&G.b3[o], gb3[o]);
      atomicAdd(loss_sum, lsum);
    }
  }
}

// AdamW (decoupled weight decay) over a flat parameter vector.
__global__ void k_adamw(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                        float wd, float c1, float c2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i];
  float mi = b1 * m[i] + (1.f - b1) * gi;
  float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float mh = mi / c1, vh = vi / c2;
  p[i] -= lr * (mh / (sqrtf(vh) + eps) + wd * p[i]);
}

}  // namespace ecg

using namespace ecg;

struct ecg_trainer {
  int nin = 0;
  int nout = 1;
  int nparam = 0;
  float* p = nullptr;   // flat: w1 b1 w2 b2 w3[nout][H] b3[nout]
  float* g = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  float* loss = nullptr;
  float* dx = nullptr;
  float* dy = nullptr;
  float* dyhat = nullptr;
  size_t cap = 0;
  long step = 0;
  std::vector<float> host;  // export copy
  float in_shift[ECG_MLP_MAX_IN] = {}, in_scale[ECG_MLP_MAX_IN] = {};
  float out_shift[2] = {0.f, 0.f}, out_scale[2] = {1.f, 1.f};
  cudaStream_t stream = nullptr;
};

namespace {

MlpDev views(float* base, int nin, int nout) {
  MlpDev d;
  d.w1 = base;
  d.b1 = d.w1 + TH * nin;
  d.w2 = d.b1 + TH;
  d.b2 = d.w2 + TH * TH;
  d.w3 = d.b2 + TH;
  d.b3 = d.w3 + TH * nout;
  return d;
}

size_t smem_bytes(int nin) {
  return sizeof(float) *
         (size_t)(TH * nin + TH * TH + TROWS * nin + 3 * TROWS * TH + 2 * TROWS + TH * nin + TH * TH);
}

ecg_status tfail(cudaError_t e, const char* w) {
  set_error(std::string(w) + ": " + cudaGetErrorString(e));
  return ECG_ERR_CUDA;
}
#define TCUDA(call)                                   \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return tfail(e_, #call);   \
  } while (0)

ecg_status ensure(ecg_trainer* tr, size_t n) {
  if (n <= tr->cap) return ECG_OK;
  cudaFree(tr->dx);
  cudaFree(tr->dy);
  cudaFree(tr->dyhat);
  TCUDA(cudaMalloc(&tr->dx, sizeof(float) * n * tr->nin));
  TCUDA(cudaMalloc(&tr->dy, sizeof(float) * n * tr->nout));
  TCUDA(cudaMalloc(&tr->dyhat, sizeof(float) * n * tr->nout));
  tr->cap = n;
  return ECG_OK;
}

ecg_status run_batch(ecg_trainer* tr, const float* dxp, const float* dyp, int n, bool train, float* yhat_dev,
                     float* loss_out) {
  MlpDev P = views(tr->p, tr->nin, tr->nout);
  MlpDev G = train ? views(tr->g, tr->nin, tr->nout) : MlpDev{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  if (train) {
    TCUDA(cudaMemsetAsync(tr->g, 0, sizeof(float) * tr->nparam, tr->stream));
    TCUDA(cudaMemsetAsync(tr->loss, 0, sizeof(float), tr->stream));
  }
  int ntiles = (n + TROWS - 1) / TROWS;
  int grid = std::min(ntiles, 148 * 4);
  if (tr->nout == 2)
    k_mlp_fwd_bwd<2><<<grid, TH, smem_bytes(tr->nin), tr->stream>>>(P, tr->nin, dxp, dyp, n, yhat_dev, G, tr->loss,
                                                                   1.f / (float)n);
  else
    k_mlp_fwd_bwd<1><<<grid, TH, smem_bytes(tr->nin), tr->stream>>>(P, tr->nin, dxp, dyp, n, yhat_dev, G, tr->loss,
                                                                   1.f / (float)n);
  TCUDA(cudaGetLastError());
  if (loss_out) {
    float l = 0.f;
    TCUDA(cudaMemcpyAsync(&l, tr->loss, sizeof(float), cudaMemcpyDeviceToHost, tr->stream));
    TCUDA(cudaStreamSynchronize(tr->stream));
    *loss_out = l / (float)n;
  }
  return ECG_OK;
}

}  // namespace

extern "C" ecg_status ecg_trainer_create(int32_t nin, int32_t hidden, uint64_t seed, ecg_trainer** out) {
  return ecg_trainer_create_n(nin, 1, hidden, seed, out);
}

extern "C" ecg_status ecg_trainer_create_n(int32_t nin, int32_t nout, int32_t hidden, uint64_t seed,
                                           ecg_trainer** out) {
  if (!out || nin < 1 || nin > ECG_MLP_MAX_IN || hidden != ECG_MLP_HIDDEN || nout < 1 || nout > 2) {
    set_error("trainer shape must be nin (<=16) -> 64 -> 64 -> nout (1 or 2)");
    return ECG_ERR_INVALID;
  }
  *out = nullptr;
  auto tr = new ecg_trainer();
  tr->nin = nin;
  tr->nout = nout;
  tr->nparam = TH * nin + TH + TH * TH + TH + nout * TH + nout;
  for (int i = 0; i < ECG_MLP_MAX_IN; i++) tr->in_scale[i] = 1.f;
  std::vector<float> h(tr->nparam, 0.f);
  std::mt19937_64 g(seed);
  auto fill = [&](float* w, int fan_in, int count) {
    std::normal_distribution<float> nd(0.f, std::sqrt(1.f / (float)fan_in));
    for (int i = 0; i < count; i++) w[i] = nd(g);
  };
  fill(h.data(), nin, TH * nin);
  fill(h.data() + TH * nin + TH, TH, TH * TH);
  fill(h.data() + TH * nin + TH + TH * TH + TH, TH, nout * TH);
  cudaError_t e = cudaStreamCreateWithFlags(&tr->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&tr->p, sizeof(float) * tr->nparam);
  if (e == cudaSuccess) e = cudaMalloc(&tr->g, sizeof(float) * tr->nparam);
  if (e == cudaSuccess) e = cudaMalloc(&tr->m, sizeof(float) * tr->nparam);
  if (e == cudaSuccess) e = cudaMalloc(&tr->v, sizeof(float) * tr->nparam);
  if (e == cudaSuccess) e = cudaMalloc(&tr->loss, sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(tr->p, h.data(), sizeof(float) * tr->nparam, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(tr->m, 0, sizeof(float) * tr->nparam);
  if (e == cudaSuccess) e = cudaMemset(tr->v, 0, sizeof(float) * tr->nparam);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mlp_fwd_bwd<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes(nin));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mlp_fwd_bwd<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes(nin));
  if (e != cudaSuccess) {
    ecg_trainer_destroy(tr);
    return tfail(e, "ecg_trainer_create");
  }
  *out = tr;
  return ECG_OK;
}

extern "C" void ecg_trainer_destroy(ecg_trainer* tr) {
  if (!tr) return;
  if (tr->stream) cudaStreamSynchronize(tr->stream);
  cudaFree(tr->p);
  cudaFree(tr->g);
  cudaFree(tr->m);
  cudaFree(tr->v);
  cudaFree(tr->loss);
  cudaFree(tr->dx);
  cudaFree(tr->dy);
  cudaFree(tr->dyhat);
  if (tr->stream) cudaStreamDestroy(tr->stream);
  delete tr;
}

extern "C" ecg_status ecg_trainer_epoch(ecg_trainer* tr, const float* x, const float* y, int64_t n, int32_t batch,
                                        float lr, float wd, float* mean_loss) {
  if (!tr || !x || !y || n < 1 || batch < 1) {
    set_error("bad argument");
    return ECG_ERR_INVALID;
  }
  ecg_status s = ensure(tr, (size_t)n);
  if (s != ECG_OK) return s;
  TCUDA(cudaMemcpyAsync(tr->dx, x, sizeof(float) * n * tr->nin, cudaMemcpyHostToDevice, tr->stream));
  TCUDA(cudaMemcpyAsync(tr->dy, y, sizeof(float) * n * tr->nout, cudaMemcpyHostToDevice, tr->stream));
  double total = 0.;
  int64_t nb = 0;
  for (int64_t r = 0; r < n; r += batch) {
    int cnt = (int)std::min<int64_t>(batch, n - r);
    float l = 0.f;
    s = run_batch(tr, tr->dx + r * tr->nin, tr->dy + r * tr->nout, cnt, true, nullptr, &l);
    if (s != ECG_OK) return s;
    tr->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.f - std::pow(b1, (float)tr->step), c2 = 1.f - std::pow(b2, (float)tr->step);
    k_adamw<<<(tr->nparam + 255) / 256, 256, 0, tr->stream>>>(tr->p, tr->g, tr->m, tr->v, tr->nparam, lr, b1, b2, 1e-8f,
                                                               wd, c1, c2);
    TCUDA(cudaGetLastError());
    total += (double)l * cnt;
    nb += cnt;
  }
  TCUDA(cudaStreamSynchronize(tr->stream));
  if (mean_loss) *mean_loss = (float)(total / (double)nb);
  return ECG_OK;
}

extern "C" ecg_status ecg_trainer_grad(ecg_trainer* tr, const float* x, const float* y, int32_t n, float* loss,
                                       float* gw1, float* gb1, float* gw2, float* gb2, float* gw3, float* gb3) {
  if (!tr || !x || !y || n < 1) {
    set_error("bad argument");
    return ECG_ERR_INVALID;
  }
  ecg_status s = ensure(tr, (size_t)n);
  if (s != ECG_OK) return s;
  TCUDA(cudaMemcpyAsync(tr->dx, x, sizeof(float) * n * tr->nin, cudaMemcpyHostToDevice, tr->stream));
  TCUDA(cudaMemcpyAsync(tr->dy, y, sizeof(float) * n * tr->nout, cudaMemcpyHostToDevice, tr->stream));
  float l = 0.f;
  s = run_batch(tr, tr->dx, tr->dy, n, true, nullptr, &l);
  if (s != ECG_OK) return s;
  std::vector<float> g(tr->nparam);
  TCUDA(cudaMemcpy(g.data(), tr->g, sizeof(float) * tr->nparam, cudaMemcpyDeviceToHost));
  const int nin = tr->nin;
  const float* q = g.data();
  if (gw1) std::memcpy(gw1, q, sizeof(float) * TH * nin);
  q += TH * nin;
  if (gb1) std::memcpy(gb1, q, sizeof(float) * TH);
  q += TH;
  if (gw2) std::memcpy(gw2, q, sizeof(float) * TH * TH);
  q += TH * TH;
  if (gb2) std::memcpy(gb2, q, sizeof(float) * TH);
  q += TH;
  if (gw3) std::memcpy(gw3, q, sizeof(float) * TH * tr->nout);
  q += TH * tr->nout;
  if (gb3) std::memcpy(gb3, q, sizeof(float) * tr->nout);
  if (loss) *loss = l;
  return ECG_OK;
}

extern "C" ecg_status ecg_trainer_forward(ecg_trainer* tr, const float* x, int32_t n, float* yhat) {
  if (!tr || !x || !yhat || n < 1) {
    set_error("bad argument");
    return ECG_ERR_INVALID;
  }
  ecg_status s = ensure(tr, (size_t)n);
  if (s != ECG_OK) return s;
  TCUDA(cudaMemcpyAsync(tr->dx, x, sizeof(float) * n * tr->nin, cudaMemcpyHostToDevice, tr->stream));
  s = run_batch(tr, tr->dx, tr->dy, n, false, tr->dyhat, nullptr);
  if (s != ECG_OK) return s;
  TCUDA(cudaMemcpyAsync(yhat, tr->dyhat, sizeof(float) * n * tr->nout, cudaMemcpyDeviceToHost, tr->stream));
  TCUDA(cudaStreamSynchronize(tr->stream));
  return ECG_OK;
}

extern "C" ecg_status ecg_trainer_set_norm(ecg_trainer* tr, const float* in_shift, const float* in_scale,
                                           float out_shift, float out_scale) {
  if (!tr || !in_shift || !in_scale) {
    set_error("bad argument");
    return ECG_ERR_INVALID;
  }
  for (int i = 0; i < tr->nin; i++) {
    tr->in_shift[i] = in_shift[i];
    tr->in_scale[i] = in_scale[i];
  }
  tr->out_shift[0] = out_shift;
  tr->out_scale[0] = out_scale;
  return ECG_OK;
}

// De-normalisation of the second output of a two-output network (exported as out_shift_1 / _scale_1).
extern "C" ecg_status ecg_trainer_set_norm_out1(ecg_trainer* tr, float out_shift, float out_scale) {
  if (!tr || tr->nout < 2) {
    set_error("the trainer has one output");
    return ECG_ERR_INVALID;
  }
  tr->out_shift[1] = out_shift;
  tr->out_scale[1] = out_scale;
  return ECG_OK;
}

extern "C" ecg_status ecg_trainer_export(ecg_trainer* tr, ecg_mlp* out) {
  if (!tr || !out) {
    set_error("bad argument");
    return ECG_ERR_INVALID;
  }
  tr->host.resize(tr->nparam);
  TCUDA(cudaMemcpy(tr->host.data(), tr->p, sizeof(float) * tr->nparam, cudaMemcpyDeviceToHost));
  const int nin = tr->nin;
  std::memset(out, 0, sizeof(*out));
  out->n_in = nin;
  out->hidden = TH;
  float* q = tr->host.data();
  out->w1 = q;
  q += TH * nin;
  out->b1 = q;
  q += TH;
  out->w2 = q;
  q += TH * TH;
  out->b2 = q;
  q += TH;
  out->w3 = q;
  q += TH * tr->nout;
  out->b3 = q[0];
  out->n_out = tr->nout;
  if (tr->nout == 2) out->b3_1 = q[1];
  for (int i = 0; i < nin; i++) {
    out->in_shift[i] = tr->in_shift[i];
    out->in_scale[i] = tr->in_scale[i];
  }
  out->out_shift = tr->out_shift[0];
  out->out_scale = tr->out_scale[0];
  out->out_shift_1 = tr->out_shift[1];
  out->out_scale_1 = tr->out_scale[1];
  return ECG_OK;
}

extern "C" ecg_status ecg_trainer_import(ecg_trainer* tr, const ecg_mlp* in) {
  if (!tr || !in || in->n_in != tr->nin || in->hidden != TH || (in->n_out > 1 ? in->n_out : 1) != tr->nout) {
    set_error("bad argument");
    return ECG_ERR_INVALID;
  }
  const int nin = tr->nin;
  std::vector<float> h(tr->nparam);
  float* q = h.data();
  std::memcpy(q, in->w1, sizeof(float) * TH * nin);
  q += TH * nin;
  std::memcpy(q, in->b1, sizeof(float) * TH);
  q += TH;
  std::memcpy(q, in->w2, sizeof(float) * TH * TH);
  q += TH * TH;
  std::memcpy(q, in->b2, sizeof(float) * TH);
  q += TH;
  std::memcpy(q, in->w3, sizeof(float) * TH * tr->nout);
  q += TH * tr->nout;
  q[0] = in->b3;
  if (tr->nout == 2) q[1] = in->b3_1;
  TCUDA(cudaMemcpy(tr->p, h.data(), sizeof(float) * tr->nparam, cudaMemcpyHostToDevice));
  for (int i = 0; i < nin; i++) {
    tr->in_shift[i] = in->in_shift[i];
    tr->in_scale[i] = in->in_scale[i];
  }
  tr->out_shift[0] = in->out_shift;
  tr->out_scale[0] = in->out_scale;
  tr->out_shift[1] = in->out_shift_1;
  tr->out_scale[1] = in->out_scale_1;
  return ECG_OK;
}
