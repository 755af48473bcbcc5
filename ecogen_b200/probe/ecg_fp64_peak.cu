// FP64 pipe throughput probe: the denominator of the FP64 roofline that bench.py reports beside the
// HBM one.  Measurement infrastructure, built into its own library (libecg_probe.so), not part of
// the solver's C ABI.
//
// Every thread runs NCHAIN independent chains x <- fma(x, a, b): with enough resident warps the
// FP64 pipe, not the dependency latency, limits the rate, so (threads x NCHAIN x iterations) /
// kernel time is the peak rate of FP64 instructions (one DFMA = 2 flops).  The chains stay in
// [b / (1 - a), 1] (a < 1, b > 0), so no overflow or subnormal slows them down; their sum is stored
// so the compiler keeps every FMA.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int NCHAIN = 8;

__global__ void __launch_bounds__(256) k_fp64_fma(int64_t iters, double a, double b, double* out) {
  double x[NCHAIN];
#pragma unroll
  for (int c = 0; c < NCHAIN; c++) x[c] = 0.5 + 1e-3 * (threadIdx.x + c);
#pragma unroll 4
  for (int64_t i = 0; i < iters; i++) {
#pragma unroll
    for (int c = 0; c < NCHAIN; c++) x[c] = __fma_rn(x[c], a, b);
  }
  double s = 0.;
#pragma unroll
  for (int c = 0; c < NCHAIN; c++) s += x[c];
  out[(int64_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" {

// Runs the probe on the current device: `blocks_per_sm` x SM-count blocks of 256 threads, `iters`
// iterations per chain, `reps` timed launches after one untimed launch.  Writes the best
// launch's DFMA instructions per second (thread instructions, i.e. lanes) and its time.
// Returns 0 on success, otherwise the CUDA error code.
int ecg_probe_fp64(int blocks_per_sm, long long iters, int reps, double* dfma_per_s, double* best_ms) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return (int)e;
  const int threads = 256;
  const int blocks = sms * (blocks_per_sm > 0 ? blocks_per_sm : 8);
  double* out = nullptr;
  e = cudaMalloc(&out, sizeof(double) * (size_t)blocks * threads);
  if (e != cudaSuccess) return (int)e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int r = 0; r <= reps && e == cudaSuccess; r++) {
    cudaEventRecord(e0);
    k_fp64_fma<<<blocks, threads>>>(iters, 0.999999, 1e-7, out);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess) return (int)e;
  const double fmas = (double)blocks * threads * NCHAIN * (double)iters;
  *dfma_per_s = fmas / (best * 1e-3);
  *best_ms = best;
  return 0;
}

}  // extern "C"
