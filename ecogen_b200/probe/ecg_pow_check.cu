// Device evaluation of the step kernels' table-driven pow and log (csrc/ecg_pow.cuh) over host arrays,
// for the test that compares them bit for bit with the same source built for the host.  Test infrastructure,
// built into the probe library (libecg_probe.so), not part of the solver's C ABI.
#include <cuda_runtime.h>

#include "../csrc/ecg_pow.cuh"

namespace {

__global__ void k_epow(const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ out,
                       long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = ecg::epow(x[i], y[i]);
}

__global__ void k_elog(const double* __restrict__ x, double* __restrict__ out, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = ecg::elog(x[i]);
}

}  // namespace

extern "C" {

// out[i] = epow(x[i], y[i]) on the current device for n host values (0 < n <= 2^26).  Returns 0 on
// success, otherwise the CUDA error code, or -1 for n outside the limits.
int ecg_probe_epow(const double* x, const double* y, double* out, long n) {
  if (n <= 0 || n > (1l << 26)) return -1;
  double* d = nullptr;
  const size_t bytes = sizeof(double) * (size_t)n;
  cudaError_t e = cudaMalloc(&d, 3 * bytes);
  if (e != cudaSuccess) return (int)e;
  e = cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + n, y, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_epow<<<(unsigned)((n + 255) / 256), 256>>>(d, d + n, d + 2 * n, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return (int)e;
}

// out[i] = elog(x[i]) on the current device for n host values (0 < n <= 2^26).  Returns 0 on success,
// otherwise the CUDA error code, or -1 for n outside the limits.
int ecg_probe_elog(const double* x, double* out, long n) {
  if (n <= 0 || n > (1l << 26)) return -1;
  double* d = nullptr;
  const size_t bytes = sizeof(double) * (size_t)n;
  cudaError_t e = cudaMalloc(&d, 2 * bytes);
  if (e != cudaSuccess) return (int)e;
  e = cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_elog<<<(unsigned)((n + 255) / 256), 256>>>(d, d + n, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d + n, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return (int)e;
}

}  // extern "C"
