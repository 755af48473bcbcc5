// Check of the step kernels' branch-free division and square root (csrc/ecg_ieee.cuh) against CUDA's
// correctly rounded `/` and `sqrt()`, bit for bit, on hashed operands.  Test infrastructure, built
// into the probe library (libecg_probe.so), not part of the solver's C ABI.
//
// Each thread draws `iters` operand pairs from a 64-bit hash of (seed, thread, iteration): a random
// 52-bit significand, an exponent uniform in [emin, emax] and a random sign; one draw in 256 has a
// small-integer numerator (exact quotients, signed zeros), one in 256 a divisor with an all-ones
// significand, and one in 64 a special operand (+-0, +-inf, NaN) on either side.
#include <cuda_runtime.h>

#include <cstdint>

#include "../csrc/ecg_ieee.cuh"

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double draw(uint64_t h, int emin, int emax) {
  const uint64_t m = h & 0xFFFFFFFFFFFFFull;
  const int e = emin + (int)((h >> 52) % (uint64_t)(emax - emin + 1));
  uint64_t bits = m | ((uint64_t)(e + 1023) << 52);
  if (mix64(h) & 1) bits |= 0x8000000000000000ull;
  return __longlong_as_double((long long)bits);
}

__device__ __forceinline__ double special(uint64_t h) {
  const long long v[6] = {0ll, (long long)0x8000000000000000ull, 0x7ff0000000000000ll,
                          (long long)0xfff0000000000000ull, 0x7ff8000000000000ll, 0x3ff0000000000000ll};
  return __longlong_as_double(v[h % 6]);
}

__device__ __forceinline__ bool same(double x, double y) {
  // NaNs compare equal whatever their payload
  return (x != x && y != y) || __double_as_longlong(x) == __double_as_longlong(y);
}

__global__ void k_ieee_check(uint64_t seed, int emin, int emax, int iters, unsigned long long* out) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long nd = 0, ns = 0, n = 0;
  for (int it = 0; it < iters; it++) {
    const uint64_t h1 = mix64(seed ^ (t * 0x100000001B3ull + (uint64_t)it));
    const uint64_t h2 = mix64(h1 + 0x2545F4914F6CDD1Dull);
    double a = draw(h1, emin, emax), b = draw(h2, emin, emax);
    const uint64_t h3 = mix64(h2);
    if ((h3 & 255) == 0) a = (double)((h3 >> 8) & 1023) * 0.25 - 64.;
    if (((h3 >> 20) & 255) == 1) b = __longlong_as_double(__double_as_longlong(b) | 0xFFFFFFFFFFFFFll);
    if (((h3 >> 30) & 63) == 2) a = special(h3 >> 40);
    if (((h3 >> 36) & 63) == 3) b = special(h3 >> 44);
    n++;
    if (!same(a / b, ecg::ddiv(a, b))) nd++;
    if (!same(sqrt(a), ecg::dsqrt(a))) ns++;
  }
  atomicAdd(out, n);
  if (nd) atomicAdd(out + 1, nd);
  if (ns) atomicAdd(out + 2, ns);
}

}  // namespace

extern "C" {

// Runs the check on the current device: blocks x 256 threads x iters operand pairs with exponents in
// [emin, emax] (-500 <= emin <= emax <= 500, so that every quotient of finite operands is a normal
// number).  Writes counts[0] = pairs checked, counts[1] = divisions and counts[2] = square roots that
// differ from CUDA's.  Returns 0 on success, otherwise the CUDA error code, or -1 for arguments outside
// the limits.
int ecg_probe_ieee_check(unsigned long long seed, int emin, int emax, int blocks, int iters,
                         unsigned long long counts[3]) {
  if (emin < -500 || emax > 500 || emin > emax || blocks <= 0 || iters <= 0) return -1;
  unsigned long long* d = nullptr;
  cudaError_t e = cudaMalloc(&d, 3 * sizeof(unsigned long long));
  if (e != cudaSuccess) return (int)e;
  e = cudaMemset(d, 0, 3 * sizeof(unsigned long long));
  if (e == cudaSuccess) {
    k_ieee_check<<<blocks, 256>>>(seed, emin, emax, iters, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(counts, d, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return (int)e;
}

}  // extern "C"
