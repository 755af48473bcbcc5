// Table-driven x^y for the isentropic star-state pressures of the HLLC solver, and ln x for the
// saturation solve of the p-T-mu relaxation (elog, below).
//
// The HLLC star state evaluates p0 (rho*/rho0)^gamma per phase (EosSG::computePressureIsentropic
// src/Eos/EosSG.cpp, EosIG.cpp likewise), three times per face in a three-phase case.  CUDA's double
// pow costs about 80 FP64 and 130 other instructions per call (measured with ncu on B200), a fifth
// of the face kernel's FP64 work.  epow computes x^y = exp(y ln x) by Tang's table-driven method
// (P. T. P. Tang, "Table-driven implementation of the exponential function in IEEE floating-point
// arithmetic", ACM TOMS 15(2), 1989, and "... of the logarithm function", ACM TOMS 16(4), 1990), with
// the logarithm carried as a double-double so that the result is rounded once:
//
//   ln x   x = 2^k m, m in [1, 2); row i of a 128-row table (the top 7 bits of m) gives inv_i, a
//          multiple of 2^-8 near 1 / m, and -ln(inv_i) as hi + lo; r = m inv_i - 1 is exact (one FMA,
//          |r| < 2^-7) and ln x = k ln2 + (-ln inv_i) + ln(1 + r), with ln(1 + r) = r - r^2/2 +
//          r^3 P(r), P the Taylor polynomial to r^9 (truncation below 2^-66 relative to r); the large
//          terms are added with error-free two-sums, the rest in double, to L = Lh + Ll, accurate to
//          about 2^-68 absolutely.
//   exp    Y = y L as Yh + Yl (one FMA for the product's error); kd = round(Yh 128 / ln2), rh = Yh -
//          kd C1 exactly (C1 = RN(ln2/128)), rl = Yl - kd C2; exp(Y) = 2^(kd/128) exp(rh + rl) with
//          2^(j/128) from a 128-row table as hi + lo and exp(rh) - 1 by its Taylor polynomial to rh^6
//          (|rh| <= ln2/256, truncation below 2^-71); the leading product T rh is split exactly, the
//          sum rounded once, and 2^(kd >> 7) applied to the exponent field.
//
// Accuracy: the result before its one rounding is within about 2^-64 of x^y (relative), so it is the
// correctly rounded x^y except when x^y lies within that distance of a midpoint between doubles.
// Measured on 2.4e8 arguments (x log-uniform in [1e-6, 1e6], y in {1.4, 1.43, 1.67, 2.35, 4.4, 7.15}):
// epow differs from the host glibc pow (the reference's and the oracle's) in 0.08 % of the calls, by
// one ulp, and in every one of those that were checked against 300-bit arithmetic it is epow that is
// correctly rounded (glibc's pow is accurate to about 0.5 + 2^-7 ulp).  tests/test_pow.py checks this header's
// host build against glibc and 300-bit arithmetic, tests/test_gpu_pow.py the device build against the host
// build bit for bit.
//
// Domain: x in [2^-60, 2^60] and 0 < y <= 10, which holds every density ratio and EOS gamma of the
// step; any other argument (zero, negative, infinite, NaN, far outside that range) goes to CUDA's pow,
// which keeps its special values.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
// inlining of epow itself (three call sites per face in a three-phase case): build-time choice
#ifndef ECG_EPOW_INLINE
#define ECG_EPOW_INLINE __forceinline__
#endif
#define ECG_EPOW_FN static __device__ ECG_EPOW_INLINE  // internal linkage: one copy per unit when not inlined
#define ECG_POW_FN __device__ __forceinline__
#define ECG_POW_TABLE static __device__ const
#define ECG_POW_LD(p) __ldg(p)
#else
#define ECG_POW_FN static inline
#define ECG_EPOW_FN static inline
#define ECG_POW_TABLE static const
#define ECG_POW_LD(p) (*(p))
#endif

#include "ecg_pow_tables.h"

namespace ecg {

#if defined(__CUDACC__)
ECG_POW_FN uint64_t pow_bits(double d) { return (uint64_t)__double_as_longlong(d); }
ECG_POW_FN double pow_double(uint64_t b) { return __longlong_as_double((long long)b); }
ECG_POW_FN double pow_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
static __device__ __noinline__ double pow_outside(double x, double y) { return pow(x, y); }
static __device__ __noinline__ double log_outside(double x) { return log(x); }
#else
ECG_POW_FN uint64_t pow_bits(double d) {
  uint64_t b;
  std::memcpy(&b, &d, 8);
  return b;
}
ECG_POW_FN double pow_double(uint64_t b) {
  double d;
  std::memcpy(&d, &b, 8);
  return d;
}
ECG_POW_FN double pow_fma(double a, double b, double c) { return std::fma(a, b, c); }
ECG_POW_FN double pow_outside(double x, double y) { return std::pow(x, y); }
ECG_POW_FN double log_outside(double x) { return std::log(x); }
#endif

// ln x as a double-double Lh + Ll (x positive and normal), the first stage of epow (see above)
ECG_POW_FN void epow_log(double x, double& Lh, double& Ll) {
  const uint64_t ix = pow_bits(x);
  const int k = (int)(ix >> 52) - 1023;
  const int i = (int)((ix >> 45) & 127);
  const double m = pow_double((ix & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
  const double inv = ECG_POW_LD(&ecg_pow_logt[i][0]), th = ECG_POW_LD(&ecg_pow_logt[i][1]),
               tl = ECG_POW_LD(&ecg_pow_logt[i][2]);
  const double r = pow_fma(m, inv, -1.0);  // exact
  const double kd0 = (double)k;
  // t1 + e1 = k L2H + th (two-sum), t2 + e2 = t1 + r and t3 + e3 = t2 - r^2/2 (fast two-sums: |t1|
  // >= |r| unless t1 = 0, and |r^2/2| <= |r|^2)
  const double a1 = kd0 * ECG_POW_L2H;
  const double t1 = a1 + th, bb = t1 - a1, e1 = (a1 - (t1 - bb)) + (th - bb);
  const double t2 = t1 + r, e2 = r - (t2 - t1);
  const double r2 = r * r, r2l = pow_fma(r, r, -r2);
  const double hr2 = -0.5 * r2;
  const double t3 = t2 + hr2, e3 = hr2 - (t3 - t2);
  double p = pow_fma(r, 1. / 9., -1. / 8.);
  p = pow_fma(p, r, 1. / 7.);
  p = pow_fma(p, r, -1. / 6.);
  p = pow_fma(p, r, 1. / 5.);
  p = pow_fma(p, r, -0.25);
  p = pow_fma(p, r, 1. / 3.);
  const double lo = e1 + e2 + e3 + (kd0 * ECG_POW_L2L + tl) - 0.5 * r2l + (r2 * r) * p;
  Lh = t3 + lo;
  Ll = lo - (Lh - t3);
}

// ln x rounded once from the double-double of epow_log: the correctly rounded logarithm except within
// the double-double's error (about 2^-75 relative) of a midpoint.  Measured against the host glibc log:
// identical on 8e6 arguments in [50, 2000] and [1e3, 1e10] (the saturation solve's temperatures and
// pressures), different by one ulp in 1 call in 700 for x in [0.5, 2], where glibc's log is the one not
// correctly rounded (300-bit arithmetic); tests/test_pow.py.  x outside the positive normal range goes to
// the library's log.
ECG_POW_FN double elog(double x) {
  if (!(x >= 0x1p-1022 && x <= 0x1.fffffffffffffp1023)) return log_outside(x);
  double Lh, Ll;
  epow_log(x, Lh, Ll);
  return Lh;
}

// x^y by the tables (see above); pow_fma is the fused multiply-add of the device or of the host libm
ECG_EPOW_FN double epow(double x, double y) {
  if (!(x >= 0x1p-60 && x <= 0x1p60 && y > 0. && y <= 10.)) return pow_outside(x, y);
  double Lh, Ll;
  epow_log(x, Lh, Ll);
  // ---- Y = y ln x = Yh + Yl
  const double Yh = y * Lh;
  const double Yl = pow_fma(y, Lh, -Yh) + y * Ll;
  // ---- exp(Y) = 2^(ki / 128) exp(rh + rl)
  const double SHIFT = 0x1.8p52;
  const double t = pow_fma(Yh, ECG_POW_INVC, SHIFT);
  const double kd = t - SHIFT;
  const int ki = (int)(uint32_t)(pow_bits(t) & 0xFFFFFFFFull);
  const double rh = pow_fma(-kd, ECG_POW_C1, Yh);  // exact
  const double rl = pow_fma(-kd, ECG_POW_C2, Yl);
  const int j = ki & 127;
  const int e = ki >> 7;
  const double Th = ECG_POW_LD(&ecg_pow_expt[j][0]), Tl = ECG_POW_LD(&ecg_pow_expt[j][1]);
  double q = pow_fma(rh, 1. / 720., 1. / 120.);
  q = pow_fma(q, rh, 1. / 24.);
  q = pow_fma(q, rh, 1. / 6.);
  q = pow_fma(q, rh, 0.5);
  q = q * (rh * rh);
  const double bh = Th * rh, bl = pow_fma(Th, rh, -bh);
  const double s = Th + bh, se = bh - (s - Th);
  const double small = se + bl + Th * (rl + rh * rl + q) + Tl + Tl * rh;
  const double res = s + small;
  return pow_double(pow_bits(res) + ((uint64_t)(int64_t)e << 52));
}

}  // namespace ecg
