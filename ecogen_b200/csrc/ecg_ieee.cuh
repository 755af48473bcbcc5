// Branch-free IEEE-754 binary64 division and square root for the step kernels.
//
// CUDA's `a / b` and `sqrt(x)` on doubles are correctly rounded (round to nearest even).  They are
// computed from a hardware reciprocal (or reciprocal square root) approximation, Newton steps and a
// final correction, with a test for operands the fast sequence cannot handle and a branch to a
// slower routine for them.  That branch ends a basic block at every division, so the compiler cannot
// interleave independent divisions: in the face and cell kernels (about fifty divisions and eight
// square roots per face of a three-phase case, FP64-latency-bound) consecutive divisions run one
// after another.  ddiv / dsqrt return the same correctly rounded results from straight-line code:
//
//   ddiv(a, b): y0 = rcp.approx(b) (relative error below 2^-19.9, measured on B200 over 2.5e9
//     operands), three Newton steps y += y (1 - b y) with fused multiply-adds, so that the last one
//     starts within one ulp of 1/b and returns RN(1/b) (Markstein's reciprocal theorem), except for a
//     divisor whose significand is all ones, 2^e (2 - 2^-52): there 1/b lies just above the midpoint
//     of its two neighbours and every step from either of them rounds a tie to the lower one, so y is
//     moved up by one ulp; then q = RN(a y), the exact remainder r = a - b q (one FMA) and
//     RN(q + r y), which is RN(a / b) when y = RN(1/b) and q is within one ulp of a / b (Markstein's
//     division theorem, P. Markstein, "Computation of elementary functions on the IBM RISC
//     System/6000 processor", IBM J. Res. Dev. 34(1), 1990).  The sign of a zero quotient is taken
//     from q (the sign of a b).
//   dsqrt(x): y0 = rsqrt.approx(x), two coupled Newton steps on g ~ sqrt(x) and h ~ 1/(2 sqrt(x)),
//     then the exact residual d = x - g^2 (one FMA) and RN(g + d h) (the same correction scheme).
//
// Operands outside the normal range: a zero, infinite or NaN divisor or dividend makes the Newton
// sequence NaN, and then the raw product a * rcp.approx(b), which is IEEE's answer there (+-inf, +-0
// or NaN), is returned; dsqrt returns x for +-0 and +inf and NaN for x < 0.  What is not reproduced:
// subnormal operands and results (the approximations flush them to zero) and divisors above 2^1022 in
// magnitude, far outside every quantity of the step (densities, pressures, velocities, energies, cell
// sizes).
//
// Both functions are checked against `/` and `sqrt()` bit for bit on hashed operands with exponents
// from -500 to 500, exact quotients, all-ones-significand divisors and zero, infinite and NaN operands
// (tests/test_gpu_ieee.py, 3e8 pairs per run; 2.5e9 when the method was chosen), and every parity
// test of the step kernels compares their fields with the oracle, which divides with the host's IEEE
// division.
#pragma once

namespace ecg {

__device__ __forceinline__ double rcp_approx(double b) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  return y;
}

__device__ __forceinline__ double rsqrt_approx(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return y;
}

// a / b, correctly rounded (see above)
__device__ __forceinline__ double ddiv(double a, double b) {
  const double y0 = rcp_approx(b);
  const double q0 = a * y0;  // IEEE's result when a or b is zero, infinite or NaN
  double e = fma(-b, y0, 1.0);
  double y = fma(y0, e, y0);
  e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  // a divisor whose significand is all ones: the last step lands on a tie and settles one ulp below
  // RN(1/b), so y is moved up by one ulp (a select, no branch)
  const long long bb = __double_as_longlong(b);
  y = __longlong_as_double(__double_as_longlong(y) + ((bb & 0xFFFFFFFFFFFFFll) == 0xFFFFFFFFFFFFFll ? 1 : 0));
  const double q = a * y;
  const double r = fma(-b, q, a);
  const double q1 = copysign(fma(r, y, q), q);
  return (q1 == q1) ? q1 : q0;  // NaN only when an operand is zero, infinite or NaN
}

// sqrt(x), correctly rounded (see above)
__device__ __forceinline__ double dsqrt(double x) {
  const double y0 = rsqrt_approx(x);
  double g = x * y0, h = 0.5 * y0;
  double r = fma(-g, h, 0.5);
  g = fma(g, r, g);
  h = fma(h, r, h);
  r = fma(-g, h, 0.5);
  g = fma(g, r, g);
  h = fma(h, r, h);
  const double d = fma(-g, g, x);
  const double s = fma(d, h, g);
  const bool normal = (x > 0.) && (x < __longlong_as_double(0x7ff0000000000000ll));
  return normal ? s : ((x < 0.) ? __longlong_as_double(0x7ff8000000000000ll) : x);
}

}  // namespace ecg
