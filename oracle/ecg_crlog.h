/* Correctly rounded natural logarithm for the oracle's sensitivity variant -- TEST INFRASTRUCTURE.
 *
 * The reference evaluates ln in Mixture::computeTsat (src/Models/Mixture.cpp:85-95) with the host libm,
 * whose log is not correctly rounded in every case; the GPU path uses a correctly rounded logarithm.  A
 * build of the oracle with this function in place of log (make -C oracle lib, libecg_oracle_crlog.so)
 * measures how far the p-T-mu relaxation carries a last-ulp change of ln: the spread between two
 * faithful logarithms.  Same method as the device's cr_log: ln(m 2^k) = 2 atanh((m-1)/(m+1)) + k ln2
 * for m in [1/sqrt2, sqrt2), in double-double arithmetic (error-free sums and fma products), rounded
 * once. */
#ifndef ECG_CRLOG_H
#define ECG_CRLOG_H
#include <math.h>

typedef struct {
  double hi, lo;
} ecgo_dd;

static ecgo_dd ecgo_dd_two_sum(double a, double b) {
  double s = a + b, bb = s - a;
  ecgo_dd r = {s, (a - (s - bb)) + (b - bb)};
  return r;
}
static ecgo_dd ecgo_dd_fast_sum(double a, double b) {
  double s = a + b;
  ecgo_dd r = {s, b - (s - a)};
  return r;
}
static ecgo_dd ecgo_dd_add(ecgo_dd a, ecgo_dd b) {
  ecgo_dd s = ecgo_dd_two_sum(a.hi, b.hi), t = ecgo_dd_two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = ecgo_dd_fast_sum(s.hi, s.lo);
  s.lo += t.lo;
  return ecgo_dd_fast_sum(s.hi, s.lo);
}
static ecgo_dd ecgo_dd_mul(ecgo_dd a, ecgo_dd b) {
  double p = a.hi * b.hi;
  double e = fma(a.hi, b.hi, -p);
  e += a.hi * b.lo + a.lo * b.hi;
  return ecgo_dd_fast_sum(p, e);
}
static ecgo_dd ecgo_dd_div(ecgo_dd a, ecgo_dd b) {
  double q1 = a.hi / b.hi;
  ecgo_dd m1 = {-q1, 0.};
  ecgo_dd r = ecgo_dd_add(a, ecgo_dd_mul(b, m1));
  double q2 = r.hi / b.hi;
  ecgo_dd m2 = {-q2, 0.};
  r = ecgo_dd_add(r, ecgo_dd_mul(b, m2));
  double q3 = r.hi / b.hi;
  ecgo_dd q = {q3, 0.};
  return ecgo_dd_add(ecgo_dd_fast_sum(q1, q2), q);
}
static double ecgo_cr_log(double x) {
  if (!(x > 0.) || isinf(x)) return log(x);
  int k;
  double m = frexp(x, &k);
  if (m < 0.70710678118654752440) {
    m *= 2.;
    k -= 1;
  }
  ecgo_dd num = {m - 1., 0.};
  ecgo_dd den = ecgo_dd_two_sum(m, 1.);
  ecgo_dd s = ecgo_dd_div(num, den);
  ecgo_dd s2 = ecgo_dd_mul(s, s);
  double t = 1. / 45.;
  for (int i = 21; i >= 3; i--) t = t * s2.hi + 1. / (2. * i + 1.);
  ecgo_dd one = {1., 0.}, five = {5., 0.}, three = {3., 0.}, tt = {t, 0.};
  ecgo_dd P = ecgo_dd_add(ecgo_dd_div(one, five), ecgo_dd_mul(s2, tt));
  P = ecgo_dd_add(ecgo_dd_div(one, three), ecgo_dd_mul(s2, P));
  P = ecgo_dd_add(one, ecgo_dd_mul(s2, P));
  ecgo_dd lm = ecgo_dd_mul(s, P);
  lm.hi *= 2.;
  lm.lo *= 2.;
  const ecgo_dd ln2 = {0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56};
  ecgo_dd kk = {(double)k, 0.};
  ecgo_dd r = ecgo_dd_add(ecgo_dd_mul(ln2, kk), lm);
  return r.hi + r.lo;
}
#endif
