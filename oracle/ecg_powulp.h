/* pow with last-ulp changes, for the oracle's second sensitivity variant -- TEST INFRASTRUCTURE.
 *
 * The reference evaluates pow in the isentropic star pressure of HLLC (EosIG/SG/NASG::
 * computePressureIsentropic, src/Eos/EosSG.cpp:129-132) with the host libm; the GPU path uses CUDA's
 * pow, whose result can differ from the host's in the last bit.  A build of the oracle with this
 * function in place of pow (libecg_oracle_powulp.so) moves the result of 1 call in 100 by one ulp,
 * up or down, chosen by a hash of the arguments (deterministic), and so measures how far the scheme
 * carries last-ulp differences of pow: the spread a different faithful pow leaves after N steps. */
#ifndef ECG_POWULP_H
#define ECG_POWULP_H
#include <math.h>
#include <stdint.h>
#include <string.h>

static double ecgo_pow_ulp(double x, double y) {
  double r = pow(x, y);
  uint64_t hx, hy;
  memcpy(&hx, &x, 8);
  memcpy(&hy, &y, 8);
  uint64_t h = hx ^ (hy * 0x9E3779B97F4A7C15ull);
  h ^= h >> 33;
  h *= 0xff51afd7ed558ccdull;
  h ^= h >> 33;
  if (h % 100ull == 0ull && isfinite(r)) r = nextafter(r, (h & (1ull << 40)) ? INFINITY : -INFINITY);
  return r;
}
#endif
