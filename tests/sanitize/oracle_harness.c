/* The oracle (oracle/ecg_oracle.c) under AddressSanitizer / UndefinedBehaviorSanitizer -- TEST
 * INFRASTRUCTURE (tests/test_sanitizers.py builds and runs it on the CPU).
 *
 *   oracle_harness <blob> <steps>
 * <blob>: the ecgo_case record, then int64 n, then alpha[np*n], rho[np*n], p[n], u[3*n] (the initial
 * state oracle.py passes to ecgo_create).  Runs <steps> steps and prints the sum of the output fields
 * with 17 digits, which the test compares with the same run of the regular oracle build. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "ecg_oracle.h"

static int read_all(FILE* f, void* p, size_t n) { return fread(p, 1, n, f) == n; }

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  ecgo_case c;
  int64_t n = 0;
  if (!read_all(f, &c, sizeof c) || !read_all(f, &n, sizeof n) || n <= 0 || c.nphases < 1 || c.nphases > 3) return 2;
  const int np = c.nphases;
  double* a = malloc(sizeof(double) * np * n);
  double* r = malloc(sizeof(double) * np * n);
  double* p = malloc(sizeof(double) * n);
  double* u = malloc(sizeof(double) * 3 * n);
  if (!read_all(f, a, sizeof(double) * np * n) || !read_all(f, r, sizeof(double) * np * n) ||
      !read_all(f, p, sizeof(double) * n) || !read_all(f, u, sizeof(double) * 3 * n))
    return 2;
  fclose(f);
  ecgo_sim* S = ecgo_create(&c, a, r, p, u, NULL);
  if (!S) return 3;
  double dt = 1e-15, t = 0.;
  ecgo_stats st;
  ecgo_step(S, atoi(argv[2]), &dt, &t, &st);
  double* oa = malloc(sizeof(double) * np * n);
  double* orr = malloc(sizeof(double) * np * n);
  double* oT = malloc(sizeof(double) * np * n);
  double* oY = malloc(sizeof(double) * np * n);
  double* orm = malloc(sizeof(double) * n);
  double* op = malloc(sizeof(double) * n);
  double* oE = malloc(sizeof(double) * n);
  double* ou = malloc(sizeof(double) * 3 * n);
  ecgo_get(S, oa, orr, oT, oY, orm, op, oE, ou);
  double sum = 0.;
  for (int64_t i = 0; i < np * n; i++) sum += oa[i] + orr[i];
  for (int64_t i = 0; i < n; i++) sum += op[i] + oE[i];
  for (int64_t i = 0; i < 3 * n; i++) sum += ou[i];
  printf("%.17g %.17g\n", sum, dt);
  ecgo_destroy(S);
  free(a); free(r); free(p); free(u);
  free(oa); free(orr); free(oT); free(oY); free(orm); free(op); free(oE); free(ou);
  return 0;
}
