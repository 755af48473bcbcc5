// Host build of the table-driven pow of the step kernels (ecogen_b200/csrc/ecg_pow.cuh), for the tests:
// the same source compiled for the CPU, beside the host libm's pow, over arrays.
#include "../../ecogen_b200/csrc/ecg_pow.cuh"

extern "C" {

void host_epow(const double* x, const double* y, double* out, long n) {
  for (long i = 0; i < n; i++) out[i] = ecg::epow(x[i], y[i]);
}

void host_libm_pow(const double* x, const double* y, double* out, long n) {
  for (long i = 0; i < n; i++) out[i] = std::pow(x[i], y[i]);
}

}  // extern "C"

extern "C" {

// ln x by elog (the first stage of epow, rounded once), and the host libm's log
void host_elog(const double* x, double* out, long n) {
  for (long i = 0; i < n; i++) {
    out[i] = ecg::elog(x[i]);
  }
}

void host_libm_log(const double* x, double* out, long n) {
  for (long i = 0; i < n; i++) out[i] = std::log(x[i]);
}

}  // extern "C"
