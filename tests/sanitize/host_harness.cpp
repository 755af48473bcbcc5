// Host-side checks of the library's case input code under AddressSanitizer / UndefinedBehaviorSanitizer
// -- TEST INFRASTRUCTURE (tests/test_sanitizers.py builds and runs it on the CPU).
//
// Links the host translation units of the C ABI that need no GPU -- the XML reader (ecg_xml.cpp), the
// case reader, initial fill and restart fill (ecg_input.cpp), the case checks (ecg_case.cpp) -- and
// drives them over case folders: read, check, fill, and for a folder that must be refused, the status.
//   host_harness ok <case_dir> <eos_dir> <out> read + check + fill; prints "ok <n>" and writes the filled
//                                              fields (field after field, n doubles each) to <out>
//   host_harness refuse <case_dir> <eos_dir>   expects a non-OK status; prints "refused <status>"
//   host_harness restart <case_dir> <eos_dir> <out>  the same, then ecg_restart_fill over the filled fields
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

extern "C" {
#include "ecogen_b200.h"
}
#include "ecg_internal.h"

namespace ecg {
static std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
}  // namespace ecg

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: host_harness ok|refuse|restart <case_dir> <eos_dir> [out]\n");
    return 2;
  }
  const std::string mode = argv[1];
  ecg_input* in = nullptr;
  ecg_status s = ecg_input_read(argv[2], argv[3], &in);
  ecg_case c;
  if (s == ECG_OK) s = ecg_input_case(in, &c);
  if (s == ECG_OK) s = ecg::validate_case(&c);
  if (mode == "refuse") {
    ecg_input_free(in);
    std::printf("refused %d\n", (int)s);
    return s == ECG_OK ? 1 : 0;
  }
  if (s != ECG_OK) {
    std::printf("error %d\n", (int)s);
    ecg_input_free(in);
    return 1;
  }
  const int64_t n = (int64_t)c.ncells[0] * c.ncells[1] * c.ncells[2];
  const int nf = ecg::abi_nfields(c);
  std::vector<std::vector<double>> f(nf, std::vector<double>((size_t)n));
  std::vector<double*> ptr;
  for (auto& v : f) ptr.push_back(v.data());
  s = ecg_input_fill(in, ptr.data(), n);
  if (s == ECG_OK && mode == "restart") s = ecg_restart_fill(&c, ptr.data(), n);
  int32_t freq = 0, bin = 0, prec = 0, rf = 0;
  double tf = 0.;
  if (s == ECG_OK) s = ecg_input_print_control(in, &freq, &tf);
  if (s == ECG_OK) s = ecg_input_output_control(in, &bin, &prec, &rf);
  for (int k = 0; s == ECG_OK && k < c.nphases; k++)
    if (!ecg_input_eos_name(in, k)) s = ECG_ERR_INVALID;
  ecg_input_free(in);
  if (s != ECG_OK) {
    std::printf("error %d\n", (int)s);
    return 1;
  }
  if (argc > 4) {
    FILE* o = std::fopen(argv[4], "wb");
    if (!o) return 1;
    for (auto& v : f) std::fwrite(v.data(), sizeof(double), v.size(), o);
    std::fclose(o);
  }
  std::printf("ok %lld\n", (long long)n);
  return 0;
}
