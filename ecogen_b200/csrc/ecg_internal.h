// Host-side helpers shared by the library's translation units.
#pragma once
#include <algorithm>
#include <string>

#include "../../include/ecogen_b200.h"

namespace ecg {

void set_error(const std::string& msg);

// Checks a case against what the library runs; ECG_OK, or the status and message of the first
// violation (ecg_create and ecg_step_noalloc accept the same cases).
ecg_status validate_case(const ecg_case* c);

struct DevStats;
// Host copy of the device counters of a step call -> the ABI record (cell_updates = updates).
void stats_out(const DevStats& d, int64_t updates, ecg_step_stats* st);

// Number of field pointers in the ABI layout of a case (see include/ecogen_b200.h).
inline int abi_nfields(const ecg_case& c) {
  if (c.model == ECG_MODEL_EULER) return 6 + c.ntransports;
  if (c.model == ECG_MODEL_PTUEQ) return 2 * c.nphases + 6 + c.ntransports;  // + the mixture temperature
  return 2 * c.nphases + 5 + c.ntransports;
}

// EOS internal energy e(rho, p), same expression as the kernels and the reference EOS classes.
inline double host_eos_e(const ecg_eos& q, double eps, double rho, double p) {
  if (q.type == ECG_EOS_IG) return p / (q.gamma - 1.) / std::max(rho, eps) + q.eref;
  if (q.type == ECG_EOS_SG) return (p + q.gamma * q.pinf) / (q.gamma - 1.) / std::max(rho, eps) + q.eref;
  return (p + q.gamma * q.pinf) * std::max(1. - rho * q.b, eps) / (q.gamma - 1.) / std::max(rho, eps) + q.eref;
}

// Eos::verifyAndModifyPressure (EosIG.cpp, EosSG.cpp, EosNASG.cpp): pressure floors.
inline double host_eos_fix_p(const ecg_eos& q, double p) {
  if (q.type == ECG_EOS_IG) return (p < 1.e-8) ? 1.e-8 : p;
  double floor = -(1. - 1.e-15) * q.pinf + 1.e-15;
  return (p <= floor) ? floor : p;
}

}  // namespace ecg
