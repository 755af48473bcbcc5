// Host-side helpers shared by the library's translation units.
#pragma once
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/ecogen_b200.h"

namespace ecg {

void set_error(const std::string& msg);

// Checks a case against what the library runs; ECG_OK, or the status and message of the first
// violation (ecg_create and ecg_step_noalloc accept the same cases).
ecg_status validate_case(const ecg_case* c);

// Cell sizes and centres along one axis of a case: MeshCartesian::meshStretching
// src/Meshes/MeshCartesian.cpp:168-210 (uniform: length / n and (i + 0.5) d) with stretchZone::stretching
// src/Meshes/stretchZone.cpp:45-66 for each zone of a stretched axis (geometric progression of ratio
// factor, or uniform when |factor - 1| < 1e-6).  Same arithmetic as the reference, operation for
// operation (std::pow), so the sizes and centres carry the reference's bits.
inline void axis_cells(const ecg_case& c, int ax, std::vector<double>& d, std::vector<double>& pos) {
  const int n = c.ncells[ax];
  d.clear();
  pos.clear();
  if (c.nstretch[ax] == 0 || n == 1) {
    const double dd = c.length[ax] / static_cast<double>(n);
    for (int i = 0; i < n; i++) {
      d.push_back(dd);
      pos.push_back((i + 0.5) * dd);
    }
    return;
  }
  for (int z = 0; z < c.nstretch[ax]; z++) {
    const ecg_stretch_zone& st = c.stretch[ax][z];
    double dX0 = (st.end - st.start) / st.ncells;
    if (std::fabs(st.factor - 1.) < 1e-6) {
      for (int i = 0; i < st.ncells; i++) {
        d.push_back(dX0);
        pos.push_back(st.start + (i + 0.5) * dX0);
      }
    } else {
      dX0 = (st.end - st.start) * (1. - st.factor) / (1. - std::pow(st.factor, st.ncells));
      d.push_back(dX0);
      pos.push_back(st.start + 0.5 * dX0);
      size_t k = pos.size();
      for (int i = 1; i < st.ncells; i++) {
        d.push_back(dX0 * std::pow(st.factor, i));
        pos.push_back(pos[k - 1] + 0.5 * (d[k - 1] + d[k]));
        k++;
      }
    }
  }
}

// Whether any axis of the case is stretched.
inline bool case_stretched(const ecg_case& c) {
  for (int a = 0; a < 3; a++)
    if (c.nstretch[a] > 0 && c.ncells[a] > 1) return true;
  return false;
}

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
