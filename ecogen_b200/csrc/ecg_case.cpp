// Checks of a case against what the library runs: host code shared by ecg_create, the allocation-free
// step and the batched mode (declared in ecg_internal.h).  The messages follow the reference's input
// errors where the reference has one (Input::inputMesh / inputModel, src/InputOutput/Input.cpp).
#include <cstdint>

#include "ecg_internal.h"

namespace ecg {

// Checks a case against what the library runs (ecg_create and ecg_step_noalloc accept the same cases).
ecg_status validate_case(const ecg_case* c) {
  if (!c) { set_error("null case"); return ECG_ERR_INVALID; }
  if (c->model != ECG_MODEL_KAPILA && c->model != ECG_MODEL_EULER && c->model != ECG_MODEL_PTUEQ) { set_error("unknown model"); return ECG_ERR_INVALID; }
  if (c->model == ECG_MODEL_PTUEQ) {
    // MixPTUEq::computePressure: two phases, IG or SG (src/Models/PTUEq/MixPTUEq.cpp:96-99)
    if (c->nphases != 2) { set_error("the temperature-pressure equilibrium model has two phases"); return ECG_ERR_UNSUPPORTED; }
    for (int k = 0; k < 2; k++)
      if (c->eos[k].type == ECG_EOS_NASG) { set_error("Only IG and SG permitted in thermal equilibrium model"); return ECG_ERR_UNSUPPORTED; }
    if (c->ntransports) { set_error("solveRiemannTransportIntern not available for the temperature-pressure equilibrium model"); return ECG_ERR_UNSUPPORTED; }
    if (c->ptmu || c->pt_relaxation) { set_error("relaxations of the temperature-pressure equilibrium model"); return ECG_ERR_UNSUPPORTED; }
    if (c->alpha_null) { set_error("alphaNull is not an option of the temperature-pressure equilibrium model"); return ECG_ERR_INVALID; }
    if (c->order == 2)
      for (int i = 0; i < 6; i++)  // BoundCondWallO2Cartesian::computeSlopes sets phase velocity slopes PhasePTUEq lacks
        if (c->bc[i] == ECG_BC_SYMMETRY) { set_error("MUSCL symmetry sides of the temperature-pressure equilibrium model (setU not available)"); return ECG_ERR_UNSUPPORTED; }
  }
  if (c->model == ECG_MODEL_KAPILA && (c->nphases < 2 || c->nphases > 3)) { set_error("Kapila needs 2 or 3 phases"); return ECG_ERR_UNSUPPORTED; }
  if (c->model == ECG_MODEL_EULER && c->nphases != 1) { set_error("Euler has one phase"); return ECG_ERR_INVALID; }
  if (c->order != 1 && c->order != 2) { set_error("order must be 1 or 2"); return ECG_ERR_INVALID; }
  for (int i = 0; i < 3; i++)
    if (c->ncells[i] < 1 || !(c->length[i] > 0.)) { set_error("bad mesh"); return ECG_ERR_INVALID; }
  if (c->ncells[0] <= 1) { set_error("Number of cells in the x-direction has to be superior to 1"); return ECG_ERR_INVALID; }
  if (c->ncells[2] > 1 && c->ncells[1] <= 1) { set_error("z cells without y cells"); return ECG_ERR_INVALID; }
  for (int i = 0; i < 4; i++)
    if (c->limiter[i] < 0 || c->limiter[i] > ECG_LIM_THINC) { set_error("bad limiter"); return ECG_ERR_INVALID; }
  
  for (int i = 0; i < 6; i++)
    if (c->bc[i] != ECG_BC_NONREFLECTING && c->bc[i] != ECG_BC_SYMMETRY) { set_error("bad boundary condition"); return ECG_ERR_INVALID; }
  if (c->ntransports < 0) { set_error("negative number of transports"); return ECG_ERR_INVALID; }
  if (c->ntransports > 2) { set_error("more than two passive transports"); return ECG_ERR_UNSUPPORTED; }
  if (c->pt_relaxation) {
    if (c->model != ECG_MODEL_KAPILA || c->nphases != 2 || c->ptmu) { set_error("PT relaxation: two Kapila phases, without PTMu"); return ECG_ERR_UNSUPPORTED; }
    for (int k = 0; k < 2; k++)
      if (c->eos[k].type == ECG_EOS_NASG) { set_error("PT relaxation needs IG or SG phases"); return ECG_ERR_UNSUPPORTED; }
  }
  if (c->ptmu && (c->model != ECG_MODEL_KAPILA || c->nphases != 2)) { set_error("PTMu needs two phases"); return ECG_ERR_INVALID; }
  if (c->ptmu) {
    if (c->ptmu_liquid < 0 || c->ptmu_liquid > 1 || c->ptmu_vapor < 0 || c->ptmu_vapor > 1 ||
        c->ptmu_liquid == c->ptmu_vapor) { set_error("PTMu liquid / vapour phase indices"); return ECG_ERR_INVALID; }
    // Mixture::computeTsat (src/Models/Mixture.cpp:62-63): IG and SG phases only
    for (int k = 0; k < 2; k++)
      if (c->eos[k].type == ECG_EOS_NASG) { set_error("Only IG and SG permitted in thermal equilibrium model: MixPTUEq::computeTsat"); return ECG_ERR_UNSUPPORTED; }
  }
  int dim = (c->ncells[0] != 1) + (c->ncells[1] != 1) + (c->ncells[2] != 1);
  if (c->ptmu && dim == 3) { set_error("PTMu on 3D meshes is not built"); return ECG_ERR_UNSUPPORTED; }
  for (int a = 0; a < 3; a++) {  // mesh stretching (stretchZone::verifyStretching src/Meshes/stretchZone.cpp:74-93)
    const int nz = c->nstretch[a];
    if (nz < 0 || nz > ECG_MAX_STRETCH_ZONES) { set_error("bad number of stretch zones"); return ECG_ERR_INVALID; }
    if (nz == 0 || c->ncells[a] <= 1) continue;
    int cells = 0;
    for (int z = 0; z < nz; z++) {
      const ecg_stretch_zone& st = c->stretch[a][z];
      if (st.ncells < 1 || !(st.end > st.start) || !(st.factor > 0.)) { set_error("bad stretch zone"); return ECG_ERR_INVALID; }
      if (z == 0 ? st.start != 0. : st.start != c->stretch[a][z - 1].end) { set_error("stretch zones are not contiguous from 0"); return ECG_ERR_INVALID; }
      cells += st.ncells;
    }
    if (c->stretch[a][nz - 1].end != c->length[a]) { set_error("stretch zones do not end at the domain length"); return ECG_ERR_INVALID; }
    if (cells != c->ncells[a]) { set_error("stretch zone cells do not add up to the axis' cells"); return ECG_ERR_INVALID; }
  }
  int64_t n = (int64_t)c->ncells[0] * c->ncells[1] * c->ncells[2];
  if (n > (int64_t)1 << 31) { set_error("more than 2^31 cells"); return ECG_ERR_TOO_LARGE; }
  return ECG_OK;
}

}  // namespace ecg
