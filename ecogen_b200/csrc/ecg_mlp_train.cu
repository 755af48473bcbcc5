// MLP training kernels (forward, backward, AdamW).
#include "ecg_internal.h"

struct ecg_trainer {};

extern "C" ecg_status ecg_trainer_create(int32_t, int32_t, uint64_t, ecg_trainer** out) {
  if (out) *out = nullptr;
  ecg::set_error("trainer not built yet");
  return ECG_ERR_UNSUPPORTED;
}
extern "C" void ecg_trainer_destroy(ecg_trainer*) {}
extern "C" ecg_status ecg_trainer_epoch(ecg_trainer*, const float*, const float*, int64_t, int32_t, float, float, float*) { return ECG_ERR_UNSUPPORTED; }
extern "C" ecg_status ecg_trainer_grad(ecg_trainer*, const float*, const float*, int32_t, float*, float*, float*, float*, float*, float*, float*) { return ECG_ERR_UNSUPPORTED; }
extern "C" ecg_status ecg_trainer_forward(ecg_trainer*, const float*, int32_t, float*) { return ECG_ERR_UNSUPPORTED; }
extern "C" ecg_status ecg_trainer_export(ecg_trainer*, ecg_mlp*) { return ECG_ERR_UNSUPPORTED; }
extern "C" ecg_status ecg_trainer_import(ecg_trainer*, const ecg_mlp*) { return ECG_ERR_UNSUPPORTED; }
extern "C" ecg_status ecg_trainer_set_norm(ecg_trainer*, const float*, const float*, float, float) { return ECG_ERR_UNSUPPORTED; }
