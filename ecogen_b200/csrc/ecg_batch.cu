// Batched independent cases (persistent work-queue kernel).
#include "ecg_internal.h"

struct ecg_batch {};

extern "C" ecg_status ecg_batch_create(const ecg_case*, int32_t, ecg_batch** out) {
  if (out) *out = nullptr;
  ecg::set_error("batched mode not built yet");
  return ECG_ERR_UNSUPPORTED;
}
extern "C" void ecg_batch_destroy(ecg_batch*) {}
extern "C" ecg_status ecg_batch_upload_prim(ecg_batch*, const double* const*, int64_t) { return ECG_ERR_UNSUPPORTED; }
extern "C" ecg_status ecg_batch_download_prim(ecg_batch*, double* const*, int64_t) { return ECG_ERR_UNSUPPORTED; }
extern "C" ecg_status ecg_batch_step(ecg_batch*, int32_t, double*, double*, ecg_step_stats*) { return ECG_ERR_UNSUPPORTED; }
extern "C" ecg_status ecg_batch_set_seed_model(ecg_batch*, const ecg_mlp*) { return ECG_ERR_UNSUPPORTED; }
extern "C" ecg_status ecg_batch_set_shape(ecg_batch*, int32_t, int32_t) { return ECG_ERR_UNSUPPORTED; }
extern "C" ecg_status ecg_batch_autotune(ecg_batch*, int32_t*, int32_t*) { return ECG_ERR_UNSUPPORTED; }
extern "C" int64_t ecg_batch_total_cells(const ecg_batch*) { return 0; }
