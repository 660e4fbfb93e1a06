// dspw_train.cu -- DSP-WENO network training on the GPU (placeholder until the
// training kernels land; every entry point reports DSPW_ERR_UNSUPPORTED).
#include "../../include/dspw.h"

extern "C" {
int dspw_trainer_create(const dspw_train_cfg*, const double*, const double*, dspw_trainer** out) {
  if (out) *out = nullptr;
  return DSPW_ERR_UNSUPPORTED;
}
int dspw_trainer_destroy(dspw_trainer*) { return DSPW_ERR_UNSUPPORTED; }
int dspw_trainer_set_data(dspw_trainer*, const double*, const double*, long long) { return DSPW_ERR_UNSUPPORTED; }
int dspw_trainer_collect(dspw_trainer*, dspw_handle*, long long, long long*) { return DSPW_ERR_UNSUPPORTED; }
int dspw_trainer_epoch(dspw_trainer*, double*) { return DSPW_ERR_UNSUPPORTED; }
int dspw_trainer_loss_grad(dspw_trainer*, const double*, const double*, int, double*, double*, double*) {
  return DSPW_ERR_UNSUPPORTED;
}
int dspw_trainer_get_params(dspw_trainer*, double*, double*) { return DSPW_ERR_UNSUPPORTED; }
}
