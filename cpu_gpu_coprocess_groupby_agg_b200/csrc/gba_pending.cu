// Entry points whose implementations are not built yet: they fail loudly.
#include "gba_context.h"
#include "gba_plan.h"

gba_status gba_predict_groups(gba_context* ctx, const QDesc&, cudaStream_t, double*) {
  ctx->err = "estimator not built";
  return GBA_ERR_UNSUPPORTED;
}

extern "C" gba_status gba_groupby_batch(gba_context* ctx, int32_t, const gba_query*, const gba_output*,
                                        const gba_knobs*, void*, int64_t*) {
  if (ctx) ctx->err = "batch path not built";
  return GBA_ERR_UNSUPPORTED;
}
extern "C" gba_status gba_estimator_features(gba_context*, const gba_query*, int64_t, void*, float*) {
  return GBA_ERR_UNSUPPORTED;
}
extern "C" int64_t gba_estimator_param_count(void) { return 0; }
extern "C" gba_status gba_estimator_load(gba_context*, const float*) { return GBA_ERR_UNSUPPORTED; }
extern "C" gba_status gba_estimator_get(gba_context*, float*) { return GBA_ERR_UNSUPPORTED; }
extern "C" gba_status gba_estimator_predict(gba_context*, int32_t, const float*, float*) {
  return GBA_ERR_UNSUPPORTED;
}
extern "C" gba_status gba_estimator_train(gba_context*, int32_t, const float*, const float*, int32_t, int32_t, float,
                                          uint64_t, float*) {
  return GBA_ERR_UNSUPPORTED;
}
extern "C" gba_status gba_estimator_grad(gba_context*, int32_t, const float*, const float*, float*, float*) {
  return GBA_ERR_UNSUPPORTED;
}
