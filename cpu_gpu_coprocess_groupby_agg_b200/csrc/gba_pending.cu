// Entry points whose implementations are not built yet: they fail loudly.
#include "gba_context.h"
#include "gba_plan.h"

extern "C" gba_status gba_groupby_batch(gba_context* ctx, int32_t, const gba_query*, const gba_output*,
                                        const gba_knobs*, void*, int64_t*) {
  if (ctx) ctx->err = "batch path not built";
  return GBA_ERR_UNSUPPORTED;
}
