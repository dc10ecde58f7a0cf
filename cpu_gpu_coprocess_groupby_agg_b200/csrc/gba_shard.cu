// Sharded GROUP BY across ranks: gba_avg_divide, SUM / COUNT in place for an
// AVG merged from partial SUMs and COUNTs (k_avg_finish).
//
// No reference counterpart: the reference runs on one device
// (test/test.cu:35).
#include "gba_context.h"

extern "C" gba_status gba_avg_divide(gba_context* ctx, int32_t n_cols, void* const* sums, const int32_t* sum_is_fp,
                                     const int64_t* counts, int64_t n, void* stream) {
  if (!ctx || n_cols < 0 || n_cols > GBA_MAX_AGGS || n < 0 || (n > 0 && n_cols > 0 && (!sums || !sum_is_fp || !counts)))
    return GBA_ERR_INVALID_ARG;
  if (n == 0 || n_cols == 0) return GBA_OK;
  GBA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  AvgDesc d{};
  for (int i = 0; i < n_cols; ++i) {
    if (!sums[i]) return GBA_ERR_INVALID_ARG;
    d.col[i] = static_cast<unsigned long long*>(sums[i]);
    d.fp[i] = sum_is_fp[i] != 0;
  }
  d.n = n_cols;
  d.count = reinterpret_cast<const unsigned long long*>(counts);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  GBA_CUDA_TRY(ctx, gba_launch_avg_finish(d, n, ctx->sms, s));
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return GBA_OK;
}
