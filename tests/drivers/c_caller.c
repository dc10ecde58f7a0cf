#include <stdio.h>
/* A C11 caller of the C ABI, as the integration guide shows it (compile and link check
 * only: tests/test_abi.py builds it with gcc; it is never run). */
#include "gba.h"
int run(void* d_keys, void* d_vals, void* d_vals_valid, void* d_k1, void* d_k2, void* d_out_keys, void* d_out_sum,
        void* d_out_count, unsigned char* d_sum_valid, void* d_out_k2, int64_t n, int64_t capacity, void* stream) {
  gba_context* ctx;            gba_create(&ctx, /*device*/ 0);
  gba_query q = {0};           q.n_rows = n;
  q.key = (gba_column){GBA_I64, d_keys};
  q.n_cols = 1;                q.cols[0] = (gba_column){GBA_I64, d_vals};
  q.n_aggs = 2;                q.aggs[0] = (gba_agg){GBA_SUM, 0}; q.aggs[1] = (gba_agg){GBA_COUNT, 0};
  gba_output out = {d_out_keys, {d_out_sum, d_out_count}, capacity};
  gba_knobs k;                 gba_default_knobs(&k);
  int64_t groups;
  if (gba_groupby(ctx, &q, &out, &k, stream, &groups) != GBA_OK) puts(gba_last_error(ctx));
  q.cols[0] = (gba_column){GBA_I64, d_vals, d_vals_valid};
  q.aggs[1] = (gba_agg){GBA_COUNT_VALID, 0};
  out.agg_valid[0] = d_sum_valid;
  q.key = (gba_column){GBA_I32, d_k1};
  q.key2 = (gba_column){GBA_I32, d_k2};
  out.keys2 = d_out_k2;
  k.sort_output = 1;
  gba_groupby(ctx, &q, &out, &k, stream, &groups);
  return gba_destroy(ctx);
}
