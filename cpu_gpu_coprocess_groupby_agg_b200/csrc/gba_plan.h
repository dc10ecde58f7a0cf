// Internal planning interface between the single-query driver, the partition
// strategy and the estimator.
#pragma once
#include "gba_context.h"

// bytes of one input row: key + value columns
inline size_t gba_row_bytes(const QDesc& q) {
  size_t b = q.key64 ? 8 : 4;
  for (int c = 0; c < q.ncols; ++c) b += gba_type_bytes(q.col_type[c]);
  return b;
}

struct GbaPlan {
  int grid, block;
  int tile_rows;
  int nstages;
  int use_tma;
  int coalesce;
  int preagg;
  int smem_slots;
  int smem_probe_cap;
  uint64_t table_slots;
  int probe_cap;
  int partition_bits;
};

void gba_make_plan(const gba_context* ctx, const QDesc& q, const gba_knobs& k, double predicted_groups,
                   GbaPlan* p);
int gba_choose_strategy(const gba_context* ctx, const QDesc& q, const gba_knobs& k, double predicted_groups,
                        const GbaPlan& p);
gba_status gba_run_table(gba_context* ctx, const QDesc& q, const gba_output* out, const gba_knobs& k, GbaPlan p,
                         cudaStream_t s, int64_t* n_groups);
gba_status gba_run_partition(gba_context* ctx, const QDesc& q, const gba_output* out, const gba_knobs& k,
                             const GbaPlan& p, double predicted_groups, cudaStream_t s, int64_t* n_groups);
// Estimator inference for one device-resident query: predicted group count.
gba_status gba_predict_groups(gba_context* ctx, const QDesc& q, cudaStream_t s, double* groups);
// Second growable device buffer used for host-resident inputs (staging).
gba_status gba_stage_reserve(gba_context* ctx, size_t bytes, cudaStream_t s);
