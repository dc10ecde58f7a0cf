// Host-visible interface of the batched-query kernels (k_agg.cu).
#pragma once
#include "gba_kernels.h"

// One query of a batch group, as the persistent kernel reads it.
struct BatchQ {
  QDesc q;
  GTable gt;
  OutDesc out;
  unsigned* flags;  // this query's status bits
  int S;            // its shared-table slots (0 = no pre-aggregation)
  int pad;
};

// One work-queue item: a row range of one query.
struct BatchItem {
  int qi;
  int pad;
  int64_t row_begin, row_end;
};

size_t gba_batch_smem_bytes(const QDesc& q, int S, int T);
cudaError_t gba_launch_batch_preagg(const QDesc& proto, const BatchQ* d_qs, const BatchItem* d_items, int nitems,
                                    unsigned* item_ctr, int S_max, int sprobe, int T, int grid, cudaStream_t s);
cudaError_t gba_launch_batch_init(const BatchQ* d_qs, int nq, int gx, cudaStream_t s);
cudaError_t gba_launch_batch_compact(const BatchQ* d_qs, int nq, int gx, cudaStream_t s);
size_t gba_batch_static_smem();
