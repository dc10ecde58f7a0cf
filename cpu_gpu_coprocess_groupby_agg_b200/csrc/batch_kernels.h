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

// dynamic shared memory of a batch CTA: miss list of T rows + a table of S
// slots laid out for 64-bit keys (one launch serves both key widths)
size_t gba_batch_smem_bytes(const QDesc& q, int S, int T);
size_t gba_batch_static_smem();
// which compiled signature serves q (queries with equal ids share a launch)
int gba_batch_sig_id(const QDesc& q);
// sets the kernel's dynamic shared-memory limit (outside any stream capture)
cudaError_t gba_prepare_batch_preagg(const QDesc& proto, size_t smem);
cudaError_t gba_launch_batch_preagg(const QDesc& proto, const BatchQ* d_qs, const BatchItem* d_items, int nitems,
                                    unsigned* item_ctr, size_t smem, int sprobe, int T, int grid, int block,
                                    cudaStream_t s);
// blk_prefix[i]: first block of query i (nq + 1 entries, blk_prefix[nq] = nblocks)
cudaError_t gba_launch_batch_init(const BatchQ* d_qs, const int64_t* blk_prefix, int nq, int64_t nblocks,
                                  cudaStream_t s);
cudaError_t gba_launch_batch_compact(const BatchQ* d_qs, const int64_t* blk_prefix, int nq, int64_t nblocks,
                                     cudaStream_t s);
