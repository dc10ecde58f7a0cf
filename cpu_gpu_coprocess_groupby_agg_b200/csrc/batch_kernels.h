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
  int pad;          // bit 0: keys and columns 16-byte aligned (vector loads)
};

// The work-queue items of one query, described at once: items first_item ..
// of item_rows rows each (the last one shorter) over query qi's rows.  A
// launch takes its queries' spans in queue order; item it belongs to the last
// span whose first_item <= it.
struct BatchSpan {
  int qi;
  int pad;
  int64_t item_rows;
  int64_t first_item;
};

size_t gba_batch_static_smem();
// which compiled signature serves q (queries with equal ids share a launch)
int gba_batch_sig_id(const QDesc& q);
// Streaming aggregation (k_stream.cu): one persistent launch over the nitems
// work items of nspans query spans (item_rows a multiple of 256).  *item_ctr
// must be zero at launch.  minb = CTAs per SM the launch is built for: 1 (512
// threads with the whole shared memory and all registers), 2, 3 or 4 (that
// many such CTAs, each with its share of both).  hbm: every query of the
// launch has BatchQ.S == 0 (no shared table): a kernel without table code
// (minb 2 or 3; others run the general kernel).
size_t gba_stream_smem_bytes(const QDesc& q, int S);
int gba_stream_rows_per_chunk(const QDesc& q, int minb);
cudaError_t gba_prepare_stream_agg(const QDesc& proto, int minb, bool hbm);
cudaError_t gba_launch_stream_agg(const QDesc& proto, int minb, bool hbm, const BatchQ* d_qs,
                                  const BatchSpan* d_spans, int nspans, int64_t nitems, unsigned* item_ctr,
                                  size_t smem, int sprobe, int grid, cudaStream_t s);
// Table init and compaction of the table entries whose blocks are block0 ..
// block0 + nblocks - 1: blk_prefix[i] is the first block of entry i (entries
// 0 .. nq - 1 searched, blk_prefix[nq] >= block0 + nblocks)
cudaError_t gba_launch_batch_init(const BatchQ* d_qs, const int64_t* blk_prefix, int nq, int64_t nblocks,
                                  int64_t block0, cudaStream_t s);
cudaError_t gba_launch_batch_compact(const BatchQ* d_qs, const int64_t* blk_prefix, int nq, int64_t nblocks,
                                     int64_t block0, cudaStream_t s);
// Streaming aggregation with bulk-copy staging (k_stream_tma.cu): CTAs of
// 512 threads, minb (1 or 2) per SM, or (minb 0) one CTA of 1024 threads per
// SM; every warp stages chunks of rows through
// its own ring of nstages (1..4) slots of slot_bytes each (the largest
// gba_stream_tma_slot_bytes of the launch's queries), placed before the
// shared table.  BatchQ.pad bit 1: combine equal keys within a warp before
// the shared-table update.  cluster: 1, or 2/4/8/16 CTAs (minb 1) whose
// shared tables form one table (distributed shared memory), for signatures of
// integer SUMs and COUNTs (gba_stream_tma_cluster_ok); the grid of a cluster
// launch is gba_stream_tma_cluster_grid CTAs (0: such clusters cannot be
// resident).
size_t gba_stream_tma_slot_bytes(const QDesc& q, int minb);
size_t gba_stream_tma_smem_bytes(const QDesc& q, int S, int nstages, size_t slot_bytes, int minb);
bool gba_stream_tma_cluster_ok(const QDesc& q);
int gba_stream_tma_cluster_grid(const QDesc& proto, int cluster, size_t smem, int sms);
cudaError_t gba_prepare_stream_tma(const QDesc& proto, int cluster, int minb);
cudaError_t gba_launch_stream_tma(const QDesc& proto, int cluster, int minb, const BatchQ* d_qs,
                                  const BatchSpan* d_spans, int nspans, int64_t nitems, unsigned* item_ctr,
                                  size_t smem, int sprobe, int grid, int nstages, size_t slot_bytes, cudaStream_t s);
// Owner-exchange aggregation (k_exchange.cu): one cooperative launch of `grid`
// CTAs (one per SM) over the nxq queries d_xq (indices into d_qs), each with
// a shared table of BatchQ.S slots per CTA (and a hot table of 4 x
// (BatchQ.pad >> 16 & 4095) slots).  Rows move in windows of `win` rows
// through two exchange buffers of buf_words 8-byte words each, which hold
// grid regions of `region` records of the widest record (1 + ncols words for
// rows, 1 + naccs for hot-table partials; region >= win); cursors (2 x grid),
// bar (2) and *bar_flags must be zero at launch.
// S owner-table slots and `hot` hot-table slots per CTA
size_t gba_exchange_smem_bytes(const QDesc& q, int S, int hot);
size_t gba_exchange_static_smem();
cudaError_t gba_prepare_exchange(const QDesc& proto);
int gba_exchange_grid(const QDesc& proto, size_t smem, int sms);
cudaError_t gba_launch_exchange(const QDesc& proto, const BatchQ* d_qs, const int* d_xq, int nxq, int64_t win,
                                unsigned long long* xbuf, int64_t region, int64_t buf_words, unsigned* cursors,
                                unsigned* bar, unsigned* bar_flags, size_t smem, int sprobe, int grid, cudaStream_t s);
