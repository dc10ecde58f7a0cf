// Host-visible interface of the radix-partition strategy kernels (k_part.cu).
#pragma once
#include "gba_kernels.h"

// One histogram/scatter work unit: a run of rows inside one input segment.
struct PartChunk {
  int64_t row_begin, row_end;
  int64_t count_base;  // first counts[] entry of the chunk's segment
  int seg_nchunks;     // chunks in that segment
  int chunk_in_seg;
};

// One MSD partition pass over `bits` hash bits below the `shift_hi` bits
// already used.  counts/offsets layout: [segment][digit][chunk-in-segment].
struct PartPass {
  QDesc in;   // rows read (keys + value columns)
  QDesc out;  // rows written (keys + value columns, same types)
  const PartChunk* chunks;
  int nchunks;
  int shift_hi;
  int bits;
  unsigned* counts;
  const unsigned long long* offsets;
};

// One work item of the final aggregation: whole partitions [seg_lo, seg_hi),
// or (partial = 1) the rows [row_begin, row_end) of one partition too large
// for one CTA; a partial piece merges its groups into the HBM table.
struct PartWork {
  int seg_lo, seg_hi;
  int partial;
  int pad;
  int64_t row_begin, row_end;
};

// Final aggregation: one shared-memory table per partition (or piece).
struct PartAgg {
  QDesc rows;                 // partitioned rows + aggregate spec
  const long long* seg_begin; // nsegs + 1 entries
  int nsegs;
  const PartWork* work;       // work items, largest first
  int nwork;
  unsigned* seg_ctr;          // dynamic work queue (zeroed before launch)
  int S;                      // shared table slots
  int sprobe;
  int coalesce;
  GTable fallback;            // keys whose probe window is full + pieces of split partitions
  unsigned* flags;
  OutDesc out;
};

size_t gba_part_scatter_smem(const QDesc& q, int bits, int T);
cudaError_t gba_launch_part_hist(const PartPass& p, int grid, cudaStream_t s);
cudaError_t gba_launch_scan_excl(const unsigned* in, unsigned long long* out, int64_t n,
                                 unsigned long long* status, unsigned* tile_ctr, unsigned* flags, cudaStream_t s);
cudaError_t gba_launch_part_scatter(const PartPass& p, int grid, int T, cudaStream_t s);
// seg_begin[s * 2^bits + d] = offsets[count_base[s] + d * seg_nchunks[s]] for
// every input segment s; seg_begin[nseg_in * 2^bits] = total rows
cudaError_t gba_launch_seg_begins(const unsigned long long* offsets, const long long* count_base,
                                  const int* seg_nchunks, int nseg_in, int bits, int64_t total,
                                  long long* seg_begin, cudaStream_t s);
cudaError_t gba_launch_part_agg(const PartAgg& a, int grid, cudaStream_t s);
