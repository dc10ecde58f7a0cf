// Host-visible kernel interface: the plain structs the launchers take and the
// launcher declarations.  No device code here, so host-only translation units
// can include it.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/gba.h"

// Accumulator operations.  Every aggregate becomes one 8-byte accumulator.
enum AccOp : int {
  ACC_ADD_I = 0,  // SUM of an integer column, int64 (wraps mod 2^64)
  ACC_CNT = 1,    // COUNT, int64
  ACC_MIN_I = 2,  // MIN of an integer column, int64
  ACC_MAX_I = 3,  // MAX of an integer column, int64
  ACC_ADD_F = 4,  // SUM of an fp32 or fp64 column, accumulated in fp64
};

// bytes of one value of a column type (I64 = 1 and F64 = 4 are the 8-byte
// types: bits 1 and 4 of 0x12; one shift instead of two compares in row loops)
__host__ __device__ inline int gba_type_bytes(int t) { return (0x12u >> t) & 1u ? 8 : 4; }

// One query as the kernels see it (passed by value in the parameter space).
struct QDesc {
  const void* keys;
  const void* cols[GBA_MAX_COLS];
  int64_t n;
  int key64;  // 1: 64-bit keys, 0: 32-bit keys
  int ncols;
  int col_type[GBA_MAX_COLS];
  int naccs;
  int acc_op[GBA_MAX_AGGS];
  int acc_col[GBA_MAX_AGGS];    // source column (0 for COUNT)
  int acc_ctype[GBA_MAX_AGGS];  // type of the source column
  // shared-memory layout, in 4-byte words: accumulator a starts at word
  // acc_woff[a] of a slot; COUNT takes 1 word (a shared table lives for fewer
  // than 2^32 rows), fp SUM 6 (128-bit exact fixed point + fp64 residual), the
  // others 2; nwords = 4-byte words per slot
  int acc_woff[GBA_MAX_AGGS];
  int nwords;
};

// 4-byte words one accumulator op occupies in a shared-memory slot
inline int gba_acc_smem_words(int op) { return op == ACC_CNT ? 1 : op == ACC_ADD_F ? 6 : 2; }

// HBM hash table: array-of-structs slots [key | acc0 .. acc{A-1}], 8 bytes
// each; slot `cap` is the side slot of the all-ones key (the empty marker),
// whose key word is its presence flag.
struct GTable {
  unsigned long long* base;  // (cap + 1) * gba_gt_stride(naccs) words
  uint64_t cap;
  int probe_cap;
};

// 8-byte words per HBM-table slot: the key and one word per accumulator.
// (Measured on the 256-query batch: padding 3-word slots to 4, so that no slot
// straddles a 32-byte sector, sped the largest tables' queries up by 3.5% but
// made every table a third larger to clear and compact: 0.4 ms more per step.)
__host__ __device__ constexpr int gba_gt_stride(int naccs) { return 1 + naccs; }

struct OutDesc {
  void* keys;
  unsigned long long* accs[GBA_MAX_AGGS];
  int64_t capacity;
  unsigned long long* count;  // device counter of groups written
};

// Status bits written by kernels and read by the host after the stream syncs.
enum : unsigned {
  GBA_FLAG_TABLE_OVERFLOW = 1u,  // an HBM-table insert ran out of probes
  GBA_FLAG_WAIT_TIMEOUT = 2u,    // a bounded mbarrier wait gave up
  GBA_FLAG_PART_OVERFLOW = 4u,   // a partition outgrew its shared table
  GBA_FLAG_DRAIN_TIMEOUT = 8u,   // after an abort, a copy still in flight did not land in time
};

struct PreaggCfg {
  int grid, block;
  int smem_slots;
  int smem_probe_cap;
  int tile_rows;
  int nstages;
  int use_tma;
  int coalesce;
};

// AVG finishing pass: col[i][r] (an int64 SUM, or fp64 bits when fp[i]) becomes
// the double SUM / count[r], for the first n rows.
struct AvgDesc {
  unsigned long long* col[GBA_MAX_AGGS];
  int fp[GBA_MAX_AGGS];
  int n;
  const unsigned long long* count;
};
cudaError_t gba_launch_avg_finish(const AvgDesc& d, int64_t rows, int sms, cudaStream_t s);

size_t gba_preagg_smem_bytes(const QDesc& q, int S, int T, int nstages, int use_tma);
cudaError_t gba_launch_table_init(const GTable& t, const QDesc& q, int grid, cudaStream_t s);
cudaError_t gba_launch_preagg(const QDesc& q, const GTable& t, const PreaggCfg& c, unsigned* flags,
                              cudaStream_t s);
cudaError_t gba_launch_compact(const GTable& t, const QDesc& q, const OutDesc& o, int grid, cudaStream_t s);
