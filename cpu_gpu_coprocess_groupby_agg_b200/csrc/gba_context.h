// Internal definition of gba_context and helpers shared by the host-side
// translation units (single-query path, batch path, estimator, drop-in).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "gba_kernels.h"

struct gba_context {
  int device = 0;
  int sms = 148;
  int max_smem_optin = 227 * 1024;
  // growable device workspace (tables, partitions, staging)
  void* ws = nullptr;
  size_t ws_bytes = 0;
  // growable device staging for host-resident inputs and outputs
  void* stage = nullptr;
  size_t stage_bytes = 0;
  // small device scratch: [0] flags, [8] group counter, [64..] per-query counters
  unsigned char* d_small = nullptr;
  size_t d_small_bytes = 0;
  // pinned host mirror of d_small
  unsigned char* h_small = nullptr;
  size_t h_small_bytes = 0;
  cudaStream_t copy_stream = nullptr;
  // host-resident batch: the device-to-host stream and one event per part
  cudaStream_t out_stream = nullptr;
  std::vector<cudaEvent_t> part_ev;
  cudaEvent_t ev[8] = {};
  cudaEvent_t tev[16] = {};  // timing events (gba_knobs.timing)
  // estimator (device weights + Adam state + gradient scratch)
  float* d_est = nullptr;
  bool est_loaded = false;
  // estimator sampling scratch (count tables, HLL registers, features)
  void* est_ws = nullptr;
  size_t est_ws_bytes = 0;
  // share of the last estimator sample taken by its most frequent key
  double est_skew = 0.0;
  // batch path: pinned descriptor/status staging, capture stream, and the
  // instantiated graph of the last batch shape with its key
  unsigned char* h_batch = nullptr;
  size_t h_batch_bytes = 0;
  cudaStream_t cap_stream = nullptr;
  // a second stream (and fork/join events) for batch launches that run side by side
  cudaStream_t aux_stream = nullptr;
  cudaEvent_t fork_ev[2] = {};
  cudaGraphExec_t batch_exec = nullptr;
  std::vector<int64_t> batch_key;
  // drop-in API: a tile's groups before the reference-layout partitioning
  void* rp_buf = nullptr;
  size_t rp_bytes = 0;
  // AVG without a COUNT in the query: the added COUNT's output column
  void* avg_buf = nullptr;
  size_t avg_bytes = 0;
  // composite keys: packed input and output keys of a call's queries
  void* ck_buf = nullptr;
  size_t ck_bytes = 0;
  // nullable columns: identity-filled copies, presence columns, hidden counts
  void* null_buf = nullptr;
  size_t null_bytes = 0;
  std::string err;
  gba_stats stats{};
};

#define GBA_CUDA_TRY(ctx, expr)                                                                           \
  do {                                                                                                    \
    cudaError_t _e = (expr);                                                                              \
    if (_e != cudaSuccess) {                                                                              \
      (ctx)->err = std::string(#expr) + ": " + cudaGetErrorString(_e);                                    \
      return _e == cudaErrorMemoryAllocation ? GBA_ERR_OOM : GBA_ERR_CUDA;                                \
    }                                                                                                     \
  } while (0)

// Grow-only device workspace.  Callers must not hold pointers across a call
// that may grow it; the library syncs its stream before it frees the old block.
// Kernel timing (gba_knobs.timing): mark before/after a launch of role r.
struct GbaTimer {
  gba_context* ctx;
  cudaStream_t s;
  bool on;
  int n = 0;
  int role[8];
  void begin(int r);
  void end();
  void collect();  // after the stream synced: adds to ctx->stats.kernel_ms
};

gba_status gba_ws_reserve(gba_context* ctx, size_t bytes, cudaStream_t s);
gba_status gba_small_reserve(gba_context* ctx, size_t bytes);
gba_status gba_batch_host_reserve(gba_context* ctx, size_t bytes);
gba_status gba_est_reserve(gba_context* ctx, size_t bytes, cudaStream_t s);
// estimator features of nq device queries into ctx->est_ws (device pointers)
gba_status gba_est_features_device(gba_context* ctx, const QDesc* qs, int nq, int64_t tile_rows, cudaStream_t s,
                                   float** feats_out, unsigned long long** stats_out);
gba_status gba_build_qdesc(gba_context* ctx, const gba_query* q, QDesc* d);
void gba_compact_query(const gba_query* in, gba_query* out);
size_t gba_round_up(size_t x, size_t a);
uint64_t gba_pow2_ceil(uint64_t x);
