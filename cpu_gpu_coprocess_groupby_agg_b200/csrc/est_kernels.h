// Host-visible interface of the cardinality estimator kernels (k_est.cu).
#pragma once
#include "gba_kernels.h"

#define GBA_EST_MAX_TILES 256
// largest row count of the tables the shipped weights were trained on
// (estimator_weights.f32: rows log-uniform in [2^12, 2^24])
#define GBA_EST_TRAINED_MAX_ROWS (int64_t(1) << 24)

// One query's sampling job and its scratch (all device pointers).
struct EstQuery {
  const void* keys;
  int64_t n;
  int64_t tile_rows;
  int64_t tile_step;    // sample every tile_step-th tile
  int sampled_tiles;
  int key64;
  int64_t chunk_base;         // first sampling block of this query (k_est_sample's grid is flat)
  int nchunks;                // sampling blocks of this query: kEstChunkTiles sampled tiles each
  unsigned long long* table;  // cap x {key, count}
  uint64_t cap;
  unsigned* hll;              // 64 registers
  float* feat;                // 32 features
  unsigned long long* stats;  // [0] distinct sampled keys, [1] max count, [2] sampled rows, [3] all-ones key count
  unsigned long long* freq;   // [0] distinct, [1..4] f1, f2, f3, f4+, [5] max count, [6] sampled rows
};

void gba_est_plan(EstQuery* e, int64_t n, int64_t tile_rows);
int64_t gba_est_nparam();
cudaError_t gba_launch_est_init(const EstQuery* d_qs, int nq, cudaStream_t s);
// sampled tiles per block of k_est_sample
#define GBA_EST_CHUNK_TILES 4
cudaError_t gba_launch_est_sample(const EstQuery* d_qs, int nq, int64_t total_chunks, cudaStream_t s);
cudaError_t gba_launch_est_reduce(const EstQuery* d_qs, int nq, cudaStream_t s);
cudaError_t gba_launch_mlp_forward(const float* W, const float* X, int n, float* out, cudaStream_t s);
