// Key-ordered output (gba_knobs.sort_output): the groups a call produced,
// sorted on the device by key, ascending (signed order for I32/I64 keys,
// unsigned for U32), with every aggregate column permuted alike.
#pragma once

#include "gba_context.h"

struct SortJob {
  void* keys;                                // g keys, 4 or 8 bytes each, sorted in place
  int key64;                                 // 1: 8-byte keys
  int key_signed;                            // 1: two's-complement order
  int nagg;                                  // aggregate columns (8-byte words) that follow the keys
  unsigned long long* aggs[GBA_MAX_AGGS];
  int64_t g;                                 // groups
};

// The job for a query's output holding g groups.
inline SortJob gba_sort_job(const gba_query* q, const gba_output* out, int64_t g) {
  SortJob j{};
  j.keys = out->keys;
  j.key64 = q->key.type == GBA_I64;
  j.key_signed = q->key.type != GBA_U32;
  j.nagg = q->n_aggs < GBA_MAX_AGGS ? q->n_aggs : GBA_MAX_AGGS;
  for (int a = 0; a < j.nagg; ++a) j.aggs[a] = static_cast<unsigned long long*>(out->aggs[a]);
  j.g = g;
  return j;
}

// Sorts every job's groups, one job after another on stream s, in the context
// workspace; one host round trip for all jobs' key ranges and one at the end.
gba_status gba_sort_groups(gba_context* ctx, const SortJob* jobs, int njobs, cudaStream_t s);
