// Composite keys (gba_query.key2): the pair of 32-bit keys packed into one
// order-preserving 64-bit key before a call and unpacked after it.
#pragma once

#include <vector>

#include "gba_context.h"

struct CompositeJob {
  int query;       // index among the call's queries
  unsigned s1, s2; // sign flips of the two halves (0x80000000 for I32, 0 for U32)
  size_t in_off;   // packed input keys in the context's composite buffer
  size_t out_off;  // packed output keys there
};

// For every query with a second key column: packs its keys into the context's
// composite buffer (kernels on stream s) and points q2[i] / o2[i] (copies of
// qs[i] / outs[i]) at the packed key columns.  Queries without key2 are left
// as they are.
gba_status gba_composite_prepare(gba_context* ctx, int nq, const gba_query* qs, const gba_output* outs,
                                 gba_query* q2, gba_output* o2, std::vector<CompositeJob>* jobs, cudaStream_t s);

// Unpacks each composite query's n_groups output keys into outs[i].keys and
// outs[i].keys2, then synchronizes s.
gba_status gba_composite_finish(gba_context* ctx, const std::vector<CompositeJob>& jobs, const gba_output* outs,
                                const int64_t* n_groups, cudaStream_t s);
