// Nullable value columns and COUNT(col): the rewrite around a call.
#pragma once

#include <cstdint>
#include <vector>

#include "gba_context.h"

struct NullPlan {
  int query = 0;
  int nullable_agg[GBA_MAX_AGGS];     // source column of an aggregate over a nullable column, else -1
  bool avg_on[GBA_MAX_AGGS] = {};     // an AVG over a nullable column (run as SUM, divided after)
  bool count_valid_agg[GBA_MAX_AGGS] = {};  // a COUNT(col) over a nullable column
  int count_of[GBA_MAX_COLS];         // present count of column c: rewritten aggregate k >= 0 (scratch),
                                      // or the caller's COUNT(col) aggregate -1 - k
  size_t hidden_off[GBA_MAX_AGGS];    // scratch offset of a hidden count's output, else SIZE_MAX
  int col_index[GBA_MAX_COLS][5];     // rewritten column of (source column, variant), or -1
  NullPlan() {
    for (int& x : nullable_agg) x = -1;
    for (int& x : count_of) x = 0;
    for (size_t& x : hidden_off) x = SIZE_MAX;
  }
};

// Does the query (with its output) need the rewrite: a nullable column or key,
// a COUNT(col), or a requested validity output?
bool gba_nulls_needed(const gba_query& q, const gba_output& o);

// For every query that needs it: points q2[i] / o2[i] (copies of qs[i] /
// outs[i]) at identity-filled copies and presence columns written on stream s
// into the context's null buffer, with hidden count aggregates where needed.
gba_status gba_nulls_prepare(gba_context* ctx, int nq, const gba_query* qs, const gba_output* outs, gba_query* q2,
                             gba_output* o2, std::vector<NullPlan>* plans, cudaStream_t s);

// After the call: divides nullable AVGs by their present counts and writes the
// requested validity bytes (outs), then synchronizes s.  o2 holds the
// rewritten outputs (hidden count columns).
gba_status gba_nulls_finish(gba_context* ctx, const std::vector<NullPlan>& plans, const gba_query* qs,
                            const gba_output* outs, const gba_output* o2, const int64_t* n_groups, cudaStream_t s);
