// Nullable value columns (gba_column.valid) and COUNT(col) (GBA_COUNT_VALID).
//
// A query whose aggregates read a nullable column is rewritten before the
// single-key path runs: one kernel pass over each such column writes the copies
// the aggregates need, nulls replaced by the aggregate's identity (0 for SUM
// and AVG, the type's largest value for MIN, its smallest for MAX), and a 0/1
// presence column where a count of present values is needed (COUNT(col), AVG,
// or a requested validity output).  The count is then a SUM over the presence
// column.  After the call a finish kernel writes the validity bytes (1 when a
// group saw a present value) and divides each nullable AVG by its column's
// count instead of COUNT(*).
//
// No reference counterpart: the reference's columns have no nulls
// (tiled_groupby_agg_partition/include/util.cuh:6-7).
#include <algorithm>
#include <cstring>
#include <string>

#include "nulls.h"

namespace {

enum Variant { V_RAW = 0, V_ZERO = 1, V_MINID = 2, V_MAXID = 3, V_IND = 4 };

__device__ __forceinline__ unsigned long long min_identity(int type) {
  return type == GBA_I32 ? 0x7fffffffull : type == GBA_U32 ? 0xffffffffull : 0x7fffffffffffffffull;
}
__device__ __forceinline__ unsigned long long max_identity(int type) {
  return type == GBA_I32 ? 0x80000000ull : type == GBA_U32 ? 0ull : 0x8000000000000000ull;
}

__global__ void __launch_bounds__(256) k_null_prep(const void* src, const unsigned char* valid, int type, int64_t n,
                                                   void* zero, void* minid, void* maxid, int* ind) {
  const bool w8 = gba_type_bytes(type) == 8;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const bool present = (__ldg(valid + (i >> 3)) >> (i & 7)) & 1u;
    const unsigned long long v = w8 ? __ldcs(static_cast<const unsigned long long*>(src) + i)
                                    : __ldcs(static_cast<const unsigned*>(src) + i);
    if (w8) {
      if (zero) static_cast<unsigned long long*>(zero)[i] = present ? v : 0ull;
      if (minid) static_cast<unsigned long long*>(minid)[i] = present ? v : min_identity(type);
      if (maxid) static_cast<unsigned long long*>(maxid)[i] = present ? v : max_identity(type);
    } else {
      if (zero) static_cast<unsigned*>(zero)[i] = present ? unsigned(v) : 0u;
      if (minid) static_cast<unsigned*>(minid)[i] = present ? unsigned(v) : unsigned(min_identity(type));
      if (maxid) static_cast<unsigned*>(maxid)[i] = present ? unsigned(v) : unsigned(max_identity(type));
    }
    if (ind) ind[i] = present ? 1 : 0;
  }
}

__global__ void __launch_bounds__(256) k_null_valid(const unsigned long long* count, int64_t g,
                                                    unsigned char* out) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < g; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = __ldg(count + i) > 0 ? 1 : 0;
}

int grid_for(const gba_context* ctx, int64_t n) {
  return int(std::max<int64_t>(1, std::min<int64_t>(int64_t(ctx->sms) * 8, (n + 255) / 256)));
}

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

bool reads_column(int op) { return op != GBA_COUNT; }

}  // namespace

bool gba_nulls_needed(const gba_query& q, const gba_output& o) {
  if (q.key.valid || q.key2.valid) return true;
  for (int c = 0; c < q.n_cols && c < GBA_MAX_COLS; ++c)
    if (q.cols[c].valid) return true;
  for (int a = 0; a < q.n_aggs && a < GBA_MAX_AGGS; ++a)
    if (q.aggs[a].op == GBA_COUNT_VALID || o.agg_valid[a]) return true;
  return false;
}

gba_status gba_nulls_prepare(gba_context* ctx, int nq, const gba_query* qs, const gba_output* outs, gba_query* q2,
                             gba_output* o2, std::vector<NullPlan>* plans, cudaStream_t s) {
  plans->clear();
  struct Prep {
    int query, col;
    size_t off[5];  // scratch offset of each variant (SIZE_MAX: not written)
  };
  std::vector<Prep> preps;
  size_t bytes = 0;
  for (int i = 0; i < nq; ++i) {
    const gba_query& q = qs[i];
    const gba_output& o = outs[i];
    if (!gba_nulls_needed(q, o)) continue;
    const std::string who = "query " + std::to_string(i) + ": ";
    if (q.key.valid || q.key2.valid) {
      ctx->err = who + "null keys are not supported (key.valid and key2.valid must be null)";
      return GBA_ERR_UNSUPPORTED;
    }
    if (q.n_cols < 0 || q.n_cols > GBA_MAX_COLS || q.n_aggs < 0 || q.n_aggs > GBA_MAX_AGGS || q.n_rows < 0 ||
        o.capacity < 0) {
      ctx->err = who + "bad sizes";
      return GBA_ERR_INVALID_ARG;
    }
    NullPlan p;
    p.query = i;
    // new columns: (source column, variant) -> index
    int ncols = 0;
    int idx[GBA_MAX_COLS][5];
    for (auto& r : idx)
      for (int& v : r) v = -1;
    gba_column cols[GBA_MAX_COLS];
    bool too_many = false;
    auto col_of = [&](int c, int v) -> int {
      if (idx[c][v] >= 0) return idx[c][v];
      if (ncols >= GBA_MAX_COLS) {
        too_many = true;
        return 0;
      }
      cols[ncols] = gba_column{};
      cols[ncols].type = v == V_IND ? GBA_I32 : q.cols[c].type;
      cols[ncols].data = q.cols[c].data;  // V_RAW; the others are pointed at scratch below
      idx[c][v] = ncols;
      return ncols++;
    };
    gba_query& qa = q2[i];
    bool need_count[GBA_MAX_COLS] = {};
    int count_agg[GBA_MAX_COLS];  // aggregate whose output is column c's present count
    for (int& x : count_agg) x = -1;
    for (int a = 0; a < q.n_aggs; ++a) {
      const int op = q.aggs[a].op, c = q.aggs[a].col;
      if (!reads_column(op)) continue;
      if (c < 0 || c >= q.n_cols) {
        ctx->err = who + "aggregate column index out of range";
        return GBA_ERR_INVALID_ARG;
      }
      const bool nullable = q.cols[c].valid != nullptr;
      if (!nullable) {
        if (op == GBA_COUNT_VALID) {
          qa.aggs[a].op = GBA_COUNT;
          qa.aggs[a].col = 0;
        } else {
          qa.aggs[a].col = col_of(c, V_RAW);
        }
        continue;
      }
      p.nullable_agg[a] = c;
      switch (op) {
        case GBA_SUM: qa.aggs[a].col = col_of(c, V_ZERO); break;
        case GBA_AVG:
          qa.aggs[a].op = GBA_SUM;
          qa.aggs[a].col = col_of(c, V_ZERO);
          p.avg_on[a] = true;
          need_count[c] = true;
          break;
        case GBA_MIN: qa.aggs[a].col = col_of(c, V_MINID); break;
        case GBA_MAX: qa.aggs[a].col = col_of(c, V_MAXID); break;
        case GBA_COUNT_VALID:
          qa.aggs[a].op = GBA_SUM;
          qa.aggs[a].col = col_of(c, V_IND);
          if (count_agg[c] < 0) count_agg[c] = a;
          p.count_valid_agg[a] = true;
          break;
        default:
          ctx->err = who + "unknown aggregate op";
          return GBA_ERR_INVALID_ARG;
      }
      if (o.agg_valid[a]) need_count[c] = true;
    }
    // hidden present counts, summed into scratch output columns
    int naggs = q.n_aggs;
    for (int c = 0; c < q.n_cols; ++c) {
      if (!need_count[c]) continue;
      if (count_agg[c] >= 0) {
        p.count_of[c] = -1 - count_agg[c];  // the caller's own COUNT(col) output
        continue;
      }
      if (naggs >= GBA_MAX_AGGS) {
        ctx->err = who + "nullable columns: the rewritten query needs more than 8 aggregates";
        return GBA_ERR_UNSUPPORTED;
      }
      qa.aggs[naggs].op = GBA_SUM;
      qa.aggs[naggs].col = col_of(c, V_IND);
      p.count_of[c] = naggs;
      p.hidden_off[naggs] = bytes;
      bytes += a256(size_t(std::max<int64_t>(o.capacity, 1)) * 8);
      ++naggs;
    }
    if (too_many) {
      ctx->err = who + "nullable columns: the rewritten query needs more than 4 columns";
      return GBA_ERR_UNSUPPORTED;
    }
    qa.n_aggs = naggs;
    qa.n_cols = ncols;
    for (int c = 0; c < ncols; ++c) qa.cols[c] = cols[c];
    // scratch for the variants of each nullable column
    for (int c = 0; c < q.n_cols; ++c) {
      if (!q.cols[c].valid) continue;
      Prep pr{i, c, {SIZE_MAX, SIZE_MAX, SIZE_MAX, SIZE_MAX, SIZE_MAX}};
      bool any = false;
      for (int v = V_ZERO; v <= V_IND; ++v) {
        if (idx[c][v] < 0) continue;
        pr.off[v] = bytes;
        const int w = v == V_IND ? 4 : gba_type_bytes(q.cols[c].type);
        bytes += a256(size_t(std::max<int64_t>(q.n_rows, 1)) * w);
        any = true;
      }
      if (any) preps.push_back(pr);
    }
    for (int c = 0; c < GBA_MAX_COLS; ++c)
      for (int v = 0; v < 5; ++v) p.col_index[c][v] = idx[c][v];
    plans->push_back(p);
  }
  if (plans->empty()) return GBA_OK;
  if (bytes > ctx->null_bytes) {
    if (ctx->null_buf) {
      GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
      cudaFree(ctx->null_buf);
      ctx->null_buf = nullptr;
      ctx->null_bytes = 0;
    }
    GBA_CUDA_TRY(ctx, cudaMalloc(&ctx->null_buf, std::max<size_t>(bytes, 256)));
    ctx->null_bytes = std::max<size_t>(bytes, 256);
  }
  unsigned char* B = static_cast<unsigned char*>(ctx->null_buf);
  for (NullPlan& p : *plans)
    for (int a = 0; a < q2[p.query].n_aggs; ++a)
      if (p.hidden_off[a] != SIZE_MAX) o2[p.query].aggs[a] = B + p.hidden_off[a];
  for (const Prep& pr : preps) {
    const gba_query& q = qs[pr.query];
    const NullPlan* p = nullptr;
    for (const NullPlan& x : *plans)
      if (x.query == pr.query) p = &x;
    for (int v = V_ZERO; v <= V_IND; ++v)
      if (pr.off[v] != SIZE_MAX) q2[pr.query].cols[p->col_index[pr.col][v]].data = B + pr.off[v];
    if (q.n_rows > 0) {
      auto at = [&](int v) -> void* { return pr.off[v] == SIZE_MAX ? nullptr : B + pr.off[v]; };
      k_null_prep<<<grid_for(ctx, q.n_rows), 256, 0, s>>>(q.cols[pr.col].data, q.cols[pr.col].valid,
                                                          q.cols[pr.col].type, q.n_rows, at(V_ZERO), at(V_MINID),
                                                          at(V_MAXID), static_cast<int*>(at(V_IND)));
      GBA_CUDA_TRY(ctx, cudaGetLastError());
      ctx->stats.kernel_launches += 1;
    }
  }
  for (int i = 0; i < nq; ++i)
    for (int a = 0; a < GBA_MAX_AGGS; ++a) o2[i].agg_valid[a] = nullptr;  // written here, not below
  return GBA_OK;
}

gba_status gba_nulls_finish(gba_context* ctx, const std::vector<NullPlan>& plans, const gba_query* qs,
                            const gba_output* outs, const gba_output* o2, const int64_t* n_groups, cudaStream_t s) {
  int launches = 0;
  for (const NullPlan& p : plans) {
    const gba_query& q = qs[p.query];
    const gba_output& o = outs[p.query];
    const int64_t g = std::min<int64_t>(n_groups[p.query], o.capacity);
    if (g <= 0) continue;
    auto count_ptr = [&](int c) -> const unsigned long long* {
      const int k = p.count_of[c];
      return static_cast<const unsigned long long*>(k < 0 ? o.aggs[-1 - k] : o2[p.query].aggs[k]);
    };
    // AVG over nullable columns: SUM / present count, one launch per column
    for (int c = 0; c < q.n_cols; ++c) {
      AvgDesc d{};
      for (int a = 0; a < q.n_aggs; ++a)
        if (p.avg_on[a] && p.nullable_agg[a] == c) {
          d.col[d.n] = static_cast<unsigned long long*>(o.aggs[a]);
          d.fp[d.n] = q.cols[c].type == GBA_F32 || q.cols[c].type == GBA_F64;
          ++d.n;
        }
      if (d.n == 0) continue;
      d.count = count_ptr(c);
      GBA_CUDA_TRY(ctx, gba_launch_avg_finish(d, g, ctx->sms, s));
      ++launches;
    }
    for (int a = 0; a < q.n_aggs; ++a) {
      unsigned char* v = o.agg_valid[a];
      if (!v) continue;
      if (p.nullable_agg[a] >= 0 && !p.count_valid_agg[a]) {
        k_null_valid<<<grid_for(ctx, g), 256, 0, s>>>(count_ptr(p.nullable_agg[a]), g, v);
        GBA_CUDA_TRY(ctx, cudaGetLastError());
        ++launches;
      } else {
        GBA_CUDA_TRY(ctx, cudaMemsetAsync(v, 1, size_t(g), s));  // COUNT and non-null columns are never NULL
      }
    }
  }
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  ctx->stats.kernel_launches += launches;
  return GBA_OK;
}
