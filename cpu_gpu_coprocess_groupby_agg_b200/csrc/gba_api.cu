// C ABI: contexts, workspace, query validation and the single-query driver.
//
// The reference drives one query as a host loop over tiles with ~6 blocking
// stream syncs per tile (tiled_groupby_agg_partition/src/group_then_partition.cu:
// 332-424) and a second host loop over merged partitions
// (groupby_agg_intra_partition.cu:183-277).  Here one query is three to five
// kernel launches on one stream with a single host sync at the end, which reads
// the overflow flags and the group count.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "gba_context.h"
#include "gba_plan.h"
#include "composite.h"
#include "nulls.h"
#include "sort_kernels.h"

size_t gba_round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
uint64_t gba_pow2_ceil(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

extern "C" void gba_default_knobs(gba_knobs* k) {
  std::memset(k, 0, sizeof(*k));
  k->sizing = GBA_SIZING_PLAIN;
  k->strategy = GBA_STRATEGY_AUTO;
  k->load_factor = 0.5;
  k->preagg = -1;
  k->use_tma = -1;
  k->coalesce = -1;
  k->max_regrow = 4;
  k->use_graph = -1;
  k->exchange = 0;  // owner exchange: opt-in until measured
}

extern "C" const char* gba_status_string(gba_status s) {
  switch (s) {
    case GBA_OK: return "ok";
    case GBA_ERR_INVALID_ARG: return "invalid argument";
    case GBA_ERR_CUDA: return "CUDA error";
    case GBA_ERR_OOM: return "out of device memory";
    case GBA_ERR_OUTPUT_CAPACITY: return "output capacity too small";
    case GBA_ERR_TABLE_OVERFLOW: return "hash table overflow after regrow limit";
    case GBA_ERR_TIMEOUT: return "bounded device wait timed out";
    case GBA_ERR_UNSUPPORTED: return "unsupported";
    case GBA_ERR_BUDGET: return "request exceeds the device-memory budget";
  }
  return "unknown status";
}

extern "C" gba_status gba_create(gba_context** out, int32_t device) {
  if (!out) return GBA_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return GBA_ERR_CUDA;
  gba_context* ctx = new gba_context();
  ctx->device = device;
  cudaSetDevice(device);
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&ctx->max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return GBA_ERR_CUDA;
  }
  for (auto& e : ctx->ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  for (auto& e : ctx->tev) cudaEventCreate(&e);
  gba_status st = gba_small_reserve(ctx, 1 << 16);
  if (st != GBA_OK) {
    gba_destroy(ctx);
    return st;
  }
  *out = ctx;
  return GBA_OK;
}

extern "C" gba_status gba_destroy(gba_context* ctx) {
  if (!ctx) return GBA_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->stage) cudaFree(ctx->stage);
  if (ctx->d_small) cudaFree(ctx->d_small);
  if (ctx->h_small) cudaFreeHost(ctx->h_small);
  if (ctx->d_est) cudaFree(ctx->d_est);
  if (ctx->est_ws) cudaFree(ctx->est_ws);
  for (auto& e : ctx->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : ctx->tev)
    if (e) cudaEventDestroy(e);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->out_stream) cudaStreamDestroy(ctx->out_stream);
  for (auto& e : ctx->part_ev) cudaEventDestroy(e);
  if (ctx->batch_exec) cudaGraphExecDestroy(ctx->batch_exec);
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  if (ctx->aux_stream) cudaStreamDestroy(ctx->aux_stream);
  for (auto& e : ctx->fork_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->h_batch) cudaFreeHost(ctx->h_batch);
  if (ctx->rp_buf) cudaFree(ctx->rp_buf);
  if (ctx->avg_buf) cudaFree(ctx->avg_buf);
  if (ctx->ck_buf) cudaFree(ctx->ck_buf);
  if (ctx->null_buf) cudaFree(ctx->null_buf);
  delete ctx;
  return GBA_OK;
}

extern "C" const char* gba_last_error(const gba_context* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

extern "C" gba_status gba_last_stats(const gba_context* ctx, gba_stats* out) {
  if (!ctx || !out) return GBA_ERR_INVALID_ARG;
  *out = ctx->stats;
  return GBA_OK;
}

// Device buffers grow to at least 1.5 times their old size, so that a
// workload whose calls need a little more each time (a server's batches of
// varying shapes) reallocates a few times, not at every new high: each
// reallocation synchronises the device, stalling every stream on it.  If the
// larger block does not fit, the exact size is tried.
static cudaError_t grow_alloc(void** p, size_t bytes, size_t cur, size_t min_bytes, size_t* got) {
  const size_t exact = gba_round_up(std::max(bytes, min_bytes), size_t(1) << 21);
  const size_t roomy = gba_round_up(std::max(exact, cur + cur / 2), size_t(1) << 21);
  cudaError_t e = cudaMalloc(p, roomy);
  if (e == cudaSuccess) {
    *got = roomy;
    return e;
  }
  cudaGetLastError();
  if (roomy == exact) return e;
  e = cudaMalloc(p, exact);
  if (e == cudaSuccess) *got = exact;
  return e;
}

gba_status gba_ws_reserve(gba_context* ctx, size_t bytes, cudaStream_t s) {
  if (bytes <= ctx->ws_bytes) return GBA_OK;
  const size_t cur = ctx->ws_bytes;
  if (ctx->ws) {
    GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    GBA_CUDA_TRY(ctx, cudaDeviceSynchronize());
    cudaFree(ctx->ws);
    ctx->ws = nullptr;
    ctx->ws_bytes = 0;
  }
  size_t want = 0;
  cudaError_t e = grow_alloc(&ctx->ws, bytes, cur, size_t(1) << 24, &want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    ctx->ws = nullptr;
    ctx->err = std::string("workspace cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e);
    return GBA_ERR_OOM;
  }
  ctx->ws_bytes = want;
  return GBA_OK;
}

gba_status gba_stage_reserve(gba_context* ctx, size_t bytes, cudaStream_t s) {
  if (bytes <= ctx->stage_bytes) return GBA_OK;
  const size_t cur = ctx->stage_bytes;
  if (ctx->stage) {
    GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    GBA_CUDA_TRY(ctx, cudaDeviceSynchronize());
    cudaFree(ctx->stage);
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
  }
  size_t want = 0;
  cudaError_t e = grow_alloc(&ctx->stage, bytes, cur, size_t(1) << 24, &want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    ctx->stage = nullptr;
    ctx->err = std::string("staging cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e);
    return GBA_ERR_OOM;
  }
  ctx->stage_bytes = want;
  return GBA_OK;
}

gba_status gba_est_reserve(gba_context* ctx, size_t bytes, cudaStream_t s) {
  if (bytes <= ctx->est_ws_bytes) return GBA_OK;
  const size_t cur = ctx->est_ws_bytes;
  if (ctx->est_ws) {
    GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    GBA_CUDA_TRY(ctx, cudaDeviceSynchronize());
    cudaFree(ctx->est_ws);
    ctx->est_ws = nullptr;
    ctx->est_ws_bytes = 0;
  }
  size_t want = 0;
  GBA_CUDA_TRY(ctx, grow_alloc(&ctx->est_ws, bytes, cur, size_t(1) << 22, &want));
  ctx->est_ws_bytes = want;
  return GBA_OK;
}

gba_status gba_batch_host_reserve(gba_context* ctx, size_t bytes) {
  if (bytes <= ctx->h_batch_bytes) return GBA_OK;
  const size_t prev = ctx->h_batch_bytes;  // pinned buffers grow by 1.5 times too
  if (ctx->h_batch) cudaFreeHost(ctx->h_batch);
  ctx->h_batch = nullptr;
  ctx->h_batch_bytes = 0;
  const size_t want = gba_round_up(std::max({bytes, size_t(1) << 20, prev + prev / 2}), size_t(1) << 16);
  GBA_CUDA_TRY(ctx, cudaMallocHost(&ctx->h_batch, want));
  ctx->h_batch_bytes = want;
  return GBA_OK;
}

gba_status gba_small_reserve(gba_context* ctx, size_t bytes) {
  if (bytes <= ctx->d_small_bytes) return GBA_OK;
  cudaDeviceSynchronize();
  if (ctx->d_small) cudaFree(ctx->d_small);
  if (ctx->h_small) cudaFreeHost(ctx->h_small);
  ctx->d_small = nullptr;
  ctx->h_small = nullptr;
  ctx->d_small_bytes = ctx->h_small_bytes = 0;
  GBA_CUDA_TRY(ctx, cudaMalloc(&ctx->d_small, bytes));
  GBA_CUDA_TRY(ctx, cudaMallocHost(&ctx->h_small, bytes));
  ctx->d_small_bytes = ctx->h_small_bytes = bytes;
  return GBA_OK;
}

void GbaTimer::begin(int r) {
  if (!on || n >= 8) return;
  role[n] = r;
  cudaEventRecord(ctx->tev[2 * n], s);
}
void GbaTimer::end() {
  if (!on || n >= 8) return;
  cudaEventRecord(ctx->tev[2 * n + 1], s);
  ++n;
}
void GbaTimer::collect() {
  for (int i = 0; i < n; ++i) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->tev[2 * i], ctx->tev[2 * i + 1]) == cudaSuccess)
      ctx->stats.kernel_ms[role[i]] += ms;
  }
  n = 0;
}

gba_status gba_build_qdesc(gba_context* ctx, const gba_query* q, QDesc* d) {
  if (!q) return GBA_ERR_INVALID_ARG;
  std::memset(d, 0, sizeof(*d));
  if (q->n_rows < 0) {
    ctx->err = "n_rows < 0";
    return GBA_ERR_INVALID_ARG;
  }
  if (q->key.type != GBA_I32 && q->key.type != GBA_U32 && q->key.type != GBA_I64) {
    ctx->err = "key type must be GBA_I32, GBA_U32 or GBA_I64";
    return GBA_ERR_INVALID_ARG;
  }
  if (q->n_cols < 0 || q->n_cols > GBA_MAX_COLS || q->n_aggs < 1 || q->n_aggs > GBA_MAX_AGGS) {
    ctx->err = "n_cols must be in [0, 4] and n_aggs in [1, 8]";
    return GBA_ERR_INVALID_ARG;
  }
  if (q->n_rows > 0 && !q->key.data) {
    ctx->err = "null key column";
    return GBA_ERR_INVALID_ARG;
  }
  if (q->key2.data) {
    ctx->err = "composite keys are supported by gba_groupby and gba_groupby_batch only";
    return GBA_ERR_UNSUPPORTED;
  }
  bool nullable = q->key.valid != nullptr;
  for (int c = 0; c < q->n_cols && c < GBA_MAX_COLS; ++c) nullable = nullable || q->cols[c].valid != nullptr;
  for (int a = 0; a < q->n_aggs && a < GBA_MAX_AGGS; ++a) nullable = nullable || q->aggs[a].op == GBA_COUNT_VALID;
  if (nullable) {
    ctx->err = "nullable columns and COUNT(col) are supported by gba_groupby and gba_groupby_batch only";
    return GBA_ERR_UNSUPPORTED;
  }
  d->keys = q->key.data;
  d->n = q->n_rows;
  d->key64 = q->key.type == GBA_I64;
  d->ncols = q->n_cols;
  for (int c = 0; c < q->n_cols; ++c) {
    const int t = q->cols[c].type;
    if (t != GBA_I32 && t != GBA_U32 && t != GBA_I64 && t != GBA_F32 && t != GBA_F64) {
      ctx->err = "bad column type";
      return GBA_ERR_INVALID_ARG;
    }
    if (q->n_rows > 0 && !q->cols[c].data) {
      ctx->err = "null value column";
      return GBA_ERR_INVALID_ARG;
    }
    d->cols[c] = q->cols[c].data;
    d->col_type[c] = t;
  }
  d->naccs = q->n_aggs;
  for (int a = 0; a < q->n_aggs; ++a) {
    const int op = q->aggs[a].op, c = q->aggs[a].col;
    if (op == GBA_COUNT) {
      d->acc_op[a] = ACC_CNT;
      d->acc_col[a] = 0;
      d->acc_ctype[a] = GBA_I64;
      continue;
    }
    if (c < 0 || c >= q->n_cols) {
      ctx->err = "aggregate column index out of range";
      return GBA_ERR_INVALID_ARG;
    }
    const int t = q->cols[c].type;
    d->acc_col[a] = c;
    d->acc_ctype[a] = t;
    if ((t == GBA_F32 || t == GBA_F64) && op != GBA_AVG) {
      if (op != GBA_SUM) {
        ctx->err = "only SUM (and AVG) are supported on fp32 and fp64 columns";
        return GBA_ERR_UNSUPPORTED;
      }
      d->acc_op[a] = ACC_ADD_F;
    } else if (op == GBA_SUM) d->acc_op[a] = ACC_ADD_I;
    else if (op == GBA_MIN) d->acc_op[a] = ACC_MIN_I;
    else if (op == GBA_MAX) d->acc_op[a] = ACC_MAX_I;
    else if (op == GBA_AVG) {
      ctx->err = "AVG is supported by gba_groupby and gba_groupby_batch only";
      return GBA_ERR_UNSUPPORTED;
    } else {
      ctx->err = "unknown aggregate op";
      return GBA_ERR_INVALID_ARG;
    }
  }
  int w = 0;
  for (int a = 0; a < q->n_aggs; ++a) {
    d->acc_woff[a] = w;
    w += gba_acc_smem_words(d->acc_op[a]);
  }
  d->nwords = w;
  return GBA_OK;
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Drops value columns no aggregate reads (they are never streamed) and remaps
// the aggregates' column indices; aggregate order is unchanged.
void gba_compact_query(const gba_query* in, gba_query* out) {
  *out = *in;
  int remap[GBA_MAX_COLS];
  int nc = 0;
  for (int c = 0; c < in->n_cols && c < GBA_MAX_COLS; ++c) {
    bool used = false;
    for (int a = 0; a < in->n_aggs && a < GBA_MAX_AGGS; ++a)
      used = used || (in->aggs[a].op != GBA_COUNT && in->aggs[a].col == c);
    remap[c] = used ? nc : -1;
    if (used) out->cols[nc++] = in->cols[c];
  }
  out->n_cols = nc;
  for (int a = 0; a < in->n_aggs && a < GBA_MAX_AGGS; ++a) {
    const int c = in->aggs[a].col;
    if (in->aggs[a].op == GBA_COUNT) out->aggs[a].col = 0;
    else out->aggs[a].col = (c >= 0 && c < in->n_cols && c < GBA_MAX_COLS) ? remap[c] : c;
  }
}

// ---------------------------------------------------------------------------
// Plan: everything the single-query driver decides before launching.
void gba_make_plan(const gba_context* ctx, const QDesc& q, const gba_knobs& k, double predicted_groups,
                   GbaPlan* p) {
  p->block = k.block_threads > 0 ? k.block_threads : 1024;
  p->block = std::min(1024, std::max(128, p->block / 32 * 32));
  // TMA staging: about 96 KB of bulk copies in flight per SM reach the HBM read
  // peak with one CTA per SM (measured: 2 x 32 KB -> 6.9 TB/s, 3 x 32 KB ->
  // 7.3 TB/s, 2 x 16 KB -> 4.7 TB/s); tiles of at least 24 KB, 2-4 stages
  size_t rb = q.key64 ? 8 : 4;
  for (int c = 0; c < q.ncols; ++c) rb += gba_type_bytes(q.col_type[c]);
  // Tiles are long enough that the per-tile barriers stay a small share of the
  // work (measured with ncu on 2048-row tiles: barrier stalls dominated).
  int T = 2048;
  while (T < 8192 && size_t(T) * rb < 32 * 1024) T *= 2;
  p->tile_rows = k.tile_rows > 0 ? k.tile_rows : T;
  // tiles are multiples of the block; miss lists index a tile with 16 bits
  p->tile_rows = std::min(32768, std::max(p->block, p->tile_rows / p->block * p->block));
  const size_t stage = size_t(p->tile_rows) * rb;
  p->nstages = k.nstages > 0 ? std::min(4, k.nstages) : int(std::min<size_t>(4, std::max<size_t>(2, (98304 + stage - 1) / stage)));
  const int64_t ntiles = (q.n + p->tile_rows - 1) / p->tile_rows;
  const int bps = k.blocks_per_sm > 0 ? k.blocks_per_sm : 1;
  p->grid = int(std::max<int64_t>(1, std::min<int64_t>(ntiles, int64_t(ctx->sms) * bps)));

  bool tma_ok = aligned16(q.keys) && q.n >= p->tile_rows;
  for (int c = 0; c < q.ncols; ++c) tma_ok = tma_ok && aligned16(q.cols[c]);
  p->use_tma = k.use_tma == 0 ? 0 : (tma_ok ? 1 : 0);
  // measured: __match_any_sync pre-combining costs more than it saves unless a
  // warp sees long runs of one key, so it is opt-in
  p->coalesce = k.coalesce == 1 ? 1 : 0;

  // HBM table capacity.  PLAIN: the only bound known without an estimate is the
  // row count, at a fixed load factor (default 0.5), rounded to a power of two.
  // LEARNED: 1.25x the predicted groups at load learned_load (default 0.35;
  // any size: slots are addressed by a multiply-shift of the hash), so most
  // keys sit in their home slot (measured on the 256-query batch: a whole step
  // takes 24.6 ms at 0.35, 26.2 ms at 0.5, 29.2 ms at 0.7); an
  // under-estimate overflows and regrows.
  const double lf = (k.load_factor > 0.05 && k.load_factor < 0.95) ? k.load_factor : 0.5;
  const double llf = (k.learned_load > 0.05 && k.learned_load < 0.95) ? k.learned_load : 0.35;
  uint64_t cap;
  // GROW: the plain capacity, capped at a modest start (table_slots, default
  // 2^16 slots); a table that overflows regrows 4x per rerun, the estimator-free
  // alternative to sizing by the row count.
  if (k.sizing == GBA_SIZING_FIXED && k.table_slots > 0) cap = uint64_t(k.table_slots);
  else if (k.sizing == GBA_SIZING_GROW)
    cap = std::min<uint64_t>(gba_pow2_ceil(uint64_t(double(std::max<int64_t>(q.n, 1)) / lf)),
                             k.table_slots > 0 ? uint64_t(k.table_slots) : (uint64_t(1) << 16));
  else if (k.sizing == GBA_SIZING_LEARNED && predicted_groups > 0)
    cap = uint64_t(std::min(double(std::max<int64_t>(q.n, 1)), predicted_groups * 1.25 + 64.0) / llf) + 1;
  else cap = gba_pow2_ceil(uint64_t(double(std::max<int64_t>(q.n, 1)) / lf));
  p->table_slots = std::max<uint64_t>(cap, 64);
  p->probe_cap = k.probe_cap > 0 ? k.probe_cap : 256;

  // shared-memory table: whatever the pipeline leaves of the opt-in budget
  int preagg = k.preagg;
  if (preagg < 0) {
    preagg = 1;
    if (k.sizing == GBA_SIZING_LEARNED && predicted_groups > 0 && q.n > 0) {
      // A CTA's shared table catches a row when its key is among the few
      // thousand the table holds: worth it when the groups fit a handful of
      // tables, or when the sample shows hot keys (the top key alone holds
      // >= 0.1% of the rows); otherwise every row pays a lookup and a miss.
      const double slots = double(ctx->max_smem_optin) / double((q.key64 ? 8 : 4) + 4 * q.nwords);
      if (predicted_groups > 4.0 * slots && ctx->est_skew < 1e-3) preagg = 0;
      if (predicted_groups > 0.5 * double(q.n)) preagg = 0;  // nearly all keys distinct
    }
  }
  p->preagg = preagg;
  const size_t slot_bytes = (q.key64 ? 8 : 4) + 4 * size_t(q.nwords);
  auto slots_with = [&](int use_tma) {
    const size_t fixed = gba_preagg_smem_bytes(q, 0, p->tile_rows, p->nstages, use_tma);
    const size_t room = size_t(ctx->max_smem_optin) > fixed + 1024 ? size_t(ctx->max_smem_optin) - fixed - 1024 : 0;
    int S = int(std::min<size_t>(room / slot_bytes, 16384));
    if (k.smem_slots > 0) S = std::min(S, k.smem_slots);
    return S < 32 ? 0 : S;
  };
  // The staging competes with the shared table.  When the groups are known to
  // exceed what the table left beside the TMA stages can hold, drop TMA and
  // give the table all of shared memory (rows are then loaded straight into
  // registers, two per thread in flight).
  if (p->use_tma && k.use_tma < 0 && preagg && predicted_groups > 0 &&
      predicted_groups > 0.5 * slots_with(1))
    p->use_tma = 0;
  if (!p->use_tma && k.tile_rows <= 0) {
    // without staging a tile costs only its 2-byte miss entries
    p->tile_rows = std::max(p->block, 8192 / p->block * p->block);
    const int64_t nt = (q.n + p->tile_rows - 1) / p->tile_rows;
    p->grid = int(std::max<int64_t>(1, std::min<int64_t>(nt, int64_t(ctx->sms) * (k.blocks_per_sm > 0 ? k.blocks_per_sm : 1))));
  }
  p->smem_slots = preagg ? slots_with(p->use_tma) : 0;
  // a full table makes every miss walk the whole probe window: keep it short
  p->smem_probe_cap = k.smem_probe_cap > 0 ? k.smem_probe_cap : 8;
  p->partition_bits = k.partition_bits;
}

// One attempt of the table strategy with capacity p.table_slots.
static gba_status run_table_once(gba_context* ctx, const QDesc& q, const gba_output* out, const GbaPlan& p,
                                 cudaStream_t s, bool timing, unsigned* flags_out, unsigned long long* count_out) {
  GbaTimer tm{ctx, s, timing};
  const size_t stride = size_t(gba_gt_stride(q.naccs));
  const size_t table_bytes = (p.table_slots + 1) * stride * 8;
  gba_status st = gba_ws_reserve(ctx, table_bytes, s);
  if (st != GBA_OK) return st;
  unsigned* d_flags = reinterpret_cast<unsigned*>(ctx->d_small);
  unsigned long long* d_count = reinterpret_cast<unsigned long long*>(ctx->d_small + 8);
  GBA_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_small, 0, 64, s));
  GTable t;
  t.base = static_cast<unsigned long long*>(ctx->ws);
  t.cap = p.table_slots;
  t.probe_cap = p.probe_cap;
  const int init_grid = int(std::min<uint64_t>(uint64_t(ctx->sms) * 16, (table_bytes / 8 + 255) / 256 + 1));
  tm.begin(0);
  GBA_CUDA_TRY(ctx, gba_launch_table_init(t, q, init_grid, s));
  tm.end();
  int launches = 1;
  if (q.n > 0) {
    PreaggCfg c;
    c.grid = p.grid;
    c.block = p.block;
    c.smem_slots = p.smem_slots;
    c.smem_probe_cap = p.smem_probe_cap;
    c.tile_rows = p.tile_rows;
    c.nstages = p.nstages;
    c.use_tma = p.use_tma;
    c.coalesce = p.coalesce;
    tm.begin(1);
    GBA_CUDA_TRY(ctx, gba_launch_preagg(q, t, c, d_flags, s));
    tm.end();
    ++launches;
    ctx->stats.main_rows += q.n;
    ctx->stats.main_bytes += q.n * int64_t(gba_row_bytes(q));
  }
  OutDesc o;
  o.keys = out->keys;
  for (int a = 0; a < GBA_MAX_AGGS; ++a) o.accs[a] = static_cast<unsigned long long*>(out->aggs[a]);
  o.capacity = out->capacity;
  o.count = d_count;
  const int cgrid = int(std::min<uint64_t>(uint64_t(ctx->sms) * 8, (p.table_slots + 255) / 256));
  tm.begin(2);
  GBA_CUDA_TRY(ctx, gba_launch_compact(t, q, o, std::max(cgrid, 1), s));
  tm.end();
  ++launches;
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_small, ctx->d_small, 16, cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  tm.collect();
  *flags_out = *reinterpret_cast<unsigned*>(ctx->h_small);
  *count_out = *reinterpret_cast<unsigned long long*>(ctx->h_small + 8);
  ctx->stats.kernel_launches += launches;
  return GBA_OK;
}

gba_status gba_run_table(gba_context* ctx, const QDesc& q, const gba_output* out, const gba_knobs& k, GbaPlan p,
                         cudaStream_t s, int64_t* n_groups) {
  ctx->stats.strategy = GBA_STRATEGY_TABLE;
  for (int attempt = 0;; ++attempt) {
    unsigned flags = 0;
    unsigned long long count = 0;
    gba_status st = run_table_once(ctx, q, out, p, s, k.timing != 0, &flags, &count);
    if (st != GBA_OK) return st;
    ctx->stats.table_slots = int64_t(p.table_slots);
    ctx->stats.preagg = p.smem_slots > 0;
    if (flags & GBA_FLAG_WAIT_TIMEOUT) {
      ctx->err = "a bounded TMA wait timed out";
      return GBA_ERR_TIMEOUT;
    }
    if (flags & GBA_FLAG_TABLE_OVERFLOW) {
      if (attempt >= k.max_regrow) {
        ctx->err = "HBM hash table overflow after " + std::to_string(attempt) + " regrows";
        return GBA_ERR_TABLE_OVERFLOW;
      }
      ctx->stats.regrows++;
      p.table_slots *= 4;
      continue;
    }
    *n_groups = int64_t(count);
    ctx->stats.n_groups = int64_t(count);
    if (int64_t(count) > out->capacity) {
      ctx->err = "output capacity " + std::to_string(out->capacity) + " < " + std::to_string(count) + " groups";
      return GBA_ERR_OUTPUT_CAPACITY;
    }
    return GBA_OK;
  }
}

static gba_status check_output(gba_context* ctx, const gba_query* q, const gba_output* out) {
  if (!out || out->capacity < 0 || (out->capacity > 0 && !out->keys)) {
    ctx->err = "bad output descriptor";
    return GBA_ERR_INVALID_ARG;
  }
  for (int a = 0; a < q->n_aggs; ++a)
    if (out->capacity > 0 && !out->aggs[a]) {
      ctx->err = "null output aggregate column";
      return GBA_ERR_INVALID_ARG;
    }
  return GBA_OK;
}

static gba_status groupby_device(gba_context* ctx, const gba_query* q, const gba_output* out,
                                 const gba_knobs* knobs, void* stream, int64_t* n_groups);

static gba_status groupby_avg(gba_context* ctx, const gba_query* q, const gba_output* out,
                              const gba_knobs* knobs, void* stream, int64_t* n_groups);

// Composite keys are packed into one 64-bit key around the call; key order
// (knobs->sort_output) is a device sort of the finished groups.
extern "C" gba_status gba_groupby(gba_context* ctx, const gba_query* q, const gba_output* out,
                                  const gba_knobs* knobs, void* stream, int64_t* n_groups) {
  if (!ctx || !q || !n_groups) return GBA_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // nullable columns: rewritten columns and aggregates (qn, on)
  gba_query qn = *q;
  gba_output on = out ? *out : gba_output{};
  std::vector<NullPlan> np;
  if (out && gba_nulls_needed(*q, *out)) {
    cudaSetDevice(ctx->device);
    gba_status st = gba_nulls_prepare(ctx, 1, q, out, &qn, &on, &np, s);
    if (st != GBA_OK) return st;
  }
  // composite keys: packed key columns (qq, oo)
  gba_query qq = qn;
  gba_output oo = on;
  std::vector<CompositeJob> cj;
  if (qn.key2.data) {
    if (!out) return GBA_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    gba_status st = gba_composite_prepare(ctx, 1, &qn, &on, &qq, &oo, &cj, s);
    if (st != GBA_OK) return st;
  }
  gba_status st = groupby_avg(ctx, &qq, out ? &oo : nullptr, knobs, stream, n_groups);
  if (st != GBA_OK) return st;
  if (knobs && knobs->sort_output) {
    SortJob j = gba_sort_job(&qq, &oo, std::min<int64_t>(*n_groups, oo.capacity));
    if (!cj.empty()) j.key_signed = 0;  // the packed pair orders as an unsigned word
    st = gba_sort_groups(ctx, &j, 1, s);
    if (st != GBA_OK) return st;
  }
  if (!cj.empty()) {
    st = gba_composite_finish(ctx, cj, &on, n_groups, s);
    if (st != GBA_OK) return st;
  }
  if (!np.empty()) return gba_nulls_finish(ctx, np, q, out, &on, n_groups, s);
  return GBA_OK;
}

// AVG: the query runs with each AVG as a SUM into the caller's column and one
// COUNT (the query's own, or one added into a context buffer); a last kernel
// turns each SUM column into SUM / COUNT in place.
static gba_status groupby_avg(gba_context* ctx, const gba_query* q, const gba_output* out,
                              const gba_knobs* knobs, void* stream, int64_t* n_groups) {
  if (!ctx || !q || !n_groups) return GBA_ERR_INVALID_ARG;
  int navg = 0, cnt = -1;
  for (int a = 0; a < q->n_aggs && a < GBA_MAX_AGGS; ++a) {
    navg += q->aggs[a].op == GBA_AVG;
    if (q->aggs[a].op == GBA_COUNT && cnt < 0) cnt = a;
  }
  if (navg == 0) return groupby_device(ctx, q, out, knobs, stream, n_groups);
  if (!out || out->capacity < 0) return GBA_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  gba_query qa = *q;
  gba_output oa = *out;
  AvgDesc ad{};
  for (int a = 0; a < q->n_aggs; ++a) {
    if (q->aggs[a].op != GBA_AVG) continue;
    const int c = q->aggs[a].col;
    if (c < 0 || c >= q->n_cols) {
      ctx->err = "aggregate column index out of range";
      return GBA_ERR_INVALID_ARG;
    }
    qa.aggs[a].op = GBA_SUM;
    ad.col[ad.n] = static_cast<unsigned long long*>(out->aggs[a]);
    ad.fp[ad.n] = q->cols[c].type == GBA_F32 || q->cols[c].type == GBA_F64;
    ++ad.n;
  }
  if (cnt < 0) {
    if (qa.n_aggs >= GBA_MAX_AGGS) {
      ctx->err = "AVG needs a COUNT: at most 7 aggregates with AVG and no COUNT";
      return GBA_ERR_INVALID_ARG;
    }
    const size_t bytes = size_t(std::max<int64_t>(out->capacity, 1)) * 8;
    if (bytes > ctx->avg_bytes) {
      if (ctx->avg_buf) {
        GBA_CUDA_TRY(ctx, cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
        cudaFree(ctx->avg_buf);
        ctx->avg_buf = nullptr;
        ctx->avg_bytes = 0;
      }
      GBA_CUDA_TRY(ctx, cudaMalloc(&ctx->avg_buf, bytes));
      ctx->avg_bytes = bytes;
    }
    cnt = qa.n_aggs++;
    qa.aggs[cnt].op = GBA_COUNT;
    qa.aggs[cnt].col = 0;
    oa.aggs[cnt] = ctx->avg_buf;
  }
  ad.count = static_cast<const unsigned long long*>(oa.aggs[cnt]);
  gba_status st = groupby_device(ctx, &qa, &oa, knobs, stream, n_groups);
  if (st != GBA_OK) return st;
  const int64_t g = std::min<int64_t>(*n_groups, out->capacity);
  if (g > 0) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    GBA_CUDA_TRY(ctx, gba_launch_avg_finish(ad, g, ctx->sms, s));
    GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    ctx->stats.kernel_launches += 1;
  }
  return GBA_OK;
}

static gba_status groupby_device(gba_context* ctx, const gba_query* q, const gba_output* out,
                                 const gba_knobs* knobs, void* stream, int64_t* n_groups) {
  if (!ctx || !q || !n_groups) return GBA_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  ctx->stats = gba_stats{};
  ctx->stats.predicted_groups = -1;
  gba_knobs k;
  if (knobs) k = *knobs;
  else gba_default_knobs(&k);
  gba_query qc;
  gba_compact_query(q, &qc);
  q = &qc;
  QDesc qd;
  gba_status st = gba_build_qdesc(ctx, q, &qd);
  if (st != GBA_OK) return st;
  st = check_output(ctx, q, out);
  if (st != GBA_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  double pred = -1;
  // A query whose plain-sized table is small (<= 256 MB: about 5M rows with two
  // aggregates) costs less with that table than the estimator's sampling pass
  // and host round trip (measured: a 2^20-row query takes 0.13 ms plain, 0.37
  // ms with the estimator), so learned sizing sizes it plainly.  A batch pays
  // for one sampling pass over all its queries and always uses the estimate.
  // (knobs.learned_min_rows overrides the rule: a row count, or -1 for never)
  const double plain_table_bytes =
      double(gba_pow2_ceil(uint64_t(std::max<int64_t>(qd.n, 1)) * 2)) * 8.0 * double(1 + qd.naccs);
  const bool small = k.learned_min_rows > 0   ? qd.n < k.learned_min_rows
                     : k.learned_min_rows == 0 ? plain_table_bytes <= double(int64_t(256) << 20)
                                               : false;
  if (k.sizing == GBA_SIZING_LEARNED && small) k.sizing = GBA_SIZING_PLAIN;
  if (k.sizing == GBA_SIZING_LEARNED) {
    if (!ctx->est_loaded) {
      ctx->err = "learned sizing requested but no estimator weights are loaded";
      return GBA_ERR_INVALID_ARG;
    }
    st = gba_predict_groups(ctx, qd, s, &pred);
    if (st != GBA_OK) return st;
    ctx->stats.predicted_groups = pred;
  }
  GbaPlan p;
  gba_make_plan(ctx, qd, k, pred, &p);
  int strategy = k.strategy;
  if (strategy == GBA_STRATEGY_AUTO) strategy = gba_choose_strategy(ctx, qd, k, pred, p);
  if (strategy == GBA_STRATEGY_PARTITION) return gba_run_partition(ctx, qd, out, k, p, pred, s, n_groups);
  return gba_run_table(ctx, qd, out, k, p, s, n_groups);
}
