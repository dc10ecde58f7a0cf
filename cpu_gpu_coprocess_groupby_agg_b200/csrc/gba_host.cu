// Host-resident inputs: the reference's "coprocess" mode.
//
// The reference copies each tile H2D, aggregates it, copies the partitioned
// tile result back over the caller's input buffer and later streams the
// partitions back again (group_then_partition.cu:353-418,
// groupby_agg_intra_partition.cu:208-276): every row crosses PCIe three times.
// Here rows cross once: chunks are copied on a copy stream while the compute
// stream pre-aggregates the previous chunk into one HBM table, and only the
// final groups come back.
#include <algorithm>
#include <cstring>
#include <string>

#include "gba_context.h"
#include "gba_plan.h"
#include "sort_kernels.h"

static int tbytes(int t) { return gba_type_bytes(t); }

extern "C" gba_status gba_groupby_host(gba_context* ctx, const gba_query* q, const gba_output* out,
                                       const gba_knobs* knobs, void* stream, int64_t* n_groups) {
  if (!ctx || !q || !out || !n_groups) return GBA_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  ctx->stats = gba_stats{};
  ctx->stats.predicted_groups = -1;
  gba_knobs k;
  if (knobs) k = *knobs;
  else gba_default_knobs(&k);
  gba_query qc;
  gba_compact_query(q, &qc);
  q = &qc;
  QDesc hq;
  gba_status st = gba_build_qdesc(ctx, q, &hq);
  if (st != GBA_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t n = q->n_rows;
  const int kb = tbytes(q->key.type);

  // staging layout: inputs, then output columns sized to min(capacity, n)
  const int64_t ocap = std::min<int64_t>(out->capacity, std::max<int64_t>(n, 1) + 1);
  size_t off = 0;
  size_t in_off[1 + GBA_MAX_COLS];
  in_off[0] = off;
  off = gba_round_up(off + size_t(n) * kb, 256);
  for (int c = 0; c < q->n_cols; ++c) {
    in_off[1 + c] = off;
    off = gba_round_up(off + size_t(n) * tbytes(q->cols[c].type), 256);
  }
  const size_t out_off = off;
  off = gba_round_up(off + size_t(ocap) * kb, 256);
  size_t acc_off[GBA_MAX_AGGS];
  for (int a = 0; a < q->n_aggs; ++a) {
    acc_off[a] = off;
    off = gba_round_up(off + size_t(ocap) * 8, 256);
  }
  st = gba_stage_reserve(ctx, off, s);
  if (st != GBA_OK) return st;
  unsigned char* base = static_cast<unsigned char*>(ctx->stage);

  QDesc dq = hq;
  dq.keys = base + in_off[0];
  for (int c = 0; c < q->n_cols; ++c) dq.cols[c] = base + in_off[1 + c];
  gba_output dout;
  std::memset(&dout, 0, sizeof(dout));
  dout.keys = base + out_off;
  for (int a = 0; a < q->n_aggs; ++a) dout.aggs[a] = base + acc_off[a];
  dout.capacity = ocap;

  double pred = -1;
  GbaPlan p;
  int strategy = k.strategy;
  const bool learned = k.sizing == GBA_SIZING_LEARNED;
  // Learned sizing and the partition strategy read the whole key column first,
  // so those runs stage everything before planning.
  bool staged = false;
  auto stage_all = [&]() -> gba_status {
    GBA_CUDA_TRY(ctx, cudaMemcpyAsync(const_cast<void*>(dq.keys), q->key.data, size_t(n) * kb,
                                      cudaMemcpyHostToDevice, s));
    for (int c = 0; c < q->n_cols; ++c)
      GBA_CUDA_TRY(ctx, cudaMemcpyAsync(const_cast<void*>(dq.cols[c]), q->cols[c].data,
                                        size_t(n) * tbytes(q->cols[c].type), cudaMemcpyHostToDevice, s));
    staged = true;
    return GBA_OK;
  };
  if (learned) {
    if (!ctx->est_loaded) {
      ctx->err = "learned sizing requested but no estimator weights are loaded";
      return GBA_ERR_INVALID_ARG;
    }
    st = stage_all();
    if (st != GBA_OK) return st;
    st = gba_predict_groups(ctx, dq, s, &pred);
    if (st != GBA_OK) return st;
    ctx->stats.predicted_groups = pred;
  }
  gba_make_plan(ctx, dq, k, pred, &p);
  if (strategy == GBA_STRATEGY_AUTO) strategy = gba_choose_strategy(ctx, dq, k, pred, p);

  int64_t ng = 0;
  if (strategy == GBA_STRATEGY_PARTITION || staged) {
    if (!staged) {
      st = stage_all();
      if (st != GBA_OK) return st;
    }
    st = strategy == GBA_STRATEGY_PARTITION ? gba_run_partition(ctx, dq, &dout, k, p, pred, s, &ng)
                                            : gba_run_table(ctx, dq, &dout, k, p, s, &ng);
  } else {
    // Chunked pipeline: H2D of chunk i+1 overlaps the pre-aggregation of chunk i.
    const int64_t chunk = std::max<int64_t>(int64_t(p.tile_rows), int64_t(1) << 23) / p.tile_rows * p.tile_rows;
    const size_t stride = size_t(gba_gt_stride(dq.naccs));
    const size_t table_bytes = (p.table_slots + 1) * stride * 8;
    st = gba_ws_reserve(ctx, table_bytes, s);
    if (st != GBA_OK) return st;
    unsigned* d_flags = reinterpret_cast<unsigned*>(ctx->d_small);
    unsigned long long* d_count = reinterpret_cast<unsigned long long*>(ctx->d_small + 8);
    GBA_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_small, 0, 64, s));
    GTable t;
    t.base = static_cast<unsigned long long*>(ctx->ws);
    t.cap = p.table_slots;
    t.probe_cap = p.probe_cap;
    const int init_grid = int(std::min<uint64_t>(uint64_t(ctx->sms) * 16, (table_bytes / 8 + 255) / 256 + 1));
    GBA_CUDA_TRY(ctx, gba_launch_table_init(t, dq, init_grid, s));
    // the copy stream must not overwrite staging still read by an earlier call
    GBA_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[7], s));
    GBA_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->ev[7], 0));
    int launches = 1;
    int64_t i = 0;
    for (int64_t r0 = 0; r0 < n; r0 += chunk, ++i) {
      const int64_t rows = std::min(chunk, n - r0);
      GBA_CUDA_TRY(ctx, cudaMemcpyAsync(static_cast<unsigned char*>(const_cast<void*>(dq.keys)) + r0 * kb,
                                        static_cast<const unsigned char*>(q->key.data) + r0 * kb, size_t(rows) * kb,
                                        cudaMemcpyHostToDevice, ctx->copy_stream));
      for (int c = 0; c < q->n_cols; ++c) {
        const int cb = tbytes(q->cols[c].type);
        GBA_CUDA_TRY(ctx, cudaMemcpyAsync(static_cast<unsigned char*>(const_cast<void*>(dq.cols[c])) + r0 * cb,
                                          static_cast<const unsigned char*>(q->cols[c].data) + r0 * cb,
                                          size_t(rows) * cb, cudaMemcpyHostToDevice, ctx->copy_stream));
      }
      cudaEvent_t e = ctx->ev[i % 6];
      GBA_CUDA_TRY(ctx, cudaEventRecord(e, ctx->copy_stream));
      GBA_CUDA_TRY(ctx, cudaStreamWaitEvent(s, e, 0));
      QDesc cq = dq;
      cq.n = rows;
      cq.keys = static_cast<const unsigned char*>(dq.keys) + r0 * kb;
      for (int c = 0; c < q->n_cols; ++c)
        cq.cols[c] = static_cast<const unsigned char*>(dq.cols[c]) + r0 * tbytes(q->cols[c].type);
      GbaPlan cp = p;
      const int64_t ntiles = (rows + p.tile_rows - 1) / p.tile_rows;
      cp.grid = int(std::max<int64_t>(1, std::min<int64_t>(ntiles, p.grid)));
      PreaggCfg c;
      c.grid = cp.grid;
      c.block = cp.block;
      c.smem_slots = cp.smem_slots;
      c.smem_probe_cap = cp.smem_probe_cap;
      c.tile_rows = cp.tile_rows;
      c.nstages = cp.nstages;
      c.use_tma = cp.use_tma && rows >= cp.tile_rows;
      c.coalesce = cp.coalesce;
      GBA_CUDA_TRY(ctx, gba_launch_preagg(cq, t, c, d_flags, s));
      ++launches;
      ctx->stats.main_rows += cq.n;
      ctx->stats.main_bytes += cq.n * int64_t(gba_row_bytes(cq));
    }
    OutDesc o;
    o.keys = dout.keys;
    for (int a = 0; a < GBA_MAX_AGGS; ++a) o.accs[a] = static_cast<unsigned long long*>(dout.aggs[a]);
    o.capacity = dout.capacity;
    o.count = d_count;
    const int cgrid = int(std::min<uint64_t>(uint64_t(ctx->sms) * 8, (p.table_slots + 255) / 256));
    GBA_CUDA_TRY(ctx, gba_launch_compact(t, dq, o, std::max(cgrid, 1), s));
    ++launches;
    GBA_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_small, ctx->d_small, 16, cudaMemcpyDeviceToHost, s));
    GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    const unsigned flags = *reinterpret_cast<unsigned*>(ctx->h_small);
    const unsigned long long count = *reinterpret_cast<unsigned long long*>(ctx->h_small + 8);
    ctx->stats.kernel_launches += launches;
    ctx->stats.strategy = GBA_STRATEGY_TABLE;
    ctx->stats.table_slots = int64_t(p.table_slots);
    ctx->stats.preagg = p.smem_slots > 0;
    if (flags & GBA_FLAG_WAIT_TIMEOUT) {
      ctx->err = "a bounded TMA wait timed out";
      return GBA_ERR_TIMEOUT;
    }
    if (flags & GBA_FLAG_TABLE_OVERFLOW) {
      // all rows are resident now: finish with the device path and regrow
      GbaPlan rp = p;
      rp.table_slots *= 4;
      ctx->stats.regrows++;
      st = gba_run_table(ctx, dq, &dout, k, rp, s, &ng);
    } else {
      ng = int64_t(count);
      ctx->stats.n_groups = ng;
      st = ng > dout.capacity ? GBA_ERR_OUTPUT_CAPACITY : GBA_OK;
    }
  }
  *n_groups = ng;
  if (st == GBA_OK && ng > out->capacity) st = GBA_ERR_OUTPUT_CAPACITY;
  if (st != GBA_OK) {
    if (st == GBA_ERR_OUTPUT_CAPACITY)
      ctx->err = "output capacity " + std::to_string(out->capacity) + " < " + std::to_string(ng) + " groups";
    return st;
  }
  if (k.sort_output && ng > 1) {
    const SortJob j = gba_sort_job(q, &dout, ng);
    st = gba_sort_groups(ctx, &j, 1, s);
    if (st != GBA_OK) return st;
  }
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(out->keys, dout.keys, size_t(ng) * kb, cudaMemcpyDeviceToHost, s));
  for (int a = 0; a < q->n_aggs; ++a)
    GBA_CUDA_TRY(ctx, cudaMemcpyAsync(out->aggs[a], dout.aggs[a], size_t(ng) * 8, cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return GBA_OK;
}
