// gba_groupby_batch: many independent device queries in a few launches.
//
// Every query is planned as gba_groupby would plan it (learned sizing runs the
// estimator once for the whole batch).  Queries on the table strategy share
// one launch sequence:
//   k_batch_init      every query's HBM table (blocks dealt by table size)
//   k_stream_agg      one persistent launch per aggregate signature and key
//                     width; CTAs pop (query, row range) items from a device
//                     work queue, query by query, largest queries first
//   k_batch_compact   every query's groups into its own output
// replayed from a CUDA graph while the batch's launch shapes repeat (the
// per-query descriptors are copied from pinned host memory by the graph's
// first node, so new queries of the same shapes reuse it).  Queries on the
// partition strategy run one after another behind it.  A query whose table
// overflowed is rerun alone with a larger table.
//
// No counterpart in the reference: its host loop runs one query, one tile per
// stream at a time (group_then_partition.cu:332-424).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "batch_kernels.h"
#include "est_kernels.h"
#include "gba_context.h"
#include "gba_plan.h"
#include "composite.h"
#include "nulls.h"
#include "sort_kernels.h"

namespace {

// GBA_TRACE=1 in the environment: host-side phase times of each batch call on
// stderr (where a step's time goes between the kernels).
struct PhaseTrace {
  bool on = std::getenv("GBA_TRACE") != nullptr;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now(), last = t0;
  std::string line;
  void mark(const char* what) {
    if (!on) return;
    const auto now = std::chrono::steady_clock::now();
    char buf[96];
    std::snprintf(buf, sizeof(buf), " %s=%.3fms", what, std::chrono::duration<double, std::milli>(now - last).count());
    line += buf;
    last = now;
  }
  ~PhaseTrace() {
    if (on) std::fprintf(stderr, "gba_groupby_batch:%s total=%.3fms\n", line.c_str(),
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
  }
};

struct QInfo {
  QDesc q;
  GbaPlan p;
  double pred = -1;
  int strategy = GBA_STRATEGY_TABLE;
  int S = 0;         // shared-table slots in the batch kernel (per CTA)
  int cl = 1;        // CTAs of the cluster whose tables form the query's shared table
  bool tma = false;  // streamed by the bulk-copy kernel (else the register-loading one)
  bool xch = false;  // aggregated by the owner-exchange kernel
  int hot = 0;       // exchange: hot-table slots per CTA
  int slot = -1;     // index among the table-strategy queries
};

struct Group {
  int sig;
  QDesc proto;
  std::vector<int> members;  // indices into the batch's queries
  size_t smem = 0;           // dynamic shared memory of the group's launch
  size_t stage_bytes = 0;    // bulk-copy kernel: bytes of one ring slot
  int cluster = 1;           // bulk-copy kernel: CTAs per cluster
  int minb = 1;              // CTAs per SM of the launch
  int shape = 1;             // bulk-copy kernel: its CTA shape (1 or 2 CTAs of 512 threads per SM, 0: one of 1024)
  bool tma = false;          // bulk-copy kernel (k_stream_tma) or register-loading one (k_stream_agg)
  bool hbm = false;          // register-loading kernel, queries without a shared table only
  int64_t item_begin = 0, nitems = 0;  // item_begin: index of the group's first span
  int entry_begin = 0, entry_end = 0;   // its table entries
  int nspans = 0;
  int grid = 0;
};

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Estimator predictions for every query of the batch: one sampling pass, one
// MLP launch, one copy back.
gba_status batch_predict(gba_context* ctx, const std::vector<QDesc>& qs, cudaStream_t s, std::vector<double>* pred,
                         std::vector<double>* skew) {
  const int n = int(qs.size());
  float* f;
  unsigned long long* stats;
  gba_status st = gba_est_features_device(ctx, qs.data(), n, 0, s, &f, &stats);
  if (st != GBA_OK) return st;
  const size_t y_off = 4096, s_off = round_up(y_off + 4 * size_t(n), 256);
  st = gba_small_reserve(ctx, std::max<size_t>(ctx->d_small_bytes, s_off + 32 * size_t(n)));
  if (st != GBA_OK) return st;
  float* y = reinterpret_cast<float*>(ctx->d_small + y_off);
  GBA_CUDA_TRY(ctx, gba_launch_mlp_forward(ctx->d_est, f, n, y, s));
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_small + y_off, y, 4 * size_t(n), cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_small + s_off, stats, 32 * size_t(n), cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  ctx->stats.kernel_launches += 1;
  const float* yh = reinterpret_cast<const float*>(ctx->h_small + y_off);
  const unsigned long long* sh = reinterpret_cast<const unsigned long long*>(ctx->h_small + s_off);
  pred->resize(n);
  skew->resize(n);
  for (int i = 0; i < n; ++i) {
    double g = exp2(double(yh[i]) * 32.0);
    g = std::max(g, double(sh[4 * i + 0]));
    g = std::min(g, double(std::max<int64_t>(qs[i].n, 1)));
    (*pred)[i] = g;
    (*skew)[i] = double(sh[4 * i + 1]) / double(std::max<unsigned long long>(1, sh[4 * i + 2]));
  }
  return GBA_OK;
}

// Shared-table slots a streaming CTA can hold for a query (the kernel's
// dynamic shared memory is the table alone) with `bps` CTAs per SM.
int batch_smem_slots(const gba_context* ctx, const QDesc& q, int bps) {
  // (the SM's shared memory, 1 KB more than one CTA may opt into, is split
  // between the CTAs, each losing 1 KB to the system)
  const size_t budget = (size_t(ctx->max_smem_optin) + 1024) / size_t(bps) - 1024;
  const size_t fixed = gba_stream_smem_bytes(q, 0) + gba_batch_static_smem() + 1024;
  if (budget <= fixed) return 0;
  const size_t slot = (q.key64 ? 8 : 4) + 4 * size_t(q.nwords);
  const int S = int(std::min<size_t>(16384, (budget - fixed) / slot));
  return S < 32 ? 0 : S;
}

// Shared-table slots of a query in the bulk-copy streaming kernel of CTA
// shape `shape` (1 or 2 CTAs of 512 threads per SM, 0: one of 1024 threads):
// what a CTA's share of the SM's shared memory holds beside its warps' copy
// rings (`nst` slots of `slot_bytes` each) and its static part (barriers,
// chunk starts: 2 KB at most for 16 warps, 4 KB for 32).
int tma_smem_slots(const gba_context* ctx, const QDesc& q, int shape, int nst, size_t slot_bytes) {
  const size_t budget = (size_t(ctx->max_smem_optin) + 1024) / size_t(shape == 2 ? 2 : 1) - 1024;
  const size_t fixed =
      gba_stream_tma_smem_bytes(q, 0, nst, slot_bytes, shape) + gba_batch_static_smem() + (shape == 0 ? 4096 : 2048);
  if (budget <= fixed) return 0;
  const size_t slot = (q.key64 ? 8 : 4) + 4 * size_t(q.nwords);
  const int S = int(std::min<size_t>(16384, (budget - fixed) / slot));
  return S < 32 ? 0 : S;
}

// Shared-table slots per CTA of the owner-exchange kernel (one CTA per SM;
// the table is the CTA's whole dynamic shared memory).
int exchange_smem_slots(const gba_context* ctx, const QDesc& q, int hot) {
  const size_t budget = size_t(ctx->max_smem_optin);
  const size_t fixed = gba_exchange_smem_bytes(q, 0, hot) + gba_exchange_static_smem() + 1024;
  if (budget <= fixed) return 0;
  const size_t slot = (q.key64 ? 8 : 4) + 4 * size_t(q.nwords);
  return int(std::min<size_t>(65536, (budget - fixed) / slot)) / 4 * 4;
}

// Owner-exchange launch of one aggregate signature and key width.
struct XGroup {
  QDesc proto;
  std::vector<int> members;
  size_t smem = 0;
  int64_t xq_off = 0;  // first entry of the group in the device list of query slots
};

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

static gba_status batch_device(gba_context* ctx, int32_t nq, const gba_query* qs, const gba_output* outs,
                               const gba_knobs* knobs, void* stream, int64_t* n_groups);
static gba_status batch_avg(gba_context* ctx, int32_t nq, const gba_query* qs, const gba_output* outs,
                            const gba_knobs* knobs, void* stream, int64_t* n_groups);

// Composite keys are packed into 64-bit keys around the batch; key order
// (knobs->sort_output) sorts every query's groups on the device after it, one
// query after another.
extern "C" gba_status gba_groupby_batch(gba_context* ctx, int32_t nq, const gba_query* qs, const gba_output* outs,
                                        const gba_knobs* knobs, void* stream, int64_t* n_groups) {
  if (!ctx || nq < 0 || (nq > 0 && (!qs || !outs || !n_groups))) return GBA_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // nullable columns: rewritten columns and aggregates (qn, on)
  bool nulls = false;
  for (int i = 0; i < nq && !nulls; ++i) nulls = gba_nulls_needed(qs[i], outs[i]);
  std::vector<gba_query> qn;
  std::vector<gba_output> on;
  std::vector<NullPlan> np;
  if (nulls) {
    GBA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    qn.assign(qs, qs + nq);
    on.assign(outs, outs + nq);
    gba_status st = gba_nulls_prepare(ctx, nq, qs, outs, qn.data(), on.data(), &np, s);
    if (st != GBA_OK) return st;
  }
  const gba_query* qb = nulls ? qn.data() : qs;
  const gba_output* ob = nulls ? on.data() : outs;
  // composite keys: packed key columns
  bool composite = false;
  for (int i = 0; i < nq && !composite; ++i) composite = qb[i].key2.data != nullptr;
  std::vector<gba_query> q2;
  std::vector<gba_output> o2;
  std::vector<CompositeJob> cj;
  if (composite) {
    GBA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    q2.assign(qb, qb + nq);
    o2.assign(ob, ob + nq);
    gba_status st = gba_composite_prepare(ctx, nq, qb, ob, q2.data(), o2.data(), &cj, s);
    if (st != GBA_OK) return st;
  }
  const gba_query* qa = composite ? q2.data() : qb;
  const gba_output* oa = composite ? o2.data() : ob;
  gba_status st = batch_avg(ctx, nq, qa, oa, knobs, stream, n_groups);
  if (st != GBA_OK) return st;
  if (knobs && knobs->sort_output) {
    std::vector<SortJob> jobs(nq);
    for (int i = 0; i < nq; ++i) {
      jobs[i] = gba_sort_job(&qa[i], &oa[i], std::min<int64_t>(n_groups[i], oa[i].capacity));
      if (qs[i].key2.data) jobs[i].key_signed = 0;  // the packed pair orders as an unsigned word
    }
    st = gba_sort_groups(ctx, jobs.data(), nq, s);
    if (st != GBA_OK) return st;
  }
  if (!cj.empty()) {
    st = gba_composite_finish(ctx, cj, ob, n_groups, s);
    if (st != GBA_OK) return st;
  }
  if (!np.empty()) return gba_nulls_finish(ctx, np, qs, outs, ob, n_groups, s);
  return GBA_OK;
}

// AVG, as in gba_groupby: every AVG runs as a SUM into the caller's column,
// each query with an AVG gets one COUNT (its own, or one added into a slice of
// a context buffer), and after the batch one kernel per such query turns its
// SUM columns into SUM / COUNT in place.
static gba_status batch_avg(gba_context* ctx, int32_t nq, const gba_query* qs, const gba_output* outs,
                            const gba_knobs* knobs, void* stream, int64_t* n_groups) {
  if (!ctx || nq < 0 || (nq > 0 && (!qs || !outs || !n_groups))) return GBA_ERR_INVALID_ARG;
  bool any = false;
  for (int i = 0; i < nq && !any; ++i)
    for (int a = 0; a < qs[i].n_aggs && a < GBA_MAX_AGGS; ++a) any = any || qs[i].aggs[a].op == GBA_AVG;
  if (!any) return batch_device(ctx, nq, qs, outs, knobs, stream, n_groups);
  GBA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  std::vector<gba_query> q2(qs, qs + nq);
  std::vector<gba_output> o2(outs, outs + nq);
  std::vector<AvgDesc> fin(nq);
  std::vector<int> cnt(nq, -1);
  std::vector<size_t> scratch_off(nq, SIZE_MAX);  // SIZE_MAX: the query's own COUNT
  size_t scratch = 0;
  for (int i = 0; i < nq; ++i) {
    fin[i] = AvgDesc{};
    for (int a = 0; a < qs[i].n_aggs && a < GBA_MAX_AGGS; ++a) {
      if (qs[i].aggs[a].op == GBA_COUNT && cnt[i] < 0) cnt[i] = a;
      if (qs[i].aggs[a].op != GBA_AVG) continue;
      const int c = qs[i].aggs[a].col;
      if (c < 0 || c >= qs[i].n_cols) {
        ctx->err = "query " + std::to_string(i) + ": aggregate column index out of range";
        return GBA_ERR_INVALID_ARG;
      }
      q2[i].aggs[a].op = GBA_SUM;
      fin[i].col[fin[i].n] = static_cast<unsigned long long*>(outs[i].aggs[a]);
      fin[i].fp[fin[i].n] = qs[i].cols[c].type == GBA_F32 || qs[i].cols[c].type == GBA_F64;
      ++fin[i].n;
    }
    if (fin[i].n > 0 && cnt[i] < 0) {
      if (q2[i].n_aggs >= GBA_MAX_AGGS) {
        ctx->err = "query " + std::to_string(i) + ": AVG needs a COUNT: at most 7 aggregates with AVG and no COUNT";
        return GBA_ERR_INVALID_ARG;
      }
      scratch_off[i] = scratch;
      scratch += size_t(std::max<int64_t>(outs[i].capacity, 1)) * 8;
      cnt[i] = q2[i].n_aggs++;
      q2[i].aggs[cnt[i]].op = GBA_COUNT;
      q2[i].aggs[cnt[i]].col = 0;
    }
  }
  if (scratch > ctx->avg_bytes) {
    if (ctx->avg_buf) {
      GBA_CUDA_TRY(ctx, cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
      cudaFree(ctx->avg_buf);
      ctx->avg_buf = nullptr;
      ctx->avg_bytes = 0;
    }
    GBA_CUDA_TRY(ctx, cudaMalloc(&ctx->avg_buf, scratch));
    ctx->avg_bytes = scratch;
  }
  for (int i = 0; i < nq; ++i) {
    if (fin[i].n == 0) continue;
    if (scratch_off[i] != SIZE_MAX)
      o2[i].aggs[cnt[i]] = static_cast<unsigned char*>(ctx->avg_buf) + scratch_off[i];
    fin[i].count = static_cast<const unsigned long long*>(o2[i].aggs[cnt[i]]);
  }
  gba_status st = batch_device(ctx, nq, q2.data(), o2.data(), knobs, stream, n_groups);
  if (st != GBA_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int launches = 0;
  for (int i = 0; i < nq; ++i) {
    const int64_t g = std::min<int64_t>(n_groups[i], outs[i].capacity);
    if (fin[i].n == 0 || g <= 0) continue;
    GBA_CUDA_TRY(ctx, gba_launch_avg_finish(fin[i], g, ctx->sms, s));
    ++launches;
  }
  if (launches) GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  ctx->stats.kernel_launches += launches;
  return GBA_OK;
}

static gba_status batch_device(gba_context* ctx, int32_t nq, const gba_query* qs, const gba_output* outs,
                               const gba_knobs* knobs, void* stream, int64_t* n_groups) {
  if (!ctx || nq < 0 || (nq > 0 && (!qs || !outs || !n_groups))) return GBA_ERR_INVALID_ARG;
  GBA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  ctx->stats = gba_stats{};
  ctx->stats.predicted_groups = -1;
  if (nq == 0) return GBA_OK;
  gba_knobs k;
  if (knobs) k = *knobs;
  else gba_default_knobs(&k);
  // A batch's learned-sized tables default to load 0.25 (a single query's to
  // 0.35): measured on the 256-query batch, 9.92 against 10.00 ms a step
  // (the autotuner's usual pick there too)
  if (!(k.learned_load > 0.05 && k.learned_load < 0.95)) k.learned_load = 0.25;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PhaseTrace trace;

  // ---- validate and describe every query ----
  std::vector<QInfo> qi(nq);
  std::vector<QDesc> qd(nq);
  for (int i = 0; i < nq; ++i) {
    gba_query qc;
    gba_compact_query(&qs[i], &qc);
    gba_status st = gba_build_qdesc(ctx, &qc, &qd[i]);
    if (st != GBA_OK) {
      ctx->err = "query " + std::to_string(i) + ": " + ctx->err;
      return st;
    }
    const gba_output& o = outs[i];
    bool bad = o.capacity < 0 || (o.capacity > 0 && !o.keys);
    for (int a = 0; a < qc.n_aggs; ++a) bad = bad || (o.capacity > 0 && !o.aggs[a]);
    if (bad) {
      ctx->err = "query " + std::to_string(i) + ": bad output descriptor";
      return GBA_ERR_INVALID_ARG;
    }
    qi[i].q = qd[i];
    n_groups[i] = 0;
  }

  // ---- sizing: one estimator pass for the batch ----
  std::vector<double> pred(nq, -1.0), skew(nq, 0.0);
  if (k.sizing == GBA_SIZING_LEARNED) {
    if (!ctx->est_loaded) {
      ctx->err = "learned sizing requested but no estimator weights are loaded";
      return GBA_ERR_INVALID_ARG;
    }
    trace.mark("validate");
    gba_status st = batch_predict(ctx, qd, s, &pred, &skew);
    if (st != GBA_OK) return st;
    trace.mark("estimate");
    ctx->stats.predicted_groups = std::accumulate(pred.begin(), pred.end(), 0.0);
  }
  // work items are cut at multiples of T rows (vector loads need aligned starts)
  const int T = 2048;
  // CTAs per SM of the streaming kernel (1 to 4; automatic: 3).  More CTAs
  // split each SM's shared memory and registers into smaller tables and fewer
  // rows per lane, but keep more warps and L2 requests in flight: measured on
  // the 256-query batch, the kernel takes 16.4 ms at 1, 11.1-12.3 ms at 2 and
  // 10.3 ms at 4 (where registers spill); 3 (40 registers, few spills) is 1-2%
  // faster than 4 and is what the autotuner picks there.
  // Two streaming kernels: the register-loading one (k_stream_agg, bps CTAs
  // per SM, automatic 3) and the bulk-copy one (k_stream_tma: 1 or 2 CTAs of
  // 512 threads per SM, automatic 2, or one of 1024 threads, each warp staging
  // its rows through a ring of `nst` slots).  knobs.use_tma = 0 / 1 sends every query to one of them;
  // automatic (-1): a query whose predicted groups outgrow half the
  // register-loading kernel's shared table goes to the bulk-copy kernel, the
  // rest (and every query under plain sizing) to the register-loading one.
  // Measured per cardinality class of the 256-query batch (kernel ms,
  // register-loading vs bulk-copy): ids < 256: 0.69 vs 0.89; 256-4096: 1.47 vs
  // 1.53; 4096-16384: 1.60 vs 1.40; 16384-65536: 2.60 vs 2.36; 65536-262144:
  // 1.32 vs 1.04; 262144-2^20: 2.35 vs 2.25; above 2^20: 2.94 vs 2.65.
  // ring slots per warp (automatic 2: measured 10.04-10.07 ms a step against
  // 10.16-10.22 with 3, whose larger rings leave less shared memory to the
  // tables of the 1024-thread CTAs)
  const int nst = k.nstages >= 1 && k.nstages <= 4 ? k.nstages : 2;
  const int bps = k.blocks_per_sm >= 1 && k.blocks_per_sm <= 4 ? k.blocks_per_sm : 3;
  // bulk-copy kernel CTA shape: one CTA of 1024 threads per SM (automatic;
  // one shared table of twice the slots for as many warps as two 512-thread
  // CTAs), or CTAs of 512 threads (knobs.block_threads = 512, or
  // blocks_per_sm 1 or 2: that many per SM, 2 by default).  Measured per
  // class of the 256-query batch (kernel ms, 512 x 2 against 1024 x 1): 0.92
  // against 0.85 on 65536-262143 ids, 1.93 against 1.81 on 262144-2^20, the
  // others within 1%.
  const int tshape = k.block_threads == 1024                                                   ? 0
                     : k.block_threads == 512 || k.blocks_per_sm == 1 || k.blocks_per_sm == 2 ? (k.blocks_per_sm == 1 ? 1 : 2)
                                                                                              : 0;
  bool any_tma = false;
  // buckets probed in a shared table before a row goes to the HBM table
  // (automatic 4: 9.87 against 9.92 ms a step with 2, at load 0.25)
  const int sprobe = k.smem_probe_cap > 0 ? k.smem_probe_cap : 4;
  // Strategy: a query alone leaves the HBM-table strategy once its table
  // outgrows L2 (gba_choose_strategy), but in a batch such a query still runs
  // inside the shared persistent launch, while a partition-strategy query runs
  // alone after it.  Measured on the 256-query batch: routing its two queries
  // with tables above L2 (the larger about 1 GB) through the batch kernel made
  // the step 1.4% faster.  Only tables above 2 GB leave the batch.
  constexpr double kBatchTableMax = double(int64_t(2) << 30);
  for (int i = 0; i < nq; ++i) {
    ctx->est_skew = skew[i];
    gba_make_plan(ctx, qd[i], k, pred[i], &qi[i].p);
    qi[i].pred = pred[i];
    double table_bytes = double(qi[i].p.table_slots + 1) * 8.0 * double(gba_gt_stride(qd[i].naccs));
    // A learned-sized table above 32 MB is sized at load 0.5: half the
    // footprint to clear, compact and keep in L2, at the cost of longer probes
    // (an under-estimate still regrows).
    if (k.sizing == GBA_SIZING_LEARNED && pred[i] > 0 && table_bytes > 32.0 * double(1 << 20)) {
      const double g = std::min(double(std::max<int64_t>(qd[i].n, 1)), pred[i] * 1.25 + 64.0);
      const uint64_t at_half = uint64_t(g / 0.5) + 1;
      if (at_half < qi[i].p.table_slots) qi[i].p.table_slots = at_half;
      table_bytes = double(qi[i].p.table_slots + 1) * 8.0 * double(gba_gt_stride(qd[i].naccs));
    }
    qi[i].strategy = k.strategy != GBA_STRATEGY_AUTO ? k.strategy
                     : table_bytes <= kBatchTableMax ? GBA_STRATEGY_TABLE
                                                     : gba_choose_strategy(ctx, qd[i], k, pred[i], qi[i].p);
  }

  // ---- owner exchange ----
  // A query whose predicted groups outgrow one streaming CTA's shared table
  // but fit 0.6 of the exchange kernel's tables over all SMs goes to the
  // owner-exchange kernel (learned sizing, at least 2^19 rows).  A query whose
  // sample shows a key taking 1/256 of the rows (or any query without an
  // estimate) also gets hot tables of 1024 slots, so its hottest keys are
  // aggregated where they are read instead of loading their owners.  Its HBM
  // table only takes keys whose shared probe window is full, so it is sized
  // small (an overflow reruns the query alone with a larger table).
  int xgrid = ctx->sms;
  for (int i = 0; i < nq; ++i) {
    if (qi[i].strategy != GBA_STRATEGY_TABLE || k.exchange == 0 || qd[i].n <= 0) continue;
    const int hot = (qi[i].pred <= 0 || skew[i] >= 1.0 / 256.0) ? 1024 : 0;
    const int Sx = exchange_smem_slots(ctx, qd[i], hot);
    if (Sx < 256) continue;
    if (k.exchange == 1) qi[i].xch = true;
    else
      qi[i].xch = k.sizing == GBA_SIZING_LEARNED && qi[i].pred > 0 && qi[i].p.preagg && qd[i].n >= (int64_t(1) << 19) &&
                  qi[i].pred > 0.5 * batch_smem_slots(ctx, qd[i], bps) && qi[i].pred <= 0.6 * double(xgrid) * Sx;
    if (qi[i].xch) {
      qi[i].S = Sx;
      qi[i].hot = hot;
      if (qi[i].pred > 0) {
        const uint64_t small = std::max<uint64_t>(uint64_t(1) << 16, uint64_t(qi[i].pred * 0.5) + 1);
        qi[i].p.table_slots = std::min<uint64_t>(qi[i].p.table_slots, small);
      }
    }
  }

  // ---- streaming kernel of each query ----
  for (int i = 0; i < nq; ++i) {
    if (qi[i].strategy != GBA_STRATEGY_TABLE || qi[i].xch) continue;
    if (k.use_tma == 0) qi[i].tma = false;
    else if (k.use_tma == 1) qi[i].tma = true;
    else qi[i].tma = qi[i].pred > 0 && qi[i].p.preagg && qi[i].pred > 0.5 * batch_smem_slots(ctx, qd[i], bps);
    any_tma = any_tma || qi[i].tma;
  }

  // ---- cluster tables ----
  // With knobs.cluster_ctas = c (2, 4, 8 or 16), a bulk-copy query whose
  // predicted groups outgrow one CTA's shared table (more than half its slots)
  // but fit the tables of a cluster of up to c CTAs at load 0.7 gets such a
  // cluster (the smallest that fits): its rows then meet a shared-memory
  // table spread over the cluster instead of the HBM table.  Learned sizing
  // only (the group count is needed); integer SUM/COUNT signatures only.  Off
  // by default: measured on the batch, the remote shared-memory atomics cost
  // more than the L2 traffic they save (4096-16384 ids: 1.58 ms without
  // clusters, 2.07 with 2 CTAs, 3.18 with 16).
  const int maxcl = k.cluster_ctas >= 2 && k.cluster_ctas <= 16 ? k.cluster_ctas : 1;
  for (int i = 0; i < nq && maxcl > 1; ++i) {
    if (qi[i].strategy != GBA_STRATEGY_TABLE || !qi[i].tma || !qi[i].p.preagg || qi[i].pred <= 0 ||
        k.smem_slots > 0 || !gba_stream_tma_cluster_ok(qd[i]))
      continue;
    const double S1 = tma_smem_slots(ctx, qd[i], 1, nst, gba_stream_tma_slot_bytes(qd[i], 1));
    if (S1 <= 0 || qi[i].pred <= 0.5 * S1) continue;
    for (int c = 2; c <= maxcl; c *= 2)
      if (qi[i].pred <= 0.7 * c * S1) {
        qi[i].cl = c;
        break;
      }
  }

  // ---- group the table-strategy queries by aggregate signature (and cluster) ----
  constexpr bool kHbmLaunch = true;
  // CTAs per SM of that launch: measured 10.09 ms a step at 3 (40 registers,
  // 2 rows per lane) against 10.20 at 2 (4 rows per lane, no spills)
  constexpr int kHbmCtas = 3;
  std::vector<Group> groups;
  std::vector<int> tq;  // table-strategy queries, group by group
  for (int i = 0; i < nq; ++i) {
    if (qi[i].strategy != GBA_STRATEGY_TABLE || qi[i].xch) continue;
    // one launch per signature, key width, kernel and cluster size
    // register-loading queries without a shared table get a launch of their
    // own, on the kernel built without table code (measured on the batch:
    // 10.20 against 11.04 ms a step in one call)
    const bool hbm = kHbmLaunch && !qi[i].tma && !qi[i].p.preagg;
    const int sig =
        (((2 * gba_batch_sig_id(qd[i]) + (qd[i].key64 ? 1 : 0)) * 2 + (qi[i].tma ? 1 : 0)) * 2 + (hbm ? 1 : 0)) * 32 +
        qi[i].cl;
    auto it = std::find_if(groups.begin(), groups.end(), [&](const Group& g) { return g.sig == sig; });
    if (it == groups.end()) {
      groups.push_back(Group{sig, qd[i], {}});
      groups.back().cluster = qi[i].cl;
      groups.back().tma = qi[i].tma;
      groups.back().hbm = hbm;
      it = groups.end() - 1;
    }
    it->members.push_back(i);
  }
  for (auto& g : groups) {
    g.smem = gba_stream_smem_bytes(g.proto, 0);
    g.shape = g.cluster > 1 ? 1 : tshape;
    // (the launch of queries without a shared table: kHbmCtas CTAs per SM
    // unless blocks_per_sm is set)
    g.minb = !g.tma ? (g.hbm && k.blocks_per_sm <= 0 ? kHbmCtas : bps) : (g.shape == 2 ? 2 : 1);
    if (g.tma) {
      // one ring slot holds a chunk of any member (run-time signatures may
      // differ in columns per member)
      for (int i : g.members) g.stage_bytes = std::max(g.stage_bytes, gba_stream_tma_slot_bytes(qd[i], g.shape));
      g.smem = gba_stream_tma_smem_bytes(g.proto, 0, nst, g.stage_bytes, g.shape);
    }
    g.entry_begin = int(tq.size());
    for (int i : g.members) {
      // run-time signatures may differ in accumulator words per member
      int S = !qi[i].p.preagg ? 0
              : g.tma         ? tma_smem_slots(ctx, qd[i], g.shape, nst, g.stage_bytes)
                              : batch_smem_slots(ctx, qd[i], bps);
      if (k.smem_slots > 0) S = std::min(S, k.smem_slots);
      // a known-small group count needs only a small shared table (cheaper
      // to clear and flush per work item)
      // (4 slots per expected group keep nearly every key in its home bucket)
      if (S > 0 && qi[i].pred > 0) S = std::min<int64_t>(S, std::max<int64_t>(256, int64_t(qi[i].pred * 4.0 + 31) / 32 * 32));
      S = S / 4 * 4;  // whole 16-byte buckets
      qi[i].S = S;
      g.smem = std::max(g.smem, g.tma ? gba_stream_tma_smem_bytes(qd[i], S, nst, g.stage_bytes, g.shape)
                                           : gba_stream_smem_bytes(qd[i], S));
      qi[i].slot = int(tq.size());
      tq.push_back(i);
    }
    g.entry_end = int(tq.size());
    // a cluster launch fills as many clusters as can be resident at once;
    // where none can, its queries run as single CTAs (smaller tables, same
    // results)
    g.grid = ctx->sms * g.minb;
    if (g.cluster > 1) {
      GBA_CUDA_TRY(ctx, gba_prepare_stream_tma(g.proto, g.cluster, 1));
      const int cg = gba_stream_tma_cluster_grid(g.proto, g.cluster, g.smem, ctx->sms);
      if (cg >= g.cluster) g.grid = cg;
      else {
        g.cluster = 1;
        for (int i : g.members) qi[i].cl = 1;
      }
    }
  }
  // exchange launches: one per signature and key width, queries largest first
  const int x_entry_begin = int(tq.size());
  std::vector<XGroup> xgroups;
  int64_t xwin = 0, xstride = 1;
  int xhot = 0;
  for (int i = 0; i < nq; ++i) {
    if (!qi[i].xch) continue;
    const int sig = 2 * gba_batch_sig_id(qd[i]) + (qd[i].key64 ? 1 : 0);
    auto it = std::find_if(xgroups.begin(), xgroups.end(), [&](const XGroup& g) {
      return 2 * gba_batch_sig_id(g.proto) + (g.proto.key64 ? 1 : 0) == sig;
    });
    if (it == xgroups.end()) {
      xgroups.push_back(XGroup{qd[i], {}});
      it = xgroups.end() - 1;
    }
    it->members.push_back(i);
    it->smem = std::max(it->smem, gba_exchange_smem_bytes(qd[i], qi[i].S, qi[i].hot));
    qi[i].slot = int(tq.size());
    tq.push_back(i);
    xwin = std::max<int64_t>(xwin, qd[i].n);
    xstride = std::max<int64_t>(xstride, 1 + qd[i].ncols);
    if (qi[i].hot) {  // hot tables leave as partial records of 1 + naccs words
      xstride = std::max<int64_t>(xstride, 1 + qd[i].naccs);
      xhot = std::max(xhot, qi[i].hot);
    }
  }
  for (auto& g : xgroups) {
    std::stable_sort(g.members.begin(), g.members.end(), [&](int a, int b) { return qd[a].n > qd[b].n; });
    GBA_CUDA_TRY(ctx, gba_prepare_exchange(g.proto));
    const int gg = gba_exchange_grid(g.proto, g.smem, ctx->sms);
    if (gg < 1) {
      ctx->err = "owner-exchange kernel: no CTA fits an SM";
      return GBA_ERR_CUDA;
    }
    xgrid = std::min(xgrid, gg);
  }
  // rows per window: 2^20 (two buffers of 2^20 records of 16 bytes stay in
  // L2); an owner's region also holds the partial records of every CTA's hot
  // table
  xwin = std::min<int64_t>(xwin, int64_t(1) << 20);
  const int64_t xregion = std::max<int64_t>(xwin, int64_t(xgrid) * (xhot + 1));
  const int nt = int(tq.size());

  // ---- work items ----
  // Query-major: all row ranges of one query are consecutive in the queue and
  // the largest queries come first, so at any moment the CTAs work on one or
  // two queries and only their HBM tables compete for L2 (with items dealt
  // longest-first across queries, every large query's table was live at once
  // and the random table updates spilled from L2 to DRAM).  A query's rows
  // are cut into about one item per CTA (at least one tile, at most
  // item_rows or 2^20 rows), so one query occupies the whole grid.
  const int64_t item_cap = k.item_rows > 0 ? std::max<int64_t>(T, int64_t(k.item_rows)) : (int64_t(1) << 20);
  std::vector<BatchSpan> spans;
  for (auto& g : groups) {
    g.item_begin = int64_t(spans.size());  // the group's first span
    std::vector<int> order = g.members;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return qd[a].n > qd[b].n; });
    int64_t first = 0;
    // work-item takers of the launch: CTAs, or clusters of g.cluster CTAs
    const int takers = g.cluster > 1 ? std::max(1, g.grid / g.cluster) : ctx->sms * g.minb;
    for (int i : order) {
      int64_t ir = (qd[i].n + takers - 1) / takers;
      // an item ends by merging its shared table into HBM (one insert per
      // group it saw, up to the table's slots): items of at least 16 such
      // merges' worth of rows keep that merge a small share of the item's L2
      // traffic
      const double tslots = double(qi[i].S) * qi[i].cl;
      const int64_t merges =
          qi[i].S > 0 ? int64_t(std::min<double>(qi[i].pred > 0 ? qi[i].pred : tslots, tslots)) : 0;
      ir = std::max<int64_t>(ir, 16 * merges);
      ir = std::min(item_cap, std::max<int64_t>(T, (ir + T - 1) / T * T));
      const int64_t nit = (qd[i].n + ir - 1) / ir;
      if (nit == 0) continue;
      spans.push_back(BatchSpan{qi[i].slot, 0, ir, first});
      first += nit;
    }
    g.nspans = int(int64_t(spans.size()) - g.item_begin);
    g.nitems = first;
    if (g.cluster == 1) g.grid = int(std::max<int64_t>(1, std::min<int64_t>(g.nitems, int64_t(ctx->sms) * g.minb)));
  }
  const int ng = int(groups.size());
  if (trace.on) {
    for (const auto& g : groups) {
      int64_t rows = 0;
      for (int i : g.members) rows += qd[i].n;
      std::fprintf(stderr, "gba_groupby_batch: launch sig=%d cluster=%d grid=%d smem=%zu queries=%zu rows=%lld items=%lld\n",
                   g.sig / 32, g.cluster, g.grid, g.smem, g.members.size(), (long long)rows, (long long)g.nitems);
    }
  }

  // ---- device layout: descriptors | items | block prefixes | status | counters | tables ----
  size_t off = 0;
  auto take = [&](size_t b) {
    const size_t o = off;
    off = round_up(off + b, 256);
    return o;
  };
  const size_t o_q = take(sizeof(BatchQ) * size_t(nt));
  const size_t o_items = take(sizeof(BatchSpan) * spans.size());
  const size_t o_ipre = take(8 * size_t(nt + 1));
  const size_t o_cpre = take(8 * size_t(nt + 1));
  int64_t nxq = 0;
  for (auto& g : xgroups) {
    g.xq_off = nxq;
    nxq += int64_t(g.members.size());
  }
  const size_t o_xq = take(4 * size_t(std::max<int64_t>(nxq, 1)));
  const size_t desc_bytes = off;
  // status: per query flags + group count, per launch item counters, then the
  // exchange kernel's barrier words, flags and per-owner cursors of two buffers
  const size_t xstat = nxq ? 16 + 8 * size_t(xgrid) : 0;
  const size_t o_stat = take(16 * size_t(nt) + 4 * size_t(ng) + xstat);
  const size_t stat_bytes = 16 * size_t(nt) + 4 * size_t(ng) + xstat;
  const size_t o_xstat = o_stat + 16 * size_t(nt) + 4 * size_t(ng);
  const size_t o_xbuf = nxq ? take(2 * size_t(xgrid) * size_t(xregion) * size_t(xstride) * 8) : 0;
  std::vector<size_t> o_tab(nt);
  std::vector<int64_t> ipre(nt + 1, 0), cpre(nt + 1, 0);
  for (int j = 0; j < nt; ++j) {
    const QInfo& x = qi[tq[j]];
    const size_t words = (x.p.table_slots + 1) * size_t(gba_gt_stride(x.q.naccs));
    o_tab[j] = take(words * 8);
    ipre[j + 1] = ipre[j] + int64_t(std::max<size_t>(1, (words + 256 * 16 - 1) / (256 * 16)));
    cpre[j + 1] = cpre[j] + int64_t(std::max<uint64_t>(1, (x.p.table_slots + 2047) / 2048));
  }
  if (nt > 0) {
    gba_status st = gba_ws_reserve(ctx, off, s);
    if (st != GBA_OK) return st;
    st = gba_batch_host_reserve(ctx, desc_bytes + stat_bytes + 256);
    if (st != GBA_OK) return st;
  }
  unsigned char* d = static_cast<unsigned char*>(ctx->ws);
  unsigned char* h = ctx->h_batch;
  const size_t h_stat = round_up(desc_bytes, 256);
  if (nt > 0) {
    BatchQ* hq = reinterpret_cast<BatchQ*>(h + o_q);
    for (int j = 0; j < nt; ++j) {
      const int i = tq[j];
      BatchQ b;
      std::memset(&b, 0, sizeof(b));
      b.q = qd[i];
      b.gt.base = reinterpret_cast<unsigned long long*>(d + o_tab[j]);
      b.gt.cap = qi[i].p.table_slots;
      b.gt.probe_cap = qi[i].p.probe_cap;
      b.out.keys = outs[i].keys;
      for (int a = 0; a < GBA_MAX_AGGS; ++a) b.out.accs[a] = static_cast<unsigned long long*>(outs[i].aggs[a]);
      b.out.capacity = outs[i].capacity;
      b.out.count = reinterpret_cast<unsigned long long*>(d + o_stat + 16 * size_t(j) + 8);
      b.flags = reinterpret_cast<unsigned*>(d + o_stat + 16 * size_t(j));
      b.S = qi[i].S;
      bool vec = aligned16(qd[i].keys);
      for (int c = 0; c < qd[i].ncols; ++c) vec = vec && aligned16(qd[i].cols[c]);
      // bits 8..15: buckets probed per row; a table the query's groups will
      // overfill keeps only what reaches its home bucket
      const double tslots = double(qi[i].S) * (qi[i].xch ? xgrid : qi[i].cl);
      const int nbk = (qi[i].S > 0 && qi[i].pred > 2.0 * tslots) ? 1 : 0;
      // bit 1 (bulk-copy kernel): combine equal keys within a warp first, for
      // queries whose sample shows a key taking at least 1/32 of the rows (one
      // lane of a warp on average) or when the knob forces it
      // (measured on the batch's queries of fewer than 256 ids: combining made
      // the kernel slower, 1.37 against 0.89 ms, so it is opt-in)
      const bool comb = qi[i].tma && k.coalesce == 1;
      // bits 16..27 (exchange): hot-table slots / 4
      b.pad = (vec ? 1 : 0) | (comb ? 2 : 0) | (nbk << 8) | ((qi[i].hot / 4) << 16);  // bit 0: vector loads
      hq[j] = b;
    }
    if (!spans.empty()) std::memcpy(h + o_items, spans.data(), sizeof(BatchSpan) * spans.size());
    std::memcpy(h + o_ipre, ipre.data(), 8 * size_t(nt + 1));
    std::memcpy(h + o_cpre, cpre.data(), 8 * size_t(nt + 1));
    for (const auto& g : xgroups)
      for (size_t m = 0; m < g.members.size(); ++m)
        reinterpret_cast<int*>(h + o_xq)[g.xq_off + int64_t(m)] = qi[g.members[m]].slot;
  }

  // ---- the launch sequence (direct or as a replayed graph) ----
  const BatchQ* d_qs = reinterpret_cast<const BatchQ*>(d + o_q);
  const BatchSpan* d_spans = reinterpret_cast<const BatchSpan*>(d + o_items);
  unsigned* d_ctr = reinterpret_cast<unsigned*>(d + o_stat + 16 * size_t(nt));
  // with timing on, events around the three kernel roles (recorded as graph
  // nodes when captured): [0] table init, [1] pre-aggregation, [2] compaction
  const bool timing = k.timing != 0;
  const bool as_graph = k.use_graph != 0;
  auto mark = [&](int i, cudaStream_t cs) -> cudaError_t {
    if (!timing) return cudaSuccess;
    // inside a capture the event record must be an external graph node
    return as_graph ? cudaEventRecordWithFlags(ctx->tev[i], cs, cudaEventRecordExternal) : cudaEventRecord(ctx->tev[i], cs);
  };
  const int64_t* d_ipre = reinterpret_cast<const int64_t*>(d + o_ipre);
  const int64_t* d_cpre = reinterpret_cast<const int64_t*>(d + o_cpre);
  // table init / compaction of the entries [jb, je)
  auto init_range = [&](int jb, int je, cudaStream_t st) {
    return gba_launch_batch_init(d_qs, d_ipre, je, ipre[je] - ipre[jb], ipre[jb], st);
  };
  auto compact_range = [&](int jb, int je, cudaStream_t st) {
    return gba_launch_batch_compact(d_qs, d_cpre, je, cpre[je] - cpre[jb], cpre[jb], st);
  };
  auto launch_group = [&](int g, cudaStream_t st) {
    return groups[g].tma ? gba_launch_stream_tma(groups[g].proto, groups[g].cluster, groups[g].shape, d_qs,
                                                 d_spans + groups[g].item_begin, groups[g].nspans, groups[g].nitems,
                                                 d_ctr + g, groups[g].smem, sprobe, groups[g].grid, nst,
                                                 groups[g].stage_bytes, st)
                         : gba_launch_stream_agg(groups[g].proto, groups[g].minb, groups[g].hbm, d_qs, d_spans + groups[g].item_begin,
                                                 groups[g].nspans, groups[g].nitems, d_ctr + g, groups[g].smem,
                                                 sprobe, groups[g].grid, st);
  };
  // The streaming launches alternate between two streams, so one launch's
  // tail (its last, small items) overlaps the next launch.  Each launch's
  // tables are cleared just before it and compacted just after it on its own
  // stream, so that the other stream's latency-bound streaming kernel runs
  // beside those bandwidth-bound passes.  With kernel timing on, every clear
  // runs before and every compaction after all streaming launches (the three
  // roles' times are then separate).
  const bool fork = ng >= 2;
  const bool per_group = fork && !timing;
  auto enqueue = [&](cudaStream_t cs) -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(d, h, desc_bytes, cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess) e = cudaMemsetAsync(d + o_stat, 0, stat_bytes, cs);
    if (e == cudaSuccess) e = mark(0, cs);
    if (e == cudaSuccess) e = per_group ? init_range(x_entry_begin, nt, cs) : init_range(0, nt, cs);
    if (e == cudaSuccess) e = mark(1, cs);
    if (fork && e == cudaSuccess) e = cudaEventRecord(ctx->fork_ev[0], cs);
    if (fork && e == cudaSuccess) e = cudaStreamWaitEvent(ctx->aux_stream, ctx->fork_ev[0], 0);
    for (int g = 0; g < ng && e == cudaSuccess; ++g) {
      const cudaStream_t st = fork && (g & 1) ? ctx->aux_stream : cs;
      if (per_group) e = init_range(groups[g].entry_begin, groups[g].entry_end, st);
      if (e == cudaSuccess) e = launch_group(g, st);
      if (per_group && e == cudaSuccess) e = compact_range(groups[g].entry_begin, groups[g].entry_end, st);
    }
    if (fork && e == cudaSuccess) e = cudaEventRecord(ctx->fork_ev[1], ctx->aux_stream);
    if (fork && e == cudaSuccess) e = cudaStreamWaitEvent(cs, ctx->fork_ev[1], 0);
    for (size_t g = 0; g < xgroups.size() && e == cudaSuccess; ++g)
      e = gba_launch_exchange(xgroups[g].proto, d_qs, reinterpret_cast<const int*>(d + o_xq) + xgroups[g].xq_off,
                              int(xgroups[g].members.size()), xwin,
                              reinterpret_cast<unsigned long long*>(d + o_xbuf), xregion,
                              int64_t(xgrid) * xregion * xstride,
                              reinterpret_cast<unsigned*>(d + o_xstat + 16),
                              reinterpret_cast<unsigned*>(d + o_xstat),
                              reinterpret_cast<unsigned*>(d + o_xstat + 8), xgroups[g].smem, sprobe, xgrid, cs);
    if (e == cudaSuccess) e = mark(2, cs);
    if (e == cudaSuccess) e = per_group ? compact_range(x_entry_begin, nt, cs) : compact_range(0, nt, cs);
    if (e == cudaSuccess) e = mark(3, cs);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h + h_stat, d + o_stat, stat_bytes, cudaMemcpyDeviceToHost, cs);
    return e;
  };
  trace.mark("plan");
  if (nt > 0 && ng >= 2 && !ctx->aux_stream) {
    GBA_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->aux_stream, cudaStreamNonBlocking));
    for (auto& ev : ctx->fork_ev) GBA_CUDA_TRY(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  }
  if (nt > 0) {
    for (int g = 0; g < ng; ++g)
      GBA_CUDA_TRY(ctx, groups[g].tma ? gba_prepare_stream_tma(groups[g].proto, groups[g].cluster, groups[g].shape)
                                   : gba_prepare_stream_agg(groups[g].proto, groups[g].minb, groups[g].hbm));
    if (as_graph) {
      // the graph depends only on launch shapes and buffer addresses
      std::vector<int64_t> key = {nt,
                                  int64_t(spans.size()),
                                  ipre[nt],
                                  cpre[nt],
                                  int64_t(desc_bytes),
                                  int64_t(stat_bytes),
                                  int64_t(reinterpret_cast<uintptr_t>(d)),
                                  int64_t(reinterpret_cast<uintptr_t>(h)),
                                  sprobe,
                                  bps,
                                  any_tma ? nst : 0,
                                  timing ? 1 : 0};
      for (const auto& g : groups) {
        key.push_back(g.sig);
        key.push_back(int64_t(g.smem));
        key.push_back(g.item_begin);
        key.push_back(g.nitems);
        key.push_back(g.nspans);
        key.push_back(g.grid);
        key.push_back(int64_t(g.stage_bytes));
        key.push_back(((g.cluster * 16 + g.minb) * 4 + g.shape) * 2 + (g.tma ? 1 : 0));
        // its clear and compaction launches
        key.push_back(g.entry_begin);
        key.push_back(g.entry_end);
        key.push_back(ipre[g.entry_begin]);
        key.push_back(cpre[g.entry_begin]);
      }
      key.push_back(x_entry_begin);
      key.push_back(ipre[x_entry_begin]);
      key.push_back(cpre[x_entry_begin]);
      key.push_back(nxq);
      key.push_back(xwin);
      key.push_back(xregion);
      key.push_back(xgrid);
      for (const auto& g : xgroups) {
        key.push_back(2 * gba_batch_sig_id(g.proto) + (g.proto.key64 ? 1 : 0));
        key.push_back(int64_t(g.smem));
        key.push_back(int64_t(g.members.size()));
      }
      if (!ctx->batch_exec || key != ctx->batch_key) {
        if (ctx->batch_exec) {
          cudaGraphExecDestroy(ctx->batch_exec);
          ctx->batch_exec = nullptr;
        }
        if (!ctx->cap_stream) GBA_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
        GBA_CUDA_TRY(ctx, cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t e = enqueue(ctx->cap_stream);
        cudaGraph_t graph = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(ctx->cap_stream, &graph);
        GBA_CUDA_TRY(ctx, e);
        GBA_CUDA_TRY(ctx, e2);
        const cudaError_t e3 = cudaGraphInstantiate(&ctx->batch_exec, graph, 0);
        cudaGraphDestroy(graph);
        GBA_CUDA_TRY(ctx, e3);
        ctx->batch_key = key;
      }
      GBA_CUDA_TRY(ctx, cudaGraphLaunch(ctx->batch_exec, s));
    } else {
      GBA_CUDA_TRY(ctx, enqueue(s));
    }
    trace.mark("launch");
    GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    trace.mark("table_queries");
    for (int r = 0; timing && r < 3; ++r) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ctx->tev[r], ctx->tev[r + 1]) == cudaSuccess) ctx->stats.kernel_ms[r] += ms;
    }
    ctx->stats.kernel_launches += 2 + ng + int(xgroups.size());
    for (int i : tq) {
      ctx->stats.main_rows += qd[i].n;
      ctx->stats.main_bytes += qd[i].n * int64_t(gba_row_bytes(qd[i]));
    }
  }

  // ---- results; reruns of overflowed queries; partition-strategy queries ----
  gba_status result = GBA_OK;
  gba_stats acc = ctx->stats;
  if (nxq > 0 && (*reinterpret_cast<const unsigned*>(h + h_stat + (o_xstat - o_stat) + 8) & GBA_FLAG_WAIT_TIMEOUT)) {
    ctx->err = "owner-exchange kernel: a bounded grid-barrier wait timed out";
    return GBA_ERR_TIMEOUT;
  }
  std::vector<int> rerun;
  for (int j = 0; j < nt; ++j) {
    const int i = tq[j];
    const unsigned flags = *reinterpret_cast<const unsigned*>(h + h_stat + 16 * size_t(j));
    acc.table_slots += int64_t(qi[i].p.table_slots);
    const unsigned long long cnt = *reinterpret_cast<const unsigned long long*>(h + h_stat + 16 * size_t(j) + 8);
    if (flags & GBA_FLAG_WAIT_TIMEOUT) {
      ctx->err = "query " + std::to_string(i) + ": a bounded device wait timed out";
      return GBA_ERR_TIMEOUT;
    }
    if (flags & GBA_FLAG_TABLE_OVERFLOW) {
      rerun.push_back(i);
      continue;
    }
    n_groups[i] = int64_t(cnt);
    if (int64_t(cnt) > outs[i].capacity && result == GBA_OK) {
      ctx->err = "query " + std::to_string(i) + ": output capacity " + std::to_string(outs[i].capacity) + " < " +
                 std::to_string(cnt) + " groups";
      result = GBA_ERR_OUTPUT_CAPACITY;
    }
  }
  auto run_alone = [&](int i) -> gba_status {
    GbaPlan p = qi[i].p;
    gba_status st;
    if (qi[i].strategy == GBA_STRATEGY_TABLE) {
      p.table_slots *= 4;
      acc.regrows++;
      st = gba_run_table(ctx, qd[i], &outs[i], k, p, s, &n_groups[i]);
    } else {
      st = gba_run_partition(ctx, qd[i], &outs[i], k, p, qi[i].pred, s, &n_groups[i]);
    }
    acc.regrows += ctx->stats.regrows;
    acc.kernel_launches += ctx->stats.kernel_launches;
    acc.main_rows += ctx->stats.main_rows;
    acc.main_bytes += ctx->stats.main_bytes;
    for (int r = 0; r < 4; ++r) acc.kernel_ms[r] += ctx->stats.kernel_ms[r];
    acc.partition_bits = std::max(acc.partition_bits, ctx->stats.partition_bits);
    ctx->stats = gba_stats{};
    return st;
  };
  for (int i : rerun) {
    ctx->stats = gba_stats{};
    const gba_status st = run_alone(i);
    if (st != GBA_OK) {
      ctx->stats = acc;
      ctx->err = "query " + std::to_string(i) + ": " + ctx->err;
      return st;
    }
  }
  for (int i = 0; i < nq; ++i) {
    if (qi[i].strategy == GBA_STRATEGY_TABLE) continue;
    ctx->stats = gba_stats{};
    const gba_status st = run_alone(i);
    if (st != GBA_OK) {
      ctx->stats = acc;
      ctx->err = "query " + std::to_string(i) + ": " + ctx->err;
      return st;
    }
  }
  trace.mark("partition_queries_and_reruns");
  acc.strategy = nt == nq ? GBA_STRATEGY_TABLE : (nt == 0 ? GBA_STRATEGY_PARTITION : GBA_STRATEGY_AUTO);
  acc.preagg = 0;
  for (int j = 0; j < nt; ++j) acc.preagg += qi[tq[j]].S > 0;
  acc.n_groups = 0;
  for (int i = 0; i < nq; ++i) acc.n_groups += n_groups[i];
  ctx->stats = acc;
  return result;
}
