// The reference's two-phase, host-resident entry points, built on the C ABI.
//
//   gba_groupby_partition_u32   (C ABI) one tile: exact GROUP BY SUM of u32
//                               values by u32 key, groups ordered by partition
//                               murmur3_32(key, 0) % P.  Replaces
//                               compute_groupby_agg_result + compute_partition_result
//                               (tiled_groupby_agg_partition/src/group_then_partition.cu:24-306).
//   groupby_agg_partition<u32,u32>, groupby_agg_intra_partition
//                               (C++, include/tiled_groupby_agg_partition.hpp)
//                               the reference's phase 1 (group_then_partition.cu:308-528)
//                               and phase 2 (groupby_agg_intra_partition.cu:159-411).
//
// The reference aggregates each tile with a chain of seven kernels, three CUB
// scans and three blocking host round trips, then partitions it with two more
// kernels and a scan.  Here a tile is one gba_groupby call (shared-memory
// pre-aggregation into an HBM table, one compaction), then three small kernels
// lay its groups out by partition; the host syncs once per call.  Host workers
// (one CUDA stream and one library context each) overlap one tile's copies
// with another tile's aggregation.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <map>
#include <mutex>
#include <queue>
#include <stdexcept>
#include <string>
#include <thread>

#include "../../include/tiled_groupby_agg_partition.hpp"
#include "gba_context.h"
#include "refpart_kernels.h"

static gba_status rp_reserve(gba_context* ctx, size_t bytes, cudaStream_t s) {
  if (bytes <= ctx->rp_bytes) return GBA_OK;
  if (ctx->rp_buf) {
    GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    cudaFree(ctx->rp_buf);
    ctx->rp_buf = nullptr;
    ctx->rp_bytes = 0;
  }
  const size_t want = gba_round_up(std::max(bytes, size_t(1) << 20), size_t(1) << 20);
  GBA_CUDA_TRY(ctx, cudaMalloc(&ctx->rp_buf, want));
  ctx->rp_bytes = want;
  return GBA_OK;
}

extern "C" gba_status gba_groupby_partition_u32(gba_context* ctx, const uint32_t* keys, const uint32_t* vals,
                                                int64_t n_rows, int32_t P, uint32_t* out_keys, uint32_t* out_vals,
                                                uint64_t* part_offsets, void* stream) {
  if (!ctx || !part_offsets) return GBA_ERR_INVALID_ARG;
  if (n_rows < 0 || P < 1 || P > GBA_REFPART_MAX_P) {
    ctx->err = "need n_rows >= 0 and 1 <= P <= " + std::to_string(GBA_REFPART_MAX_P);
    return GBA_ERR_INVALID_ARG;
  }
  if (n_rows > 0 && (!keys || !vals || !out_keys || !out_vals)) {
    ctx->err = "null column";
    return GBA_ERR_INVALID_ARG;
  }
  cudaSetDevice(ctx->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // scratch: the tile's groups (u32 keys, int64 sums), histogram, offsets, cursors
  const size_t cap = size_t(n_rows) + 1;
  const size_t o_sums = gba_round_up(cap * 4, 256);
  const size_t o_hist = gba_round_up(o_sums + cap * 8, 256);
  const size_t o_offs = gba_round_up(o_hist + size_t(P) * 4, 256);
  const size_t o_cur = gba_round_up(o_offs + size_t(P + 1) * 8, 256);
  const size_t total = o_cur + size_t(P) * 8;
  gba_status st = rp_reserve(ctx, total, s);
  if (st != GBA_OK) return st;
  unsigned char* b = static_cast<unsigned char*>(ctx->rp_buf);
  unsigned* g_keys = reinterpret_cast<unsigned*>(b);
  unsigned long long* g_sums = reinterpret_cast<unsigned long long*>(b + o_sums);

  gba_query q{};
  q.n_rows = n_rows;
  q.key.type = GBA_U32;
  q.key.data = keys;
  q.n_cols = 1;
  q.cols[0].type = GBA_U32;
  q.cols[0].data = vals;
  q.n_aggs = 1;
  q.aggs[0].op = GBA_SUM;
  q.aggs[0].col = 0;
  gba_output o{};
  o.keys = g_keys;
  o.aggs[0] = g_sums;
  o.capacity = int64_t(cap);
  int64_t g = 0;
  const auto t0 = std::chrono::steady_clock::now();
  st = gba_groupby(ctx, &q, &o, nullptr, stream, &g);
  if (st != GBA_OK) return st;
  if (std::getenv("GBA_TRACE"))
    std::fprintf(stderr, "gba_groupby_partition_u32: %lld rows, %lld groups, strategy %d, %lld slots, %.3f ms\n",
                 (long long)n_rows, (long long)g, ctx->stats.strategy, (long long)ctx->stats.table_slots,
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
  unsigned long long* offs = reinterpret_cast<unsigned long long*>(b + o_offs);
  GBA_CUDA_TRY(ctx, gba_launch_refpart(g_keys, g_sums, g, P, out_keys, out_vals, reinterpret_cast<unsigned*>(b + o_hist),
                                       offs, reinterpret_cast<unsigned long long*>(b + o_cur), ctx->sms, s));
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(part_offsets, offs, size_t(P + 1) * 8, cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  ctx->stats.kernel_launches += g > 0 ? 3 : 1;
  if (part_offsets[P] != uint64_t(g)) {
    ctx->err = "partition offsets do not add up to the group count";
    return GBA_ERR_CUDA;
  }
  return GBA_OK;
}

// ---------------------------------------------------------------------------
// C++ drop-ins
namespace {

// One merged partition's piece of the phase-1 output: `len` pairs at `src`
// of the uploaded runs, to `dst` of the partition's own rows.
struct SegCopy {
  uint64_t src, dst;
  uint64_t len;
};

// Gathers every segment of a merged partition into contiguous rows: one CTA
// per segment at a time, 128-bit copies where both ends allow them.
__global__ void k_gather_segments(const SegCopy* segs, int nseg, const uint32_t* src_k, const uint32_t* src_v,
                                  uint32_t* dst_k, uint32_t* dst_v) {
  for (int i = blockIdx.x; i < nseg; i += gridDim.x) {
    const SegCopy c = segs[i];
    for (uint64_t j = threadIdx.x; j < c.len; j += blockDim.x) {
      dst_k[c.dst + j] = src_k[c.src + j];
      dst_v[c.dst + j] = src_v[c.src + j];
    }
  }
}

// One host worker: a library context, a stream and device column buffers.
struct TileWorker {
  gba_context* ctx = nullptr;
  cudaStream_t s = nullptr;
  uint32_t* d_keys = nullptr;
  uint32_t* d_vals = nullptr;
  size_t cap = 0;
  // phase 2: the uploaded phase-1 output (keys then values) and the segment list
  uint32_t* d_runs = nullptr;
  size_t runs_cap = 0;
  SegCopy* d_segs = nullptr;
  size_t segs_cap = 0;
  int device = 0;

  explicit TileWorker(int dev) : device(dev) {
    cudaSetDevice(dev);
    if (gba_create(&ctx, dev) != GBA_OK) throw std::runtime_error("gba_create failed on device " + std::to_string(dev));
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      gba_destroy(ctx);
      throw std::runtime_error("cudaStreamCreate failed");
    }
  }
  ~TileWorker() {
    cudaSetDevice(device);
    if (s) cudaStreamSynchronize(s);
    if (d_keys) cudaFree(d_keys);
    if (d_vals) cudaFree(d_vals);
    if (d_runs) cudaFree(d_runs);
    if (d_segs) cudaFree(d_segs);
    if (s) cudaStreamDestroy(s);
    if (ctx) gba_destroy(ctx);
  }
  TileWorker(const TileWorker&) = delete;
  TileWorker& operator=(const TileWorker&) = delete;

  void reserve(size_t rows) {
    if (rows <= cap) return;
    if (d_keys) cudaFree(d_keys);
    if (d_vals) cudaFree(d_vals);
    d_keys = d_vals = nullptr;
    cap = 0;
    cuda(cudaMalloc(&d_keys, std::max<size_t>(rows, 1) * 4), "cudaMalloc");
    cuda(cudaMalloc(&d_vals, std::max<size_t>(rows, 1) * 4), "cudaMalloc");
    cap = rows;
  }
  void reserve_runs(size_t pairs, size_t nseg) {
    if (pairs > runs_cap) {
      cuda(cudaStreamSynchronize(s), "sync");
      if (d_runs) cudaFree(d_runs);
      d_runs = nullptr;
      runs_cap = 0;
      cuda(cudaMalloc(&d_runs, std::max<size_t>(pairs, 1) * 8), "cudaMalloc");
      runs_cap = pairs;
    }
    if (nseg > segs_cap) {
      cuda(cudaStreamSynchronize(s), "sync");
      if (d_segs) cudaFree(d_segs);
      d_segs = nullptr;
      segs_cap = 0;
      cuda(cudaMalloc(&d_segs, std::max<size_t>(nseg, 1) * sizeof(SegCopy)), "cudaMalloc");
      segs_cap = nseg;
    }
  }
  static void cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
  }
  void check(gba_status st) {
    if (st != GBA_OK) throw std::runtime_error(std::string("gba: ") + gba_status_string(st) + ": " + gba_last_error(ctx));
  }
  // groups of the rows now in d_keys/d_vals[0, n), ordered by partition, in place
  void group_partition(size_t n, size_t P, uint64_t* offsets) {
    check(gba_groupby_partition_u32(ctx, d_keys, d_vals, int64_t(n), int32_t(P), d_keys, d_vals, offsets, s));
  }
};

// Workers outlive the calls that use them: a process-wide pool per device
// hands each call the workers it needs (creating more only when every
// existing one is busy) and takes them back at the end, so their contexts,
// streams, pinned staging and device buffers are made once, not per call
// (measured: creating and destroying four workers per call cost more than the
// aggregation of a 2^20-row input).  Calls on other threads take other workers,
// so concurrent calls stay independent.  The pool is never torn down: its
// workers hold their device memory until the process exits.
class WorkerPool {
 public:
  TileWorker* acquire(int dev) {
    {
      std::lock_guard<std::mutex> g(mu_);
      auto& f = free_[dev];
      if (!f.empty()) {
        TileWorker* w = f.back();
        f.pop_back();
        return w;
      }
    }
    return new TileWorker(dev);
  }
  void release(TileWorker* w) {
    std::lock_guard<std::mutex> g(mu_);
    free_[w->device].push_back(w);
  }
  static WorkerPool& get() {
    static WorkerPool* p = new WorkerPool();  // intentionally never destroyed
    return *p;
  }

 private:
  std::mutex mu_;
  std::map<int, std::vector<TileWorker*>> free_;
};

int dev_of_call() {
  int dev = 0;
  cudaGetDevice(&dev);
  return dev;
}

// Runs fn(worker, item) for items [0, count) over `nw` workers; rethrows the
// first error after every worker stopped.
template <typename Fn>
void run_workers(size_t nw, size_t count, Fn fn) {
  int dev = 0;
  cudaGetDevice(&dev);
  nw = std::max<size_t>(1, std::min(nw, count));
  std::vector<TileWorker*> ws;
  try {
    for (size_t i = 0; i < nw; ++i) ws.push_back(WorkerPool::get().acquire(dev));
  } catch (...) {
    for (TileWorker* w : ws) WorkerPool::get().release(w);
    throw;
  }
  std::atomic<size_t> next{0};
  std::atomic<bool> failed{false};
  std::exception_ptr err;
  std::mutex err_lock;
  auto body = [&](TileWorker* w) {
    try {
      cudaSetDevice(dev);
      for (;;) {
        if (failed.load()) break;
        const size_t i = next.fetch_add(1);
        if (i >= count) break;
        fn(*w, i);
      }
    } catch (...) {
      std::lock_guard<std::mutex> g(err_lock);
      if (!err) err = std::current_exception();
      failed = true;
    }
  };
  std::vector<std::thread> th;
  for (size_t i = 1; i < nw; ++i) th.emplace_back(body, ws[i]);
  body(ws[0]);
  for (auto& t : th) t.join();
  for (TileWorker* w : ws) {
    cudaStreamSynchronize(w->s);  // nothing of this call in flight when the worker is handed on
    WorkerPool::get().release(w);
  }
  if (err) std::rethrow_exception(err);
}

// The reference's partition merge (groupby_agg_intra_partition.cu:13-48): a
// min-heap by size; the smallest partition absorbs the next smallest while the
// sum stays within K.  std::priority_queue with the same comparator, built
// from the same sequence and driven by the same push/pop sequence, so equal
// sizes break ties the same way and par_kv_begin comes out identical.
std::vector<par_result> merge_partitions(std::vector<par_result>& in, size_t K) {
  auto cmp = [](const par_result& l, const par_result& r) { return l.size > r.size; };
  std::priority_queue<par_result, std::vector<par_result>, decltype(cmp)> H(in.begin(), in.end(), cmp);
  while (H.size() > 1) {
    par_result acc = H.top();
    H.pop();
    if (size_t(acc.size) + H.top().size > K) {
      H.push(acc);
      break;
    }
    par_result next = H.top();
    for (;;) {
      acc.merge(next);
      H.pop();
      if (H.empty()) break;
      next = H.top();
      if (size_t(next.size) + acc.size > K) break;
    }
    H.push(acc);
  }
  std::vector<par_result> out;
  out.reserve(H.size());
  while (!H.empty()) {
    out.push_back(H.top());
    H.pop();
  }
  return out;
}

}  // namespace

template <>
void groupby_agg_partition<uint32_t, uint32_t>(uint32_t* host_keys_buffer, uint32_t* host_vals_buffer,
                                               size_t kv_buffer_len, size_t tile_len, size_t P,
                                               std::vector<par_result>& par_result_vec, size_t nstreams) {
  if (P < 1 || P > GBA_REFPART_MAX_P) throw std::invalid_argument("groupby_agg_partition: P must be in [1, 16384]");
  if (tile_len < 1 || tile_len > (size_t(1) << 32) - 2)
    throw std::invalid_argument("groupby_agg_partition: tile_len must be in [1, 2^32 - 2]");
  if (kv_buffer_len > 0 && (!host_keys_buffer || !host_vals_buffer))
    throw std::invalid_argument("groupby_agg_partition: null buffer");
  if (par_result_vec.size() < P) par_result_vec.resize(P);
  const size_t tiles = (kv_buffer_len + tile_len - 1) / tile_len;
  std::vector<uint64_t> offs(tiles * (P + 1));
  run_workers(nstreams, tiles, [&](TileWorker& w, size_t t) {
    const size_t b = t * tile_len;
    const size_t m = std::min(tile_len, kv_buffer_len - b);
    w.reserve(m);
    TileWorker::cuda(cudaMemcpyAsync(w.d_keys, host_keys_buffer + b, m * 4, cudaMemcpyHostToDevice, w.s), "H2D");
    TileWorker::cuda(cudaMemcpyAsync(w.d_vals, host_vals_buffer + b, m * 4, cudaMemcpyHostToDevice, w.s), "H2D");
    uint64_t* o = offs.data() + t * (P + 1);
    w.group_partition(m, P, o);
    const size_t g = o[P];
    // the tile's groups, partition-ordered, over the front of its own range
    TileWorker::cuda(cudaMemcpyAsync(host_keys_buffer + b, w.d_keys, g * 4, cudaMemcpyDeviceToHost, w.s), "D2H");
    TileWorker::cuda(cudaMemcpyAsync(host_vals_buffer + b, w.d_vals, g * 4, cudaMemcpyDeviceToHost, w.s), "D2H");
    TileWorker::cuda(cudaStreamSynchronize(w.s), "sync");
  });
  for (size_t t = 0; t < tiles; ++t) {
    const uint64_t* o = offs.data() + t * (P + 1);
    const size_t b = t * tile_len;
    for (size_t p = 0; p < P; ++p)
      par_result_vec[p].push(host_keys_buffer + b + o[p], host_vals_buffer + b + o[p], uint32_t(o[p + 1] - o[p]));
  }
}

void groupby_agg_intra_partition(std::vector<par_result>& par_result_vec, key_type*& host_groupby_keys_result,
                                 val_type*& host_agg_vals_result, size_t Capacity, size_t min_load_num,
                                 size_t max_load_num, size_t nstreams, std::vector<size_t>& par_kv_begin,
                                 std::vector<size_t>& par_result_kv_num) {
  (void)Capacity;
  (void)max_load_num;
  if (par_result_vec.empty()) throw std::invalid_argument("groupby_agg_intra_partition: no partitions");
  const bool trace = std::getenv("GBA_TRACE") != nullptr;
  const auto t_in = std::chrono::steady_clock::now();
  par_result_vec = merge_partitions(par_result_vec, min_load_num);
  const size_t np = par_result_vec.size();
  par_kv_begin.clear();
  par_kv_begin.reserve(np);
  par_result_kv_num.assign(np, 0);
  size_t total = 0;
  for (size_t i = 0; i < np; ++i) {
    par_kv_begin.push_back(total);
    total += par_result_vec[i].size;
  }
  host_groupby_keys_result = nullptr;
  host_agg_vals_result = nullptr;
  TileWorker::cuda(cudaMallocHost(&host_groupby_keys_result, std::max<size_t>(total, 1) * sizeof(key_type)),
                   "cudaMallocHost");
  TileWorker::cuda(cudaMallocHost(&host_agg_vals_result, std::max<size_t>(total, 1) * sizeof(val_type)),
                   "cudaMallocHost");
  if (trace)
    std::fprintf(stderr, "groupby_agg_intra_partition: merge and pinned result arrays (%zu pairs): %.3f ms\n", total,
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_in).count());
  if (total == 0) return;

  // Every segment (a tile's run of one partition) of every merged partition.
  // Phase 1 left each tile's groups contiguous at the front of the tile's own
  // range, so the segments sorted by address join into a few contiguous runs
  // (about one per tile); each run is copied to the device once, and each
  // merged partition is gathered there by one kernel.  (One host-to-device
  // copy per segment, thousands of them, had made phase 2 slower than the
  // reference, which gathers them on the host.)
  struct Seg {
    const key_type* k;
    const val_type* v;
    uint64_t len;
    size_t part;
    uint64_t dst;  // offset in the partition's gathered rows
    uint64_t src;  // offset in the uploaded runs
  };
  std::vector<Seg> segs;
  for (size_t i = 0; i < np; ++i) {
    const par_result& pr = par_result_vec[i];
    uint64_t at = 0;
    for (size_t sg = 0; sg < pr.key.size(); ++sg) {
      const uint64_t len = pr.end_indicator[sg];
      if (!len) continue;
      segs.push_back(Seg{pr.key[sg], pr.val[sg], len, i, at, 0});
      at += len;
    }
  }
  std::vector<size_t> order(segs.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return segs[a].k < segs[b].k; });
  struct Run {
    const key_type* k;
    const val_type* v;
    uint64_t len, off;
  };
  std::vector<Run> runs;
  uint64_t up = 0;
  for (size_t oi : order) {
    Seg& g = segs[oi];
    if (!runs.empty()) {
      Run& r = runs.back();
      if (g.k == r.k + r.len && g.v == r.v + r.len) {  // continues the run
        g.src = r.off + r.len;
        r.len += g.len;
        up += g.len;
        continue;
      }
      if (g.k >= r.k && g.k + g.len <= r.k + r.len && g.v == r.v + (g.k - r.k)) {  // inside the run
        g.src = r.off + uint64_t(g.k - r.k);
        continue;
      }
    }
    g.src = up;
    runs.push_back(Run{g.k, g.v, g.len, up});
    up += g.len;
  }
  // per merged partition, its segment copies (in segment order)
  std::vector<SegCopy> copies(segs.size());
  std::vector<size_t> first(np + 1, 0);
  for (const Seg& g : segs) ++first[g.part + 1];
  for (size_t i = 0; i < np; ++i) first[i + 1] += first[i];
  {
    std::vector<size_t> fill(first.begin(), first.end() - 1);
    for (const Seg& g : segs) copies[fill[g.part]++] = SegCopy{g.src, g.dst, g.len};
  }
  size_t maxpart = 0;
  for (size_t i = 0; i < np; ++i) maxpart = std::max<size_t>(maxpart, par_result_vec[i].size);

  // The runs and the segment list go up once, on the first worker's stream;
  // then the workers take merged partitions in turn, each gathering its
  // partition from the shared runs into its own buffers, aggregating it and
  // copying its groups back.
  const auto t0 = std::chrono::steady_clock::now();
  TileWorker* up_w = WorkerPool::get().acquire(dev_of_call());
  cudaEvent_t uploaded = nullptr;
  try {
    up_w->reserve_runs(up, copies.size());
    for (const Run& r : runs) {
      TileWorker::cuda(cudaMemcpyAsync(up_w->d_runs + r.off, r.k, r.len * 4, cudaMemcpyHostToDevice, up_w->s), "H2D");
      TileWorker::cuda(cudaMemcpyAsync(up_w->d_runs + up + r.off, r.v, r.len * 4, cudaMemcpyHostToDevice, up_w->s),
                       "H2D");
    }
    TileWorker::cuda(cudaMemcpyAsync(up_w->d_segs, copies.data(), copies.size() * sizeof(SegCopy),
                                     cudaMemcpyHostToDevice, up_w->s), "H2D");
    TileWorker::cuda(cudaEventCreateWithFlags(&uploaded, cudaEventDisableTiming), "event");
    TileWorker::cuda(cudaEventRecord(uploaded, up_w->s), "event");
    const uint32_t* rk = up_w->d_runs;
    const uint32_t* rv = up_w->d_runs + up;
    const SegCopy* dsegs = up_w->d_segs;
    run_workers(nstreams, np, [&](TileWorker& w, size_t i) {
      TileWorker::cuda(cudaStreamWaitEvent(w.s, uploaded, 0), "wait");
      w.reserve(par_result_vec[i].size);
      const int nseg = int(first[i + 1] - first[i]);
      if (nseg > 0) {
        k_gather_segments<<<std::min(nseg, 4 * w.ctx->sms), 256, 0, w.s>>>(dsegs + first[i], nseg, rk, rv, w.d_keys,
                                                                          w.d_vals);
        TileWorker::cuda(cudaGetLastError(), "gather");
      }
      uint64_t o[2];
      w.group_partition(par_result_vec[i].size, 1, o);
      const size_t g = o[1];
      TileWorker::cuda(cudaMemcpyAsync(host_groupby_keys_result + par_kv_begin[i], w.d_keys, g * 4,
                                       cudaMemcpyDeviceToHost, w.s), "D2H");
      TileWorker::cuda(cudaMemcpyAsync(host_agg_vals_result + par_kv_begin[i], w.d_vals, g * 4,
                                       cudaMemcpyDeviceToHost, w.s), "D2H");
      TileWorker::cuda(cudaStreamSynchronize(w.s), "sync");
      par_result_kv_num[i] = g;
    });
  } catch (...) {
    if (uploaded) cudaEventDestroy(uploaded);
    cudaStreamSynchronize(up_w->s);
    WorkerPool::get().release(up_w);
    throw;
  }
  cudaEventDestroy(uploaded);
  cudaStreamSynchronize(up_w->s);
  WorkerPool::get().release(up_w);
  if (trace)
    std::fprintf(stderr, "groupby_agg_intra_partition: %zu merged partitions, %zu runs, %zu segments, %.3f ms\n", np,
                 runs.size(), segs.size(),
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
}
