// gba_groupby_noalloc: the table strategy (k_table_init -> k_preagg ->
// k_compact) over a fixed, statically allocated device scratch instead of the
// context's growable workspace.  Nothing here calls cudaMalloc, cudaFree or any
// other allocating routine.
//
// Who needs it: callers that must not allocate device memory per call.  Two
// common cases: a process whose device memory is already reserved up front by
// its own pool allocator (a framework's caching allocator, a fixed arena), where
// a fresh cudaMalloc can fail even though the query needs only a few MB; and a
// latency-sensitive thread sharing the device with other streams, where
// cudaFree (and sometimes cudaMalloc) synchronises the whole device and stalls
// unrelated work.
//
// The scratch is one file-scope __device__ array per device (the module's
// global memory, set up by the driver when the module loads).  Its layout:
//   bytes [0, 4)     status flags        (cleared to zero by every call)
//   bytes [8, 16)    group counter       (cleared to zero by every call)
//   bytes [256, ...) HBM hash table      (initialised by k_table_init)
// Because every call on a device uses the same scratch, calls that overlap in
// time on one device (two streams, two threads, two contexts) race and corrupt
// each other's results; callers serialise them.
#include <cstring>
#include <mutex>
#include <string>

#include "gba_context.h"
#include "gba_plan.h"
#include "nulls.h"

// The fixed scratch: 16 MiB, 256-byte aligned.
static constexpr size_t kNoallocScratchBytes = size_t(16) << 20;
static constexpr size_t kNoallocTableOffset = 256;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoallocScratchBytes / 8];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Address of this device's scratch, looked up once per device with that device
// current (the caller has made it current).  The first lookup may make the
// runtime load the library's device code.  The address is kept for the life of
// the process: a caller that resets the device (cudaDeviceReset) unloads the
// module that holds the array, and must not call this entry point afterwards.
gba_status noalloc_scratch(gba_context* ctx, unsigned char** out) {
  const int dev = ctx->device;
  if (dev < 0 || dev >= kMaxDevices) {
    ctx->err = "gba_groupby_noalloc: device index " + std::to_string(dev) + " out of range";
    return GBA_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      ctx->err = std::string("gba_groupby_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return GBA_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  return GBA_OK;
}

}  // namespace

extern "C" gba_status gba_groupby_noalloc(gba_context* ctx, const gba_query* q_in, const gba_output* out,
                                          void* stream, int64_t* n_groups) {
  if (!ctx || !q_in || !out || !n_groups) return GBA_ERR_INVALID_ARG;
  GBA_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  // the call reads its group count back and synchronises the stream: it
  // cannot be part of a stream capture
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  GBA_CUDA_TRY(ctx, cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &capture));
  if (capture != cudaStreamCaptureStatusNone) {
    ctx->err = "gba_groupby_noalloc: the stream is being captured; the call synchronises it and cannot be captured";
    return GBA_ERR_INVALID_ARG;
  }
  ctx->stats = gba_stats{};
  ctx->stats.predicted_groups = -1;
  // per-aggregate validity outputs and a second key output belong to the
  // nullable-column and composite-key rewrites, which need scratch of their own
  if (gba_nulls_needed(*q_in, *out) || out->keys2 || q_in->key2.data) {
    ctx->err = "gba_groupby_noalloc: nullable columns, validity outputs (gba_output.agg_valid), COUNT(col) and "
               "composite keys are supported by gba_groupby and gba_groupby_batch only";
    return GBA_ERR_UNSUPPORTED;
  }
  gba_query qc;
  gba_compact_query(q_in, &qc);
  QDesc q;
  gba_status st = gba_build_qdesc(ctx, &qc, &q);
  if (st != GBA_OK) return st;
  if (out->capacity < 0 || (out->capacity > 0 && !out->keys)) {
    ctx->err = "bad output descriptor";
    return GBA_ERR_INVALID_ARG;
  }
  for (int a = 0; a < qc.n_aggs; ++a)
    if (out->capacity > 0 && !out->aggs[a]) {
      ctx->err = "null output aggregate column";
      return GBA_ERR_INVALID_ARG;
    }

  // Capacity 2 n + 64 (load <= 0.5 even if every key is distinct), walked to
  // the end on a collision chain, so the table cannot overflow.
  const size_t stride = size_t(gba_gt_stride(q.naccs));
  const uint64_t cap = 2 * uint64_t(q.n) + 64;
  const size_t need = kNoallocTableOffset + (cap + 1) * stride * 8;
  if (need > kNoallocScratchBytes) {
    const int64_t max_rows = int64_t(((kNoallocScratchBytes - kNoallocTableOffset) / (stride * 8) - 1 - 64) / 2);
    ctx->err = "gba_groupby_noalloc: " + std::to_string(q.n) + " rows need a " + std::to_string(need) +
               "-byte table, larger than the fixed " + std::to_string(kNoallocScratchBytes) +
               "-byte scratch (at most " + std::to_string(max_rows) + " rows with " + std::to_string(q.naccs) +
               " aggregates); use gba_groupby";
    return GBA_ERR_INVALID_ARG;
  }
  unsigned char* scratch = nullptr;
  st = noalloc_scratch(ctx, &scratch);
  if (st != GBA_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  gba_knobs k;
  gba_default_knobs(&k);
  k.sizing = GBA_SIZING_PLAIN;
  GbaPlan p;
  gba_make_plan(ctx, q, k, -1.0, &p);

  unsigned* d_flags = reinterpret_cast<unsigned*>(scratch);
  unsigned long long* d_count = reinterpret_cast<unsigned long long*>(scratch + 8);
  GBA_CUDA_TRY(ctx, cudaMemsetAsync(scratch, 0, 16, s));  // flags and group counter start at zero
  GTable t;
  t.base = reinterpret_cast<unsigned long long*>(scratch + kNoallocTableOffset);
  t.cap = cap;
  t.probe_cap = int(cap);
  const size_t words = (cap + 1) * stride;
  GBA_CUDA_TRY(ctx, gba_launch_table_init(t, q, int(std::min<size_t>(size_t(ctx->sms) * 16, words / 256 + 1)), s));
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
    GBA_CUDA_TRY(ctx, gba_launch_preagg(q, t, c, d_flags, s));
    ++launches;
  }
  OutDesc o;
  o.keys = out->keys;
  for (int a = 0; a < GBA_MAX_AGGS; ++a) o.accs[a] = static_cast<unsigned long long*>(out->aggs[a]);
  o.capacity = out->capacity;
  o.count = d_count;
  GBA_CUDA_TRY(ctx, gba_launch_compact(t, q, o, int(std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(ctx->sms) * 8, (cap + 255) / 256))), s));
  ++launches;
  unsigned long long hbuf[2] = {0, 0};
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(hbuf, scratch, 16, cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  const unsigned flags = unsigned(hbuf[0] & 0xffffffffull);
  const unsigned long long count = hbuf[1];
  ctx->stats.strategy = GBA_STRATEGY_TABLE;
  ctx->stats.preagg = p.smem_slots > 0;
  ctx->stats.table_slots = int64_t(cap);
  ctx->stats.kernel_launches = launches;
  if (flags & GBA_FLAG_WAIT_TIMEOUT) {
    ctx->err = "a bounded TMA wait timed out";
    return GBA_ERR_TIMEOUT;
  }
  if (flags & GBA_FLAG_TABLE_OVERFLOW) {
    ctx->err = "HBM hash table overflow";
    return GBA_ERR_TABLE_OVERFLOW;
  }
  *n_groups = int64_t(count);
  ctx->stats.n_groups = int64_t(count);
  if (int64_t(count) > out->capacity) {
    ctx->err = "output capacity " + std::to_string(out->capacity) + " < " + std::to_string(count) + " groups";
    return GBA_ERR_OUTPUT_CAPACITY;
  }
  return GBA_OK;
}
