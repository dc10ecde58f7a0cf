// Host-resident batch: gba_groupby_batch over inputs and outputs in host
// memory (the reference's host-resident "coprocess" mode,
// group_then_partition.cu:353-418, for many queries at once).
//
// The queries are cut, in order, into parts of about a quarter of the batch's
// input bytes.  Every input copy is queued at once on the copy stream (one
// cudaMemcpyAsync per column), with an event after each part; part p runs as
// one gba_groupby_batch call on the caller's stream once its event completed,
// so part p + 1's columns cross the host link while part p aggregates.  Part
// p's groups go back to the caller's buffers on a third stream (the link's
// other direction) while the later parts run.  Every row crosses the link
// once, every group once.
#include <algorithm>
#include <string>
#include <vector>

#include "gba_context.h"

gba_status gba_stage_reserve(gba_context* ctx, size_t bytes, cudaStream_t s);

namespace {

// input bytes of a query (keys, second keys, value columns, validity bitmaps)
size_t query_in_bytes(const gba_query& q) {
  const size_t n = size_t(std::max<int64_t>(q.n_rows, 0));
  size_t b = n * size_t(gba_type_bytes(q.key.type));
  if (q.key2.data) b += n * size_t(gba_type_bytes(q.key2.type));
  for (int c = 0; c < q.n_cols; ++c) {
    b += n * size_t(gba_type_bytes(q.cols[c].type));
    if (q.cols[c].valid) b += (n + 7) / 8;
  }
  return b;
}

struct Staged {
  gba_query q;   // device columns
  gba_output o;  // device outputs
};

// Waits (host) for both copy streams, so that no copy still reads or writes
// the caller's buffers when the call returns.
void drain(gba_context* ctx, cudaStream_t out_s) {
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  if (out_s) cudaStreamSynchronize(out_s);
}

}  // namespace

extern "C" gba_status gba_groupby_batch_host(gba_context* ctx, int32_t nq, const gba_query* qs, const gba_output* outs,
                                             const gba_knobs* knobs, void* stream, int64_t* n_groups) {
  if (!ctx || nq < 0 || (nq > 0 && (!qs || !outs || !n_groups))) return GBA_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  if (nq == 0) return GBA_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  gba_knobs k;
  if (knobs) k = *knobs;
  else gba_default_knobs(&k);
  // the parts differ in shape: direct launches, unless a graph is asked for
  if (k.use_graph < 0) k.use_graph = 0;

  // ---- device staging: every query's inputs and outputs ----
  std::vector<Staged> dv(nq);
  std::vector<size_t> in_off(nq), out_off(nq);
  size_t off = 0, total_in = 0;
  auto take = [&](size_t b) {
    const size_t o = off;
    off = gba_round_up(off + b, 256);
    return o;
  };
  struct Place {
    size_t key, key2, col[GBA_MAX_COLS], valid[GBA_MAX_COLS];
    size_t okeys, okeys2, oacc[GBA_MAX_AGGS], ovalid[GBA_MAX_AGGS];
    int64_t cap;
  };
  std::vector<Place> pl(nq);
  for (int i = 0; i < nq; ++i) {
    const gba_query& q = qs[i];
    const gba_output& o = outs[i];
    if (q.n_rows < 0 || q.n_cols < 0 || q.n_cols > GBA_MAX_COLS || q.n_aggs < 1 || q.n_aggs > GBA_MAX_AGGS ||
        o.capacity < 0 || (q.n_rows > 0 && !q.key.data)) {
      ctx->err = "query " + std::to_string(i) + ": bad host query or output descriptor";
      return GBA_ERR_INVALID_ARG;
    }
    const size_t n = size_t(q.n_rows);
    Place& p = pl[i];
    p.key = take(n * size_t(gba_type_bytes(q.key.type)));
    p.key2 = q.key2.data ? take(n * size_t(gba_type_bytes(q.key2.type))) : 0;
    for (int c = 0; c < q.n_cols; ++c) {
      p.col[c] = take(n * size_t(gba_type_bytes(q.cols[c].type)));
      p.valid[c] = q.cols[c].valid ? take((n + 7) / 8) : 0;
    }
    total_in += query_in_bytes(q);
    // a query has at most n_rows groups: the device output holds no more
    p.cap = std::min<int64_t>(o.capacity, std::max<int64_t>(q.n_rows, 1));
    const size_t cap = size_t(p.cap);
    p.okeys = take(cap * size_t(gba_type_bytes(q.key.type)));
    p.okeys2 = o.keys2 ? take(cap * size_t(gba_type_bytes(q.key2.type))) : 0;
    for (int a = 0; a < q.n_aggs; ++a) {
      p.oacc[a] = take(cap * 8);
      p.ovalid[a] = o.agg_valid[a] ? take(cap) : 0;
    }
  }
  gba_status st = gba_stage_reserve(ctx, off, s);
  if (st != GBA_OK) return st;
  unsigned char* base = static_cast<unsigned char*>(ctx->stage);
  for (int i = 0; i < nq; ++i) {
    const gba_query& q = qs[i];
    const gba_output& o = outs[i];
    const Place& p = pl[i];
    Staged& d = dv[i];
    d.q = q;
    d.q.key.data = base + p.key;
    if (q.key2.data) d.q.key2.data = base + p.key2;
    for (int c = 0; c < q.n_cols; ++c) {
      d.q.cols[c].data = base + p.col[c];
      d.q.cols[c].valid = q.cols[c].valid ? base + p.valid[c] : nullptr;
    }
    d.o = gba_output{};
    d.o.capacity = p.cap;
    d.o.keys = base + p.okeys;
    d.o.keys2 = o.keys2 ? base + p.okeys2 : nullptr;
    for (int a = 0; a < q.n_aggs; ++a) {
      d.o.aggs[a] = base + p.oacc[a];
      d.o.agg_valid[a] = o.agg_valid[a] ? base + p.ovalid[a] : nullptr;
    }
  }

  // ---- parts: about a quarter of the input bytes each (at least 64 MB) ----
  const size_t target = std::max<size_t>(size_t(64) << 20, total_in / 4 + 1);
  std::vector<int> part_end;  // one past each part's last query
  size_t acc = 0;
  for (int i = 0; i < nq; ++i) {
    acc += query_in_bytes(qs[i]);
    if (acc >= target || i == nq - 1) {
      part_end.push_back(i + 1);
      acc = 0;
    }
  }
  const int np = int(part_end.size());

  if (!ctx->copy_stream) GBA_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  if (!ctx->out_stream) GBA_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->out_stream, cudaStreamNonBlocking));
  while (int(ctx->part_ev.size()) < np + 1) {
    cudaEvent_t e;
    GBA_CUDA_TRY(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->part_ev.push_back(e);
  }
  cudaStream_t cs = ctx->copy_stream, os = ctx->out_stream;
  // the staging may still be read by earlier work on the caller's stream
  GBA_CUDA_TRY(ctx, cudaEventRecord(ctx->part_ev[np], s));
  GBA_CUDA_TRY(ctx, cudaStreamWaitEvent(cs, ctx->part_ev[np], 0));

  // ---- every input copy, in part order ----
  auto h2d = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, cs) : cudaSuccess;
  };
  cudaError_t e = cudaSuccess;
  for (int p = 0, i = 0; p < np && e == cudaSuccess; ++p) {
    for (; i < part_end[p] && e == cudaSuccess; ++i) {
      const gba_query& q = qs[i];
      const size_t n = size_t(q.n_rows);
      e = h2d(const_cast<void*>(dv[i].q.key.data), q.key.data, n * size_t(gba_type_bytes(q.key.type)));
      if (e == cudaSuccess && q.key2.data)
        e = h2d(const_cast<void*>(dv[i].q.key2.data), q.key2.data, n * size_t(gba_type_bytes(q.key2.type)));
      for (int c = 0; c < q.n_cols && e == cudaSuccess; ++c) {
        e = h2d(const_cast<void*>(dv[i].q.cols[c].data), q.cols[c].data, n * size_t(gba_type_bytes(q.cols[c].type)));
        if (e == cudaSuccess && q.cols[c].valid)
          e = h2d(const_cast<uint8_t*>(dv[i].q.cols[c].valid), q.cols[c].valid, (n + 7) / 8);
      }
    }
    if (e == cudaSuccess) e = cudaEventRecord(ctx->part_ev[p], cs);
  }
  if (e != cudaSuccess) {
    drain(ctx, os);
    ctx->err = std::string("host-to-device copies: ") + cudaGetErrorString(e);
    return GBA_ERR_CUDA;
  }

  // ---- parts in order; each part's groups back on the output stream ----
  std::vector<gba_query> pq;
  std::vector<gba_output> po;
  for (int p = 0, first = 0; p < np; first = part_end[p++]) {
    const int cnt = part_end[p] - first;
    e = cudaStreamWaitEvent(s, ctx->part_ev[p], 0);
    if (e != cudaSuccess) break;
    pq.resize(cnt);
    po.resize(cnt);
    for (int j = 0; j < cnt; ++j) {
      pq[j] = dv[first + j].q;
      po[j] = dv[first + j].o;
    }
    st = gba_groupby_batch(ctx, cnt, pq.data(), po.data(), &k, stream, n_groups + first);
    if (st != GBA_OK) {
      drain(ctx, os);
      return st;
    }
    // the part's results are complete (the batch call synchronised `s`)
    for (int j = first; j < part_end[p] && e == cudaSuccess; ++j) {
      const gba_query& q = qs[j];
      const gba_output& o = outs[j];
      const size_t g = size_t(std::max<int64_t>(n_groups[j], 0));
      if (!g) continue;
      e = cudaMemcpyAsync(o.keys, dv[j].o.keys, g * size_t(gba_type_bytes(q.key.type)), cudaMemcpyDeviceToHost, os);
      if (e == cudaSuccess && o.keys2)
        e = cudaMemcpyAsync(o.keys2, dv[j].o.keys2, g * size_t(gba_type_bytes(q.key2.type)), cudaMemcpyDeviceToHost,
                            os);
      for (int a = 0; a < q.n_aggs && e == cudaSuccess; ++a) {
        e = cudaMemcpyAsync(o.aggs[a], dv[j].o.aggs[a], g * 8, cudaMemcpyDeviceToHost, os);
        if (e == cudaSuccess && o.agg_valid[a])
          e = cudaMemcpyAsync(o.agg_valid[a], dv[j].o.agg_valid[a], g, cudaMemcpyDeviceToHost, os);
      }
    }
    if (e != cudaSuccess) break;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(os);
  drain(ctx, os);
  if (e != cudaSuccess) {
    ctx->err = std::string("host batch: ") + cudaGetErrorString(e);
    return GBA_ERR_CUDA;
  }
  return GBA_OK;
}
