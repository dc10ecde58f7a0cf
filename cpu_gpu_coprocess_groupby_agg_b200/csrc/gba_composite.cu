// Composite keys: GROUP BY (key, key2) for two 32-bit key columns.
//
// The pair is packed into one 64-bit key that orders like the pair (the sign
// bit of each signed half flipped, first key in the high word), the query runs
// on that key, and the output keys are unpacked into the caller's two key
// columns.  Packing costs one extra pass over the keys (read 8 B, write 8 B per
// row); the aggregation itself is the single-key path.
//
// No reference counterpart: the reference groups by one u32 key
// (tiled_groupby_agg_partition/include/util.cuh:6).
#include <algorithm>
#include <string>

#include "composite.h"

namespace {

__global__ void __launch_bounds__(256) k_pack_keys(const unsigned* k1, const unsigned* k2, unsigned s1, unsigned s2,
                                                   int64_t n, unsigned long long* out) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = (static_cast<unsigned long long>(__ldcs(k1 + i) ^ s1) << 32) | (__ldcs(k2 + i) ^ s2);
}

__global__ void __launch_bounds__(256) k_unpack_keys(const unsigned long long* in, int64_t g, unsigned s1,
                                                     unsigned s2, unsigned* o1, unsigned* o2) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < g; i += int64_t(gridDim.x) * blockDim.x) {
    const unsigned long long k = __ldcs(in + i);
    o1[i] = unsigned(k >> 32) ^ s1;
    o2[i] = unsigned(k) ^ s2;
  }
}

unsigned sign_flip(int type) { return type == GBA_I32 ? 0x80000000u : 0u; }

int grid_for(const gba_context* ctx, int64_t n) {
  return int(std::max<int64_t>(1, std::min<int64_t>(int64_t(ctx->sms) * 8, (n + 255) / 256)));
}

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

gba_status gba_composite_prepare(gba_context* ctx, int nq, const gba_query* qs, const gba_output* outs,
                                 gba_query* q2, gba_output* o2, std::vector<CompositeJob>* jobs, cudaStream_t s) {
  jobs->clear();
  size_t bytes = 0;
  for (int i = 0; i < nq; ++i) {
    const gba_query& q = qs[i];
    if (!q.key2.data) continue;
    const int t1 = q.key.type, t2 = q.key2.type;
    if ((t1 != GBA_I32 && t1 != GBA_U32) || (t2 != GBA_I32 && t2 != GBA_U32)) {
      ctx->err = "query " + std::to_string(i) + ": composite keys take two 32-bit key columns (I32 or U32)";
      return GBA_ERR_UNSUPPORTED;
    }
    if (q.n_rows < 0 || (q.n_rows > 0 && !q.key.data) || outs[i].capacity < 0 ||
        (outs[i].capacity > 0 && (!outs[i].keys || !outs[i].keys2))) {
      ctx->err = "query " + std::to_string(i) + ": composite keys need both key columns and both output key columns";
      return GBA_ERR_INVALID_ARG;
    }
    CompositeJob j;
    j.query = i;
    j.s1 = sign_flip(t1);
    j.s2 = sign_flip(t2);
    j.in_off = bytes;
    bytes += a256(size_t(std::max<int64_t>(q.n_rows, 1)) * 8);
    j.out_off = bytes;
    bytes += a256(size_t(std::max<int64_t>(outs[i].capacity, 1)) * 8);
    jobs->push_back(j);
  }
  if (jobs->empty()) return GBA_OK;
  if (bytes > ctx->ck_bytes) {
    if (ctx->ck_buf) {
      GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
      cudaFree(ctx->ck_buf);
      ctx->ck_buf = nullptr;
      ctx->ck_bytes = 0;
    }
    GBA_CUDA_TRY(ctx, cudaMalloc(&ctx->ck_buf, bytes));
    ctx->ck_bytes = bytes;
  }
  unsigned char* B = static_cast<unsigned char*>(ctx->ck_buf);
  for (const CompositeJob& j : *jobs) {
    const gba_query& q = qs[j.query];
    unsigned long long* packed = reinterpret_cast<unsigned long long*>(B + j.in_off);
    if (q.n_rows > 0) {
      k_pack_keys<<<grid_for(ctx, q.n_rows), 256, 0, s>>>(static_cast<const unsigned*>(q.key.data),
                                                         static_cast<const unsigned*>(q.key2.data), j.s1, j.s2,
                                                         q.n_rows, packed);
      GBA_CUDA_TRY(ctx, cudaGetLastError());
    }
    q2[j.query].key.type = GBA_I64;
    q2[j.query].key.data = packed;
    q2[j.query].key2 = gba_column{};
    o2[j.query].keys = B + j.out_off;
    o2[j.query].keys2 = nullptr;
  }
  return GBA_OK;
}

gba_status gba_composite_finish(gba_context* ctx, const std::vector<CompositeJob>& jobs, const gba_output* outs,
                                const int64_t* n_groups, cudaStream_t s) {
  const unsigned char* B = static_cast<const unsigned char*>(ctx->ck_buf);
  int launches = 0;
  for (const CompositeJob& j : jobs) {
    const int64_t g = std::min<int64_t>(n_groups[j.query], outs[j.query].capacity);
    if (g <= 0) continue;
    k_unpack_keys<<<grid_for(ctx, g), 256, 0, s>>>(reinterpret_cast<const unsigned long long*>(B + j.out_off), g,
                                                   j.s1, j.s2, static_cast<unsigned*>(outs[j.query].keys),
                                                   static_cast<unsigned*>(outs[j.query].keys2));
    GBA_CUDA_TRY(ctx, cudaGetLastError());
    ++launches;
  }
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  ctx->stats.kernel_launches += launches + int64_t(jobs.size());  // the pack launches too
  return GBA_OK;
}
