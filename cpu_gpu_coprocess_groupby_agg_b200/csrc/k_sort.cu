// Key-ordered output: a stable least-significant-digit radix sort of a call's
// groups by key, then one gather of the aggregate columns.
//
// The reference leaves each partition's groups in hash-table order
// (groupby_agg_intra_partition.cu:245-276 copies collect_kv_in_ht's output as
// it comes); key order is an option of this library, for callers that join or
// merge the groups downstream.
//
//   k_sort_range    min and max of the order-normalised key (sign bit flipped
//                   for signed keys): only the bits in which keys differ are
//                   sorted, 8 per pass, on (key - min)
//   per pass:
//   k_sort_hist     digit counts of each 4096-key tile, digit-major
//                   ([digit][tile]), so that one exclusive scan (k_scan_excl)
//                   gives every (digit, tile) its output offset
//   k_sort_scatter  each warp ranks its 512 keys in order, 32 at a time
//                   (__match_any_sync peers + per-warp digit counters in shared
//                   memory), the block adds the warps' prefix per digit, and
//                   every key and its group index goes to its place; order
//                   inside a digit is the input order, so the sort is stable
//   k_sort_gather   every aggregate column permuted by the sorted group index
//
// Bytes per group and pass: read the key twice (count, scatter) and the index
// once, write key and index once; the gather reads and writes each aggregate
// word twice (a copy to scratch, then the permuted write back).
#include <algorithm>
#include <cstring>
#include <vector>

#include "gba_internal.cuh"
#include "part_kernels.h"
#include "sort_kernels.h"

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortSteps = 16;                        // 32-key steps per warp
constexpr int kWarpSpan = 32 * kSortSteps;            // a warp's keys in a tile
constexpr int kSortTile = kSortThreads * kSortSteps;  // 4096 keys per block

template <bool K64>
__device__ __forceinline__ unsigned long long load_raw(const void* keys, int64_t i) {
  if (K64) return __ldg(static_cast<const unsigned long long*>(keys) + i);
  return __ldg(static_cast<const unsigned*>(keys) + i);
}

template <bool K64>
__device__ __forceinline__ void store_raw(void* keys, int64_t i, unsigned long long k) {
  if (K64) static_cast<unsigned long long*>(keys)[i] = k;
  else static_cast<unsigned*>(keys)[i] = unsigned(k);
}

__device__ __forceinline__ unsigned digit_of(unsigned long long raw, unsigned long long flip, unsigned long long lo,
                                             int shift) {
  return unsigned(((raw ^ flip) - lo) >> shift) & 255u;
}

template <bool K64>
__global__ void __launch_bounds__(kSortThreads) k_sort_range(const void* keys, int64_t g, unsigned long long flip,
                                                             unsigned long long* lo, unsigned long long* hi) {
  unsigned long long mn = ~0ull, mx = 0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < g; i += int64_t(gridDim.x) * blockDim.x) {
    const unsigned long long k = load_raw<K64>(keys, i) ^ flip;
    mn = k < mn ? k : mn;
    mx = k > mx ? k : mx;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long a = __shfl_xor_sync(~0u, mn, o), b = __shfl_xor_sync(~0u, mx, o);
    mn = a < mn ? a : mn;
    mx = b > mx ? b : mx;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(lo, mn);
    atomicMax(hi, mx);
  }
}

template <bool K64>
__global__ void __launch_bounds__(kSortThreads) k_sort_hist(const void* keys, int64_t g, unsigned long long flip,
                                                            unsigned long long lo, int shift, unsigned* counts,
                                                            int64_t ntiles) {
  __shared__ unsigned cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = int64_t(blockIdx.x) * kSortTile + int64_t(warp) * kWarpSpan + lane;
#pragma unroll 4
  for (int step = 0; step < kSortSteps; ++step) {
    const int64_t i = base + step * 32;
    const unsigned d = i < g ? digit_of(load_raw<K64>(keys, i), flip, lo, shift) : 256u;
    const unsigned peers = __match_any_sync(~0u, d);
    if (d < 256u && lane == __ffs(peers) - 1) atomicAdd(&cnt[d], unsigned(__popc(peers)));
  }
  __syncthreads();
  counts[int64_t(threadIdx.x) * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

template <bool K64>
__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(const void* keys_in, const unsigned* idx_in,
                                                               void* keys_out, unsigned* idx_out, int64_t g,
                                                               unsigned long long flip, unsigned long long lo,
                                                               int shift, const unsigned long long* offsets,
                                                               int64_t ntiles) {
  __shared__ unsigned wcnt[kSortWarps][256];
  __shared__ unsigned long long dbase[256];
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) wcnt[w][threadIdx.x] = 0;
  dbase[threadIdx.x] = offsets[int64_t(threadIdx.x) * ntiles + blockIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t base = int64_t(blockIdx.x) * kSortTile + int64_t(warp) * kWarpSpan + lane;
  unsigned long long key[kSortSteps];
  unsigned idx[kSortSteps], rank[kSortSteps];
#pragma unroll
  for (int step = 0; step < kSortSteps; ++step) {
    const int64_t i = base + step * 32;
    const bool ok = i < g;
    key[step] = ok ? load_raw<K64>(keys_in, i) : 0ull;
    idx[step] = ok ? (idx_in ? __ldg(idx_in + i) : unsigned(i)) : 0u;
  }
#pragma unroll
  for (int step = 0; step < kSortSteps; ++step) {
    const bool ok = base + step * 32 < g;
    const unsigned d = ok ? digit_of(key[step], flip, lo, shift) : 256u;
    const unsigned peers = __match_any_sync(~0u, d);
    const unsigned before = ok ? wcnt[warp][d] : 0u;
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) wcnt[warp][d] = before + unsigned(__popc(peers));
    __syncwarp();
    rank[step] = before + unsigned(__popc(peers & lt));
  }
  __syncthreads();
  {
    unsigned run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const unsigned c = wcnt[w][threadIdx.x];
      wcnt[w][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int step = 0; step < kSortSteps; ++step) {
    if (base + step * 32 >= g) continue;
    const unsigned d = digit_of(key[step], flip, lo, shift);
    const int64_t pos = int64_t(dbase[d]) + wcnt[warp][d] + rank[step];
    store_raw<K64>(keys_out, pos, key[step]);
    idx_out[pos] = idx[step];
  }
}

struct GatherCols {
  const unsigned long long* src[GBA_MAX_AGGS];
  unsigned long long* dst[GBA_MAX_AGGS];
  int n;
};

__global__ void __launch_bounds__(kSortThreads) k_sort_gather(GatherCols c, const unsigned* idx, int64_t g) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < g; i += int64_t(gridDim.x) * blockDim.x) {
    const unsigned j = __ldg(idx + i);
#pragma unroll
    for (int a = 0; a < GBA_MAX_AGGS; ++a)
      if (a < c.n) c.dst[a][i] = __ldg(c.src[a] + j);
  }
}

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

struct SortLayout {
  size_t keys_alt, idx0, idx1, counts, offsets, status, tile_ctr, aggs, bytes;
};

SortLayout layout_for(const SortJob& j, size_t base) {
  const int64_t ntiles = (j.g + kSortTile - 1) / kSortTile;
  const size_t entries = size_t(ntiles) * 256;
  SortLayout L;
  size_t o = base;
  L.keys_alt = o;  o += a256(size_t(j.g) * (j.key64 ? 8 : 4));
  L.idx0 = o;      o += a256(size_t(j.g) * 4);
  L.idx1 = o;      o += a256(size_t(j.g) * 4);
  L.counts = o;    o += a256(entries * 4);
  L.offsets = o;   o += a256(entries * 8);
  L.status = o;    o += a256((entries / 1024 + 2) * 8);  // look-back scan: one word per scan tile (>= 1024 entries)
  L.tile_ctr = o;  o += 256;
  L.aggs = o;      o += a256(size_t(j.g) * 8) * size_t(j.nagg);
  L.bytes = o - base;
  return L;
}

}  // namespace

gba_status gba_sort_groups(gba_context* ctx, const SortJob* jobs, int njobs, cudaStream_t s) {
  std::vector<int> todo;
  size_t per_job = 0;
  for (int j = 0; j < njobs; ++j) {
    if (jobs[j].g <= 1) continue;
    if (jobs[j].g >= (int64_t(1) << 32)) {
      ctx->err = "sort_output: more than 2^32 - 1 groups";
      return GBA_ERR_INVALID_ARG;
    }
    todo.push_back(j);
    per_job = std::max(per_job, layout_for(jobs[j], 0).bytes);
  }
  if (todo.empty()) return GBA_OK;
  const size_t nt = todo.size();
  const size_t ranges = a256(nt * 16);
  gba_status st = gba_ws_reserve(ctx, ranges + per_job, s);
  if (st != GBA_OK) return st;
  st = gba_small_reserve(ctx, std::max<size_t>(ctx->d_small_bytes, 64 + nt * 16));
  if (st != GBA_OK) return st;
  unsigned char* W = static_cast<unsigned char*>(ctx->ws);
  unsigned long long* d_lo = reinterpret_cast<unsigned long long*>(W);
  unsigned long long* d_hi = d_lo + nt;
  unsigned* d_flags = reinterpret_cast<unsigned*>(ctx->d_small);
  GBA_CUDA_TRY(ctx, cudaMemsetAsync(d_lo, 0xff, nt * 8, s));
  GBA_CUDA_TRY(ctx, cudaMemsetAsync(d_hi, 0, nt * 8, s));
  GBA_CUDA_TRY(ctx, cudaMemsetAsync(d_flags, 0, 4, s));
  int launches = 0;
  for (size_t t = 0; t < nt; ++t) {
    const SortJob& j = jobs[todo[t]];
    const unsigned long long flip = j.key_signed ? (j.key64 ? 1ull << 63 : 1ull << 31) : 0ull;
    const int grid = int(std::min<int64_t>(int64_t(ctx->sms) * 4, (j.g + kSortThreads - 1) / kSortThreads));
    if (j.key64) k_sort_range<true><<<grid, kSortThreads, 0, s>>>(j.keys, j.g, flip, d_lo + t, d_hi + t);
    else k_sort_range<false><<<grid, kSortThreads, 0, s>>>(j.keys, j.g, flip, d_lo + t, d_hi + t);
    GBA_CUDA_TRY(ctx, cudaGetLastError());
    ++launches;
  }
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_small + 64, d_lo, nt * 16, cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  std::vector<unsigned long long> lo(nt), hi(nt);
  std::memcpy(lo.data(), ctx->h_small + 64, nt * 8);
  std::memcpy(hi.data(), ctx->h_small + 64 + nt * 8, nt * 8);

  for (size_t t = 0; t < nt; ++t) {
    const SortJob& j = jobs[todo[t]];
    const unsigned long long span = hi[t] - lo[t];
    const int bits = span ? 64 - __builtin_clzll(span) : 0;
    const int passes = (bits + 7) / 8;
    if (passes == 0) continue;
    const unsigned long long flip = j.key_signed ? (j.key64 ? 1ull << 63 : 1ull << 31) : 0ull;
    const SortLayout L = layout_for(j, ranges);
    const int64_t ntiles = (j.g + kSortTile - 1) / kSortTile;
    void* alt = W + L.keys_alt;
    unsigned* idxb[2] = {reinterpret_cast<unsigned*>(W + L.idx0), reinterpret_cast<unsigned*>(W + L.idx1)};
    unsigned* counts = reinterpret_cast<unsigned*>(W + L.counts);
    unsigned long long* offsets = reinterpret_cast<unsigned long long*>(W + L.offsets);
    void* cur = j.keys;
    const unsigned* idx_cur = nullptr;
    for (int p = 0; p < passes; ++p) {
      const int shift = 8 * p;
      void* out = cur == j.keys ? alt : j.keys;
      unsigned* idx_out = idxb[p & 1];
      if (j.key64) k_sort_hist<true><<<unsigned(ntiles), kSortThreads, 0, s>>>(cur, j.g, flip, lo[t], shift, counts, ntiles);
      else k_sort_hist<false><<<unsigned(ntiles), kSortThreads, 0, s>>>(cur, j.g, flip, lo[t], shift, counts, ntiles);
      GBA_CUDA_TRY(ctx, cudaGetLastError());
      GBA_CUDA_TRY(ctx, gba_launch_scan_excl(counts, offsets, ntiles * 256,
                                             reinterpret_cast<unsigned long long*>(W + L.status),
                                             reinterpret_cast<unsigned*>(W + L.tile_ctr), d_flags, s));
      if (j.key64)
        k_sort_scatter<true><<<unsigned(ntiles), kSortThreads, 0, s>>>(cur, idx_cur, out, idx_out, j.g, flip, lo[t],
                                                                       shift, offsets, ntiles);
      else
        k_sort_scatter<false><<<unsigned(ntiles), kSortThreads, 0, s>>>(cur, idx_cur, out, idx_out, j.g, flip,
                                                                        lo[t], shift, offsets, ntiles);
      GBA_CUDA_TRY(ctx, cudaGetLastError());
      launches += 3;
      cur = out;
      idx_cur = idx_out;
    }
    if (cur != j.keys)
      GBA_CUDA_TRY(ctx, cudaMemcpyAsync(j.keys, cur, size_t(j.g) * (j.key64 ? 8 : 4), cudaMemcpyDeviceToDevice, s));
    if (j.nagg > 0) {
      GatherCols c{};
      c.n = j.nagg;
      for (int a = 0; a < j.nagg; ++a) {
        unsigned long long* tmp = reinterpret_cast<unsigned long long*>(W + L.aggs + size_t(a) * a256(size_t(j.g) * 8));
        GBA_CUDA_TRY(ctx, cudaMemcpyAsync(tmp, j.aggs[a], size_t(j.g) * 8, cudaMemcpyDeviceToDevice, s));
        c.src[a] = tmp;
        c.dst[a] = j.aggs[a];
      }
      const int grid = int(std::min<int64_t>(int64_t(ctx->sms) * 8, (j.g + kSortThreads - 1) / kSortThreads));
      k_sort_gather<<<grid, kSortThreads, 0, s>>>(c, idx_cur, j.g);
      GBA_CUDA_TRY(ctx, cudaGetLastError());
      ++launches;
    }
  }
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_small, d_flags, 4, cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  ctx->stats.kernel_launches += launches;
  if (*reinterpret_cast<unsigned*>(ctx->h_small) & GBA_FLAG_WAIT_TIMEOUT) {
    ctx->err = "sort_output: a bounded scan wait timed out";
    return GBA_ERR_TIMEOUT;
  }
  return GBA_OK;
}
