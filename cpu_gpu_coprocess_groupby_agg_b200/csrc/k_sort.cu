// Key-ordered output: a stable least-significant-digit radix sort of a call's
// groups by key, then one gather of the aggregate columns.
//
// The reference leaves each partition's groups in hash-table order
// (groupby_agg_intra_partition.cu:245-276 copies collect_kv_in_ht's output as
// it comes); key order is an option of this library, for callers that join or
// merge the groups downstream.
//
// The pass structure is the single-sweep radix sort published by Adinets and
// Merrill ("Onesweep", 2022): one upfront read of the keys counts every digit
// position, and each pass is then one kernel that ranks its tile and finds its
// global offsets by a decoupled look-back over earlier tiles, per digit.
//
//   k_sort_prep     counts of every 8-bit digit of the order-normalised key
//                   (sign bit flipped for signed keys), all positions at once
//   k_sort_mask     per job: the digit positions whose keys do not all share
//                   one digit; only those passes run (one host round trip for
//                   all jobs of a call)
//   k_sort_pass     one per pass: a CTA takes the next 4096-key tile from a
//                   counter, each warp ranks its 512 keys in order, 32 at a
//                   time (peers of equal digit from 8 ballots; their leader adds them
//                   to the warp's digit counter in shared memory), the tile publishes its digit counts and
//                   looks back over earlier tiles for their running totals
//                   (bounded spin; a timeout raises GBA_FLAG_WAIT_TIMEOUT),
//                   the tile is staged in shared memory in digit order and
//                   written out as contiguous runs, one per digit; order inside
//                   a digit is the input order, so the sort is stable
//   k_sort_gather   every aggregate column permuted by the sorted group index
//
// Bytes per group: the key read once up front; per pass the key and its index
// read and written once (the first pass reads no index); the gather reads the
// index and copies each aggregate word to scratch and back through it.
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "gba_internal.cuh"
#include "sort_kernels.h"

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortSteps = 16;                        // 32-key steps per warp
constexpr int kWarpSpan = 32 * kSortSteps;            // a warp's keys in a tile
constexpr int kSortTile = kSortThreads * kSortSteps;  // 4096 keys per tile
constexpr unsigned long long kAggregate = 1ull << 62;  // look-back word: this tile's count
constexpr unsigned long long kPrefix = 2ull << 62;     // look-back word: running total through this tile
constexpr unsigned long long kValue = (1ull << 62) - 1;
constexpr unsigned kSpinLimit = 1u << 24;   // look-back rounds without progress before giving up
constexpr int kLookWindow = 8;              // predecessor tiles read per look-back round

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

__device__ __forceinline__ unsigned digit_of(unsigned long long raw, unsigned long long flip, int shift) {
  return unsigned((raw ^ flip) >> shift) & 255u;
}

// hist[p * 256 + d]: keys whose digit p is d.  A warp whose 32 keys share a
// digit adds 32 once (the common case at the top of a narrow key range).
template <bool K64>
__global__ void __launch_bounds__(kSortThreads) k_sort_prep(const void* keys, int64_t g, unsigned long long flip,
                                                            unsigned* hist) {
  constexpr int P = K64 ? 8 : 4;
  __shared__ unsigned h[P * 256];
  for (int i = threadIdx.x; i < P * 256; i += kSortThreads) h[i] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t stride = int64_t(gridDim.x) * kSortThreads;
  for (int64_t base = int64_t(blockIdx.x) * kSortThreads; base < g; base += stride) {
    const int64_t i = base + threadIdx.x;
    const bool ok = i < g;
    const unsigned long long k = ok ? load_raw<K64>(keys, i) ^ flip : 0ull;
    const unsigned active = __ballot_sync(~0u, ok);
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const unsigned d = unsigned(k >> (8 * p)) & 255u;
      const unsigned d0 = __shfl_sync(~0u, d, 0);  // lane 0 is active whenever any lane is
      if (__all_sync(~0u, !ok || d == d0)) {
        if (lane == 0) atomicAdd(&h[p * 256 + d], unsigned(__popc(active)));
      } else if (ok) {
        atomicAdd(&h[p * 256 + d], 1u);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < P * 256; i += kSortThreads)
    if (h[i]) atomicAdd(&hist[i], h[i]);
}

// mask[j] bit p: pass p of job j moves keys (its digit is not the same for all)
__global__ void __launch_bounds__(kSortThreads) k_sort_mask(const unsigned* hists, const int64_t* gs, int npos,
                                                            unsigned* mask) {
  __shared__ unsigned m;
  if (threadIdx.x == 0) m = 0;
  __syncthreads();
  const unsigned* h = hists + size_t(blockIdx.x) * 8 * 256;
  const unsigned g = unsigned(gs[blockIdx.x]);
  for (int p = 0; p < 8; ++p)
    if (p < npos && h[p * 256 + threadIdx.x] == g) atomicOr(&m, 1u << p);  // one digit holds every key
  __syncthreads();
  if (threadIdx.x == 0) mask[blockIdx.x] = ~m & ((1u << npos) - 1u);
}

// The lanes whose 8-bit digit equals this lane's, among the lanes with ok set:
// one ballot per digit bit (the same mask __match_any_sync gives, from plain
// votes).
__device__ __forceinline__ unsigned digit_peers(unsigned d, bool ok) {
  unsigned m = __ballot_sync(~0u, ok);
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const unsigned v = __ballot_sync(~0u, (d >> b) & 1u);
    m &= (d >> b) & 1u ? v : ~v;
  }
  return m;
}

// exclusive prefix over the block's 256 threads (one value each)
__device__ __forceinline__ unsigned long long block_excl256(unsigned long long v, unsigned long long* warp_tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(~0u, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  unsigned long long before = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w)
    if (w < warp) before += warp_tot[w];
  __syncthreads();
  return before + x - v;
}

struct PassArgs {
  const void* keys_in;
  const unsigned* idx_in;   // null: the key's index is its position (first pass)
  void* keys_out;
  unsigned* idx_out;
  int64_t g;
  unsigned long long flip;
  int shift;
  const unsigned* hist;     // this pass's 256 digit counts over all keys
  unsigned long long* look; // [tile][256] look-back words, zeroed
  unsigned* tile_ctr;       // zeroed
  unsigned* flags;
};

template <bool K64>
__global__ void __launch_bounds__(kSortThreads, 3) k_sort_pass(PassArgs a) {
  using KeyT = typename std::conditional<K64, unsigned long long, unsigned>::type;
  extern __shared__ __align__(16) unsigned char stage[];
  KeyT* skeys = reinterpret_cast<KeyT*>(stage);
  unsigned* sidx = reinterpret_cast<unsigned*>(stage + sizeof(KeyT) * kSortTile);
  __shared__ unsigned wcnt[kSortWarps][256];
  __shared__ unsigned dstart[256];
  __shared__ unsigned long long gbase[256];
  __shared__ unsigned long long warp_tot[kSortWarps];
  __shared__ unsigned s_tile;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) s_tile = atomicAdd(a.tile_ctr, 1u);
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) wcnt[w][t] = 0;
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t tile0 = tile * kSortTile;
  const int tile_n = a.g - tile0 < kSortTile ? int(a.g - tile0) : kSortTile;

  // rank every key among the tile's keys of the same digit, in input order
  const unsigned lt = (1u << lane) - 1u;
  const int64_t base = tile0 + int64_t(warp) * kWarpSpan + lane;
  KeyT key[kSortSteps];
  unsigned idx[kSortSteps], rank[kSortSteps];
#pragma unroll
  for (int step = 0; step < kSortSteps; ++step) {
    const int64_t i = base + step * 32;
    const bool ok = i < a.g;
    key[step] = ok ? KeyT(load_raw<K64>(a.keys_in, i)) : KeyT(0);
    idx[step] = ok ? (a.idx_in ? __ldg(a.idx_in + i) : unsigned(i)) : 0u;
  }
#pragma unroll
  for (int step = 0; step < kSortSteps; ++step) {
    const bool ok = base + step * 32 < a.g;
    const unsigned d = ok ? digit_of(key[step], a.flip, a.shift) : 0u;
    const unsigned peers = digit_peers(d, ok);
    const int leader = __ffs(peers) - 1;
    // the leader's atomic returns the count before this step; steps do not
    // wait on one another (the warp's counter row is touched by it alone)
    unsigned before = 0;
    if (ok && lane == leader) before = atomicAdd(&wcnt[warp][d], unsigned(__popc(peers)));
    before = __shfl_sync(~0u, before, leader);
    rank[step] = before + unsigned(__popc(peers & lt));
  }
  __syncthreads();

  // thread t owns digit t: warp prefix, tile count, publish, look back
  unsigned total = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) {
    const unsigned c = wcnt[w][t];
    wcnt[w][t] = total;
    total += c;
  }
  unsigned long long* look = a.look + size_t(tile) * 256 + t;
  if (tile == 0) atomicExch(look, kPrefix | total);
  else atomicExch(look, kAggregate | total);
  const unsigned long long gstart = block_excl256(a.hist[t], warp_tot);
  dstart[t] = unsigned(block_excl256(total, warp_tot));
  unsigned long long excl = 0;
  if (tile > 0) {
    // walk back kLookWindow tiles per round of independent loads (the tiles of
    // the first wave all publish at once; one dependent load per tile would
    // make their walks serial)
    int64_t j = tile - 1;
    unsigned spins = 0;
    while (true) {
      unsigned long long w[kLookWindow];
#pragma unroll
      for (int u = 0; u < kLookWindow; ++u)
        w[u] = j - u >= 0 ? *reinterpret_cast<const volatile unsigned long long*>(a.look + size_t(j - u) * 256 + t)
                          : kPrefix;  // before tile 0: a running total of zero
      int used = 0;
      bool done = false;
#pragma unroll
      for (int u = 0; u < kLookWindow; ++u) {
        if (done || used < u) continue;        // stopped earlier in this window
        const unsigned long long f = w[u] & ~kValue;
        if (f == 0ull) continue;               // tile j - u has not published yet
        excl += w[u] & kValue;
        done = f == kPrefix;
        used = u + 1;
      }
      if (done) break;
      if (used == 0 && ++spins > kSpinLimit) {
        atomicOr(a.flags, GBA_FLAG_WAIT_TIMEOUT);
        break;
      }
      j -= used;
    }
    atomicExch(look, kPrefix | (excl + total));
  }
  gbase[t] = gstart + excl;
  __syncthreads();

  // stage the tile in digit order, then write each digit's run contiguously
#pragma unroll
  for (int step = 0; step < kSortSteps; ++step) {
    if (base + step * 32 >= a.g) continue;
    const unsigned d = digit_of(key[step], a.flip, a.shift);
    const unsigned pos = dstart[d] + wcnt[warp][d] + rank[step];
    skeys[pos] = KeyT(key[step]);
    sidx[pos] = idx[step];
  }
  __syncthreads();
  for (int i = t; i < tile_n; i += kSortThreads) {
    const unsigned long long k = skeys[i];
    const unsigned d = digit_of(k, a.flip, a.shift);
    const unsigned long long gpos = gbase[d] + unsigned(i - int(dstart[d]));
    if (gpos >= (unsigned long long)a.g) continue;  // only after a timed-out look-back
    store_raw<K64>(a.keys_out, int64_t(gpos), k);
    a.idx_out[gpos] = sidx[i];
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

size_t stage_bytes(bool key64) { return size_t(kSortTile) * ((key64 ? 8 : 4) + 4); }

struct SortLayout {
  size_t keys_alt, idx0, idx1, look, ctr, aggs, bytes;
};

SortLayout layout_for(const SortJob& j, size_t base) {
  const int64_t ntiles = (j.g + kSortTile - 1) / kSortTile;
  SortLayout L;
  size_t o = base;
  L.keys_alt = o;  o += a256(size_t(j.g) * (j.key64 ? 8 : 4));
  L.idx0 = o;      o += a256(size_t(j.g) * 4);
  L.idx1 = o;      o += a256(size_t(j.g) * 4);
  L.look = o;      o += a256(size_t(ntiles) * 256 * 8);
  L.ctr = o;       o += 256;  // one tile counter per pass
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
  const int nt = int(todo.size());
  // front of the workspace: every job's digit counts, group count and pass mask
  const size_t o_hist = 0, o_g = a256(size_t(nt) * 8 * 256 * 4), o_mask = o_g + a256(size_t(nt) * 8);
  const size_t front = o_mask + a256(size_t(nt) * 4);
  gba_status st = gba_ws_reserve(ctx, front + per_job, s);
  if (st != GBA_OK) return st;
  st = gba_small_reserve(ctx, std::max<size_t>(ctx->d_small_bytes, 64 + size_t(nt) * 4));
  if (st != GBA_OK) return st;
  static const cudaError_t smem_ok = [] {
    cudaError_t e = gba_allow_max_smem(k_sort_pass<true>);
    return e != cudaSuccess ? e : gba_allow_max_smem(k_sort_pass<false>);
  }();
  GBA_CUDA_TRY(ctx, smem_ok);
  unsigned char* W = static_cast<unsigned char*>(ctx->ws);
  unsigned* d_hist = reinterpret_cast<unsigned*>(W + o_hist);
  int64_t* d_g = reinterpret_cast<int64_t*>(W + o_g);
  unsigned* d_mask = reinterpret_cast<unsigned*>(W + o_mask);
  unsigned* d_flags = reinterpret_cast<unsigned*>(ctx->d_small);
  std::vector<int64_t> gs(nt);
  for (int t = 0; t < nt; ++t) gs[t] = jobs[todo[t]].g;
  GBA_CUDA_TRY(ctx, cudaMemsetAsync(d_hist, 0, size_t(nt) * 8 * 256 * 4, s));
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(d_g, gs.data(), size_t(nt) * 8, cudaMemcpyHostToDevice, s));
  GBA_CUDA_TRY(ctx, cudaMemsetAsync(d_flags, 0, 4, s));
  int launches = 0;
  bool any64 = false;
  for (int t = 0; t < nt; ++t) {
    const SortJob& j = jobs[todo[t]];
    const unsigned long long flip = j.key_signed ? (j.key64 ? 1ull << 63 : 1ull << 31) : 0ull;
    const int grid = int(std::min<int64_t>(int64_t(ctx->sms) * 4, (j.g + kSortThreads - 1) / kSortThreads));
    if (j.key64) k_sort_prep<true><<<grid, kSortThreads, 0, s>>>(j.keys, j.g, flip, d_hist + size_t(t) * 2048);
    else k_sort_prep<false><<<grid, kSortThreads, 0, s>>>(j.keys, j.g, flip, d_hist + size_t(t) * 2048);
    GBA_CUDA_TRY(ctx, cudaGetLastError());
    any64 = any64 || j.key64;
    ++launches;
  }
  // 32-bit jobs count 4 positions, 64-bit ones 8: the mask kernel is told the
  // larger and a 32-bit job's positions 4..7 hold zero counts (never "all")
  k_sort_mask<<<nt, kSortThreads, 0, s>>>(d_hist, d_g, any64 ? 8 : 4, d_mask);
  GBA_CUDA_TRY(ctx, cudaGetLastError());
  ++launches;
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_small + 64, d_mask, size_t(nt) * 4, cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  std::vector<unsigned> mask(nt);
  std::memcpy(mask.data(), ctx->h_small + 64, size_t(nt) * 4);

  const size_t jb = front;
  for (int t = 0; t < nt; ++t) {
    const SortJob& j = jobs[todo[t]];
    const unsigned m = mask[t] & (j.key64 ? 0xffu : 0xfu);
    if (m == 0) continue;
    const unsigned long long flip = j.key_signed ? (j.key64 ? 1ull << 63 : 1ull << 31) : 0ull;
    const SortLayout L = layout_for(j, jb);
    const int64_t ntiles = (j.g + kSortTile - 1) / kSortTile;
    void* alt = W + L.keys_alt;
    unsigned* idxb[2] = {reinterpret_cast<unsigned*>(W + L.idx0), reinterpret_cast<unsigned*>(W + L.idx1)};
    unsigned* ctr = reinterpret_cast<unsigned*>(W + L.ctr);
    GBA_CUDA_TRY(ctx, cudaMemsetAsync(ctr, 0, 8 * 4, s));
    void* cur = j.keys;
    const unsigned* idx_cur = nullptr;
    int np = 0;
    for (int p = 0; p < 8; ++p) {
      if (!(m >> p & 1u)) continue;
      PassArgs a;
      a.keys_in = cur;
      a.idx_in = idx_cur;
      a.keys_out = cur == j.keys ? alt : j.keys;
      a.idx_out = idxb[np & 1];
      a.g = j.g;
      a.flip = flip;
      a.shift = 8 * p;
      a.hist = d_hist + size_t(t) * 2048 + size_t(p) * 256;
      a.look = reinterpret_cast<unsigned long long*>(W + L.look);
      a.tile_ctr = ctr + p;
      a.flags = d_flags;
      GBA_CUDA_TRY(ctx, cudaMemsetAsync(a.look, 0, size_t(ntiles) * 256 * 8, s));
      if (j.key64) k_sort_pass<true><<<unsigned(ntiles), kSortThreads, stage_bytes(true), s>>>(a);
      else k_sort_pass<false><<<unsigned(ntiles), kSortThreads, stage_bytes(false), s>>>(a);
      GBA_CUDA_TRY(ctx, cudaGetLastError());
      ++launches;
      ++np;
      cur = a.keys_out;
      idx_cur = a.idx_out;
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
    ctx->err = "sort_output: a bounded look-back wait timed out";
    return GBA_ERR_TIMEOUT;
  }
  return GBA_OK;
}
