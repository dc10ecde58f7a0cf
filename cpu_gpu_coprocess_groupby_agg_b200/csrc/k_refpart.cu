// Reference-layout partitioning of one tile's groups (sm_100a), used by the
// drop-in entry points groupby_agg_partition / groupby_agg_intra_partition.
//
// The reference places every group of a tile in partition
// murmur3_32(key, seed 0) % P (tiled_groupby_agg_partition/src/kernel.cu:189-291:
// cal_kv_intra_group_ind ranks each key inside its block's partition histogram,
// a CUB scan gives the partition starts, kv_inter_group_insert scatters).  Here:
//
//   k_rp_hist     per-CTA shared histogram of partition ids, flushed to HBM
//                 with one atomic per (CTA, nonzero partition).
//   k_rp_scan     one CTA: exclusive scan of the P counts -> offsets[P + 1],
//                 and a copy into the scatter cursors.
//   k_rp_scatter  each warp combines the lanes that share a partition
//                 (__match_any_sync), the leader reserves their slots with one
//                 atomic on the partition cursor, and every lane writes its
//                 key and its sum narrowed to u32 (the reference's value type).
// Order inside a partition is unspecified, as in the reference.
#include "gba_internal.cuh"
#include "refpart_kernels.h"

namespace {

__global__ void __launch_bounds__(512) k_rp_hist(const unsigned* __restrict__ keys, int64_t n, unsigned P,
                                                 unsigned* __restrict__ hist) {
  extern __shared__ unsigned sh[];
  for (unsigned i = threadIdx.x; i < P; i += blockDim.x) sh[i] = 0u;
  __syncthreads();
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    atomicAdd(&sh[murmur3_32(__ldg(keys + i), 0u) % P], 1u);
  __syncthreads();
  for (unsigned i = threadIdx.x; i < P; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// one CTA of 1024 threads; P <= GBA_REFPART_MAX_P
__global__ void __launch_bounds__(1024) k_rp_scan(const unsigned* __restrict__ hist, unsigned P,
                                                  unsigned long long* __restrict__ offsets,
                                                  unsigned long long* __restrict__ cursor) {
  __shared__ unsigned long long warp_tot[32];
  const unsigned per = (P + blockDim.x - 1) / blockDim.x;
  const unsigned b = threadIdx.x * per;
  unsigned long long local = 0;
  for (unsigned j = 0; j < per; ++j)
    if (b + j < P) local += hist[b + j];
  // block exclusive scan of the per-thread totals
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  unsigned long long x = local;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned long long y = __shfl_up_sync(GBA_FULL_MASK, x, d);
    if (int(lane) >= d) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    unsigned long long w = lane < (blockDim.x >> 5) ? warp_tot[lane] : 0ull;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned long long y = __shfl_up_sync(GBA_FULL_MASK, w, d);
      if (int(lane) >= d) w += y;
    }
    warp_tot[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  unsigned long long run = x - local + (warp ? warp_tot[warp - 1] : 0ull);
  for (unsigned j = 0; j < per; ++j)
    if (b + j < P) {
      offsets[b + j] = run;
      cursor[b + j] = run;
      run += hist[b + j];
    }
  if (threadIdx.x == blockDim.x - 1) offsets[P] = warp_tot[(blockDim.x >> 5) - 1];
}

__global__ void __launch_bounds__(512) k_rp_scatter(const unsigned* __restrict__ keys,
                                                    const unsigned long long* __restrict__ sums, int64_t n,
                                                    unsigned P, unsigned long long* __restrict__ cursor,
                                                    unsigned* __restrict__ out_keys, unsigned* __restrict__ out_vals) {
  const unsigned lane = lane_id();
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  // whole warps iterate together so that __match_any_sync sees every lane
  for (int64_t base = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) & ~int64_t(31); base < n; base += stride) {
    const int64_t i = base + lane;
    const bool live = i < n;
    unsigned k = 0, pid = 0xffffffffu;
    unsigned v = 0;
    if (live) {
      k = __ldg(keys + i);
      v = unsigned(__ldg(sums + i));  // the reference's u32 sum wraps mod 2^32
      pid = murmur3_32(k, 0u) % P;
    }
    const unsigned peers = __match_any_sync(GBA_FULL_MASK, pid);
    const unsigned leader = __ffs(peers) - 1;
    unsigned long long pos0 = 0;
    if (live && lane == leader) pos0 = atomicAdd(&cursor[pid], (unsigned long long)__popc(peers));
    pos0 = __shfl_sync(GBA_FULL_MASK, pos0, leader);
    if (live) {
      const unsigned long long pos = pos0 + __popc(peers & ((1u << lane) - 1u));
      out_keys[pos] = k;
      out_vals[pos] = v;
    }
  }
}

}  // namespace

cudaError_t gba_launch_refpart(const unsigned* keys, const unsigned long long* sums, int64_t n, int P,
                               unsigned* out_keys, unsigned* out_vals, unsigned* hist, unsigned long long* offsets,
                               unsigned long long* cursor, int sms, cudaStream_t s) {
  if (P < 1 || P > GBA_REFPART_MAX_P) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemsetAsync(hist, 0, size_t(P) * 4, s);
  if (e != cudaSuccess) return e;
  const int64_t want = (n + 2047) / 2048;
  const int grid = int(want < 1 ? 1 : (want > int64_t(sms) * 4 ? int64_t(sms) * 4 : want));
  if (n > 0) {
    if (size_t(P) * 4 > 48 * 1024) {
      e = gba_allow_max_smem(k_rp_hist);
      if (e != cudaSuccess) return e;
    }
    k_rp_hist<<<grid, 512, size_t(P) * 4, s>>>(keys, n, unsigned(P), hist);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  k_rp_scan<<<1, 1024, 0, s>>>(hist, unsigned(P), offsets, cursor);
  e = cudaGetLastError();
  if (e != cudaSuccess || n == 0) return e;
  k_rp_scatter<<<grid, 512, 0, s>>>(keys, sums, n, unsigned(P), cursor, out_keys, out_vals);
  return cudaGetLastError();
}
