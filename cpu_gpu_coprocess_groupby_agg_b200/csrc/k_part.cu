// Radix hash partitioning + intra-partition aggregation (sm_100a).
//
// Replaces the reference's partitioner and phase 2:
//   * cal_kv_intra_group_ind / kv_inter_group_insert (kernel.cu:189-291) -
//     per-block shared histogram of murmur(k) % P, global atomicAdd block
//     offsets, CUB exclusive scan, unstaged 8-byte scatter;
//   * groupby_agg_and_statistic_kernel / device_reduce_kernel /
//     collect_kv_in_ht (kernel.cu:294-406) - per merged partition, a global
//     linear-probe table, a block counter tree-reduce and a CUB scan +
//     compaction, driven from host threads with a sync per chunk
//     (groupby_agg_intra_partition.cu:159-279).
// Here:
//   k_part_hist     per-chunk histogram of the next `bits` hash bits (MSD),
//                   chunks never straddle an input segment
//   k_scan_excl     single-pass decoupled-lookback exclusive scan (in place of
//                   CUB), bounded waits
//   k_part_scatter  per tile: counting sort in shared memory by digit, then
//                   each warp writes runs of equal digits contiguously
//                   (write-combined, coalesced stores)
//   k_part_agg      one CTA per final partition at a time (dynamic queue):
//                   shared-memory table with 32-bit atomics where exact,
//                   rows whose key cannot enter the table go to an HBM
//                   fallback table; groups are written straight to the output
#include "gba_internal.cuh"
#include "part_kernels.h"
#include "smem_table.cuh"

namespace {

// width of a column in the partition passes, which see fp64 columns as I64
// (gba_part_host.cu relabels them; the passes only move bytes)
__host__ __device__ inline int col_bytes_t(int t) { return t == GBA_I64 ? 8 : 4; }

// digit of a key for a pass: bits [32 - shift_hi - bits, 32 - shift_hi) of the hash
template <bool K64>
__device__ __forceinline__ unsigned digit_of(uint64_t key, int shift_hi, int bits) {
  const uint32_t h = part_hash(key);
  return (h << shift_hi) >> (32 - bits);
}

template <bool K64>
__global__ void __launch_bounds__(512) k_part_hist(PartPass p) {
  extern __shared__ unsigned hist[];
  const int nb = 1 << p.bits;
  for (int c = blockIdx.x; c < p.nchunks; c += gridDim.x) {
    const PartChunk ch = p.chunks[c];
    for (int i = threadIdx.x; i < nb; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (int64_t r = ch.row_begin + threadIdx.x; r < ch.row_end; r += blockDim.x) {
      const uint64_t k = K64 ? static_cast<const unsigned long long*>(p.in.keys)[r]
                             : static_cast<const unsigned*>(p.in.keys)[r];
      atomicAdd(&hist[digit_of<K64>(k, p.shift_hi, p.bits)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < nb; d += blockDim.x)
      p.counts[ch.count_base + int64_t(d) * ch.seg_nchunks + ch.chunk_in_seg] = hist[d];
    __syncthreads();
  }
}

// ---- decoupled-lookback exclusive scan over u64 ---------------------------------
constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr unsigned long long kFlagA = 1ull << 62, kFlagP = 2ull << 62, kValMask = (1ull << 62) - 1;

__device__ __forceinline__ unsigned long long block_excl_scan(unsigned long long v, unsigned long long* total) {
  __shared__ unsigned long long warp_sums[32];
  const unsigned lane = lane_id(), w = threadIdx.x >> 5;
  unsigned long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long y = __shfl_up_sync(GBA_FULL_MASK, x, o);
    if (lane >= unsigned(o)) x += y;
  }
  if (lane == 31) warp_sums[w] = x;
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    unsigned long long s = lane < unsigned(nw) ? warp_sums[lane] : 0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long y = __shfl_up_sync(GBA_FULL_MASK, s, o);
      if (lane >= unsigned(o)) s += y;
    }
    if (lane < unsigned(nw)) warp_sums[lane] = s;
  }
  __syncthreads();
  const unsigned long long before = (w ? warp_sums[w - 1] : 0ull) + x - v;
  *total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_excl(const unsigned* in, unsigned long long* out, int64_t n,
                                                            unsigned long long* status, unsigned* tile_ctr,
                                                            unsigned* flags) {
  __shared__ unsigned s_tile;
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t base = tile * kScanTile + int64_t(threadIdx.x) * kScanItems;
  unsigned long long v[kScanItems], sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = base + i < n ? in[base + i] : 0u;
    sum += v[i];
  }
  unsigned long long agg;
  const unsigned long long before = block_excl_scan(sum, &agg);
  if (threadIdx.x == 0) {
    unsigned long long prefix = 0;
    if (tile == 0) {
      atomicExch(&status[0], kFlagP | agg);
    } else {
      atomicExch(&status[tile], kFlagA | agg);
      int64_t j = tile - 1;
      unsigned spins = 0;
      while (j >= 0) {
        const unsigned long long s = *(volatile unsigned long long*)&status[j];
        if ((s & ~kValMask) == 0ull) {
          if (++spins > (1u << 24)) {
            atomicOr(flags, GBA_FLAG_WAIT_TIMEOUT);
            break;
          }
          continue;
        }
        prefix += s & kValMask;
        if ((s & ~kValMask) == kFlagP) break;
        --j;
      }
      atomicExch(&status[tile], kFlagP | (prefix + agg));
    }
    s_prefix = prefix;
  }
  __syncthreads();
  unsigned long long run = s_prefix + before;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = run;
    run += v[i];
  }
}

// ---- staged scatter ---------------------------------------------------------------
// shared layout: cursor[nb] (u64), lhist[nb] (u32), loff[nb] (u32), digits[T] (u16),
// staged rows: keys[T] then one array per column [T]
// NC: value columns (compile time, so only their registers exist)
template <bool K64, int NC>
__global__ void __launch_bounds__(512, 2) k_part_scatter(PartPass p, int T) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int nb = 1 << p.bits;
  unsigned long long* cursor = reinterpret_cast<unsigned long long*>(sm);
  unsigned* lhist = reinterpret_cast<unsigned*>(cursor + nb);
  unsigned* loff = lhist + nb;
  unsigned short* dig = reinterpret_cast<unsigned short*>(loff + nb);
  unsigned char* stg = reinterpret_cast<unsigned char*>(dig + T);
  stg = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(stg) + 15) & ~uintptr_t(15));
  const int kb = K64 ? 8 : 4;
  unsigned char* scol[GBA_MAX_COLS];
  {
    unsigned char* o = stg + size_t(T) * kb;
#pragma unroll
    for (int c = 0; c < GBA_MAX_COLS; ++c) {
      scol[c] = o;
      if (c < p.in.ncols) o += size_t(T) * col_bytes_t(p.in.col_type[c]);
    }
  }
  __shared__ unsigned long long s_total;

  for (int ci = blockIdx.x; ci < p.nchunks; ci += gridDim.x) {
    const PartChunk ch = p.chunks[ci];
    for (int d = threadIdx.x; d < nb; d += blockDim.x)
      cursor[d] = p.offsets[ch.count_base + int64_t(d) * ch.seg_nchunks + ch.chunk_in_seg];
    for (int64_t t0 = ch.row_begin; t0 < ch.row_end; t0 += T) {
      const int rows = int(ch.row_end - t0 < T ? ch.row_end - t0 : T);
      for (int d = threadIdx.x; d < nb; d += blockDim.x) lhist[d] = 0;
      __syncthreads();
      // pass A: every row's key and values into registers (all loads of the
      // tile issued together), its digit, and its rank among the tile's rows
      // of that digit
      constexpr int kMaxRpt = 4;  // T <= 4 * 512
      unsigned rank[kMaxRpt];
      unsigned short dg[kMaxRpt];
      uint64_t kreg[kMaxRpt];
      unsigned long long vreg[kMaxRpt][NC > 0 ? NC : 1];
#pragma unroll
      for (int i = 0; i < kMaxRpt; ++i) {
        const int j = i * blockDim.x + threadIdx.x;
        if (j < rows) {
          kreg[i] = K64 ? __ldcs(static_cast<const unsigned long long*>(p.in.keys) + t0 + j)
                        : __ldcs(static_cast<const unsigned*>(p.in.keys) + t0 + j);
#pragma unroll
          for (int c = 0; c < NC; ++c)
              vreg[i][c] = col_bytes_t(p.in.col_type[c]) == 8
                               ? __ldcs(static_cast<const unsigned long long*>(p.in.cols[c]) + t0 + j)
                               : __ldcs(static_cast<const unsigned*>(p.in.cols[c]) + t0 + j);
        }
      }
#pragma unroll
      for (int i = 0; i < kMaxRpt; ++i) {
        const int j = i * blockDim.x + threadIdx.x;
        if (j < rows) {
          dg[i] = (unsigned short)digit_of<K64>(kreg[i], p.shift_hi, p.bits);
          rank[i] = atomicAdd(&lhist[dg[i]], 1u);
        }
      }
      __syncthreads();
      // local exclusive offsets over nb digits (nb <= 4 * blockDim)
      {
        unsigned long long loc = 0;
        const int per = (nb + blockDim.x - 1) / blockDim.x;
        unsigned vals[4] = {0, 0, 0, 0};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int d = threadIdx.x * per + i;
          if (i < per && d < nb) {
            vals[i] = lhist[d];
            loc += vals[i];
          }
        }
        unsigned long long tot;
        unsigned long long run = block_excl_scan(loc, &tot);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int d = threadIdx.x * per + i;
          if (i < per && d < nb) {
            loff[d] = unsigned(run);
            run += vals[i];
          }
        }
      }
      __syncthreads();
      // pass B: stage rows in digit order
#pragma unroll
      for (int i = 0; i < kMaxRpt; ++i) {
        const int j = i * blockDim.x + threadIdx.x;
        if (j < rows) {
          const unsigned pos = loff[dg[i]] + rank[i];
          dig[pos] = dg[i];
          if (K64) reinterpret_cast<unsigned long long*>(stg)[pos] = kreg[i];
          else reinterpret_cast<unsigned*>(stg)[pos] = unsigned(kreg[i]);
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            if (col_bytes_t(p.in.col_type[c]) == 8)
              reinterpret_cast<unsigned long long*>(scol[c])[pos] = vreg[i][c];
            else
              reinterpret_cast<unsigned*>(scol[c])[pos] = unsigned(vreg[i][c]);
          }
        }
      }
      __syncthreads();
      // pass C: consecutive threads write consecutive staged rows; equal digits
      // are contiguous, so each run lands in one contiguous output range
      for (int j = threadIdx.x; j < rows; j += blockDim.x) {
        const unsigned d = dig[j];
        const unsigned long long dst = cursor[d] + (j - loff[d]);
        // QDesc carries const pointers; the pass's output buffers are writable
        if (K64)
          static_cast<unsigned long long*>(const_cast<void*>(p.out.keys))[dst] =
              reinterpret_cast<unsigned long long*>(stg)[j];
        else
          static_cast<unsigned*>(const_cast<void*>(p.out.keys))[dst] = reinterpret_cast<unsigned*>(stg)[j];
#pragma unroll
        for (int c = 0; c < GBA_MAX_COLS; ++c) {
          if (c < p.in.ncols) {
            void* oc = const_cast<void*>(p.out.cols[c]);
            if (col_bytes_t(p.in.col_type[c]) == 8)
              static_cast<unsigned long long*>(oc)[dst] = reinterpret_cast<unsigned long long*>(scol[c])[j];
            else
              static_cast<unsigned*>(oc)[dst] = reinterpret_cast<unsigned*>(scol[c])[j];
          }
        }
      }
      __syncthreads();
      for (int d = threadIdx.x; d < nb; d += blockDim.x) cursor[d] += lhist[d];
      __syncthreads();
    }
  }
  (void)s_total;
}

// ---- per-partition aggregation ------------------------------------------------------
template <bool K64, typename Sig>
__global__ void __launch_bounds__(1024, 1) k_part_agg(PartAgg a) {
  extern __shared__ __align__(16) unsigned char sm[];
  const QDesc& q = a.rows;
  __shared__ int s_item;
  __shared__ unsigned long long s_base;
  const uint64_t emptyk = K64 ? EMPTY64 : uint64_t(EMPTY32);
  for (;;) {
    if (threadIdx.x == 0) s_item = int(atomicAdd(a.seg_ctr, 1u));
    __syncthreads();
    const int item = s_item;
    if (item >= a.nwork) break;
    const PartWork w = a.work[item];
    for (int seg = w.seg_lo; seg < w.seg_hi; ++seg) {
      const int64_t b = w.partial ? w.row_begin : a.seg_begin[seg];
      const int64_t e = w.partial ? w.row_end : a.seg_begin[seg + 1];
      if (e <= b) continue;  // CTA-uniform
      // a partition never holds more groups than rows: size the table to the
      // rows (load <= 0.7) when that is smaller than the shared budget
      const int64_t want = (e - b) * 10 / 7 + 32;
      const SmemTable<K64> st = smem_table_carve<K64>(sm, int(want < a.S ? want : a.S), q.nwords);
      smem_table_init<K64, Sig>(st, q);
      __syncthreads();
      // a partition with many more rows than table slots repeats keys heavily
      // (skew): pre-combine equal keys inside each warp there
      const bool coal = a.coalesce || (e - b) > 4 * int64_t(a.S);
      constexpr int kIlp = 2;  // rows loaded per thread before any is processed (x 1024 threads)
      for (int64_t r0 = b; r0 < e; r0 += int64_t(kIlp) * blockDim.x) {
        uint64_t keys[kIlp];
        unsigned long long raw[kIlp][GBA_MAX_COLS];
#pragma unroll
        for (int u = 0; u < kIlp; ++u) {
          const int64_t r = r0 + int64_t(u) * blockDim.x + threadIdx.x;
          keys[u] = emptyk;
#pragma unroll
          for (int c = 0; c < GBA_MAX_COLS; ++c) raw[u][c] = 0ull;
          if (r < e) {
            keys[u] = K64 ? __ldg(static_cast<const unsigned long long*>(q.keys) + r)
                          : __ldg(static_cast<const unsigned*>(q.keys) + r);
#pragma unroll
            for (int c = 0; c < GBA_MAX_COLS; ++c)
              if (c < Sig::ncols(q))
                raw[u][c] = gba_type_bytes(Sig::coltype(q, c)) == 8
                                ? __ldg(static_cast<const unsigned long long*>(q.cols[c]) + r)
                                : __ldg(static_cast<const unsigned*>(q.cols[c]) + r);
          }
        }
#pragma unroll
        for (int u = 0; u < kIlp; ++u) {
          const int64_t r = r0 + int64_t(u) * blockDim.x + threadIdx.x;
          const bool valid = r < e;
          uint64_t key = keys[u];
          unsigned long long rr[GBA_MAX_COLS];
#pragma unroll
          for (int c = 0; c < GBA_MAX_COLS; ++c) rr[c] = raw[u][c];
          unsigned long long v[Sig::NA];
          row_contrib<Sig>(q, rr, v);
          const bool sent = valid && key == emptyk;
          if (sent) smem_apply_side<K64, Sig>(st, q, v);
          bool leader = valid && !sent;
          if (coal) {  // CTA-uniform, so every lane of the warp is here
            if (!leader) key = emptyk;
            leader = warp_coalesce<K64, Sig>(q, leader, key, v);
          }
          if (leader) {
            const uint32_t h = table_hash(key);
            const int slot = smem_find_or_insert<K64>(st, key, h, a.sprobe);
            if (slot >= 0) smem_apply<K64, Sig>(st, q, slot, v);
            else {
              gtable_insert<K64, Sig>(a.fallback, q, key, h, v, a.flags);
              atomicOr(a.flags, GBA_FLAG_PART_OVERFLOW);
            }
          }
        }
      }
      __syncthreads();
      if (w.partial) {
        // a piece of a split partition: its keys recur in the other pieces, so
        // its groups are merged in the HBM table and emitted from there
        smem_flush_to_gtable<K64, Sig>(q, a.fallback, st, a.flags);
        __syncthreads();
        continue;
      }
      // emit the segment's groups: block-wide compaction of occupied slots
      const int S = st.S;
      unsigned mine = 0;
      for (int i = threadIdx.x; i < S; i += blockDim.x) mine += st.keys[i] != smem_empty_key<K64>();
      unsigned long long tot;
      unsigned long long before = block_excl_scan(mine, &tot);
      const bool side = *st.side_present() != 0u;
      if (threadIdx.x == 0) s_base = atomicAdd(a.out.count, tot + (side ? 1ull : 0ull));
      __syncthreads();
      unsigned long long pos = s_base + before;
      for (int i = threadIdx.x; i < S; i += blockDim.x) {
        const uint64_t k = st.keys[i];
        if (k == uint64_t(smem_empty_key<K64>())) continue;
        if (pos < (unsigned long long)a.out.capacity) {
          if (K64) static_cast<unsigned long long*>(a.out.keys)[pos] = k;
          else static_cast<unsigned*>(a.out.keys)[pos] = unsigned(k);
#pragma unroll
          for (int x = 0; x < Sig::NA; ++x) a.out.accs[x][pos] = smem_acc_read<K64, Sig>(st, q, x, i);
        }
        ++pos;
      }
      if (side && threadIdx.x == 0) {
        const unsigned long long sp = s_base + tot;
        if (sp < (unsigned long long)a.out.capacity) {
          if (K64) static_cast<unsigned long long*>(a.out.keys)[sp] = EMPTY64;
          else static_cast<unsigned*>(a.out.keys)[sp] = EMPTY32;
#pragma unroll
          for (int x = 0; x < Sig::NA; ++x) a.out.accs[x][sp] = smem_acc_read<K64, Sig>(st, q, x, -1);
        }
      }
      __syncthreads();
    }  // segments of the item
  }
}

__global__ void k_seg_begins(const unsigned long long* offsets, const long long* count_base,
                             const int* seg_nchunks, int nseg_in, int bits, int64_t total, long long* seg_begin) {
  const int nb = 1 << bits;
  const int64_t m = int64_t(nseg_in) * nb;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i <= m; i += int64_t(gridDim.x) * blockDim.x) {
    if (i == m) {
      seg_begin[m] = total;
    } else {
      const int s = int(i / nb), d = int(i % nb);
      seg_begin[i] = (long long)offsets[count_base[s] + int64_t(d) * seg_nchunks[s]];
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
cudaError_t gba_launch_seg_begins(const unsigned long long* offsets, const long long* count_base,
                                  const int* seg_nchunks, int nseg_in, int bits, int64_t total,
                                  long long* seg_begin, cudaStream_t s) {
  const int64_t m = int64_t(nseg_in) << bits;
  const int grid = int((m + 256) / 256 < 4096 ? (m + 256) / 256 : 4096);
  k_seg_begins<<<grid, 256, 0, s>>>(offsets, count_base, seg_nchunks, nseg_in, bits, total, seg_begin);
  return cudaGetLastError();
}

size_t gba_part_scatter_smem(const QDesc& q, int bits, int T) {
  const size_t nb = size_t(1) << bits;
  size_t b = nb * 8 + nb * 4 * 2 + size_t(T) * 2 + 16;
  b += size_t(T) * (q.key64 ? 8 : 4);
  for (int c = 0; c < q.ncols; ++c) b += size_t(T) * col_bytes_t(q.col_type[c]);
  return b + 64;
}

cudaError_t gba_launch_part_hist(const PartPass& p, int grid, cudaStream_t s) {
  const size_t smem = (size_t(1) << p.bits) * 4;
  if (p.in.key64) k_part_hist<true><<<grid, 512, smem, s>>>(p);
  else k_part_hist<false><<<grid, 512, smem, s>>>(p);
  return cudaGetLastError();
}

cudaError_t gba_launch_scan_excl(const unsigned* in, unsigned long long* out, int64_t n,
                                 unsigned long long* status, unsigned* tile_ctr, unsigned* flags, cudaStream_t s) {
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(status, 0, size_t(tiles) * 8, s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(tile_ctr, 0, 4, s);
  if (e != cudaSuccess) return e;
  k_scan_excl<<<unsigned(tiles), kScanThreads, 0, s>>>(in, out, n, status, tile_ctr, flags);
  return cudaGetLastError();
}

cudaError_t gba_launch_part_scatter(const PartPass& p, int grid, int T, cudaStream_t s) {
  const size_t smem = gba_part_scatter_smem(p.in, p.bits, T);
  auto go = [&](auto kernel) -> cudaError_t {
    cudaError_t e = gba_allow_max_smem(kernel);
    if (e != cudaSuccess) return e;
    kernel<<<grid, 512, smem, s>>>(p, T);
    return cudaGetLastError();
  };
  const bool k64 = p.in.key64 != 0;
  switch (p.in.ncols) {
    case 0: return k64 ? go(k_part_scatter<true, 0>) : go(k_part_scatter<false, 0>);
    case 1: return k64 ? go(k_part_scatter<true, 1>) : go(k_part_scatter<false, 1>);
    case 2: return k64 ? go(k_part_scatter<true, 2>) : go(k_part_scatter<false, 2>);
    case 3: return k64 ? go(k_part_scatter<true, 3>) : go(k_part_scatter<false, 3>);
    case 4: return k64 ? go(k_part_scatter<true, 4>) : go(k_part_scatter<false, 4>);
  }
  return cudaErrorInvalidValue;
}

cudaError_t gba_launch_part_agg(const PartAgg& a, int grid, cudaStream_t s) {
  const size_t smem = smem_table_bytes(a.S, a.rows.key64, a.rows.nwords) + 64;
  return gba_dispatch_sig(a.rows, [&](auto K, auto sig) -> cudaError_t {
    constexpr bool k64 = decltype(K)::value;
    using Sig = decltype(sig);
    cudaError_t e = gba_allow_max_smem(k_part_agg<k64, Sig>);
    if (e != cudaSuccess) return e;
    k_part_agg<k64, Sig><<<grid, 1024, smem, s>>>(a);
    return cudaGetLastError();
  });
}
