// Streaming group-by kernel (sm_100a): the aggregation kernel of the table
// strategy for batches of queries (and single queries as a batch of one).
//
// Replaces the reference's per-tile chain (tiled_groupby_agg_partition/src/
// kernel.cu:9-186: a one-probe HBM table, CUB scans, a linear-probe spill
// table) with one persistent launch:
//
//   * A CTA takes (query, row range) items from a device work queue; for each
//     item it sets up a shared-memory open-addressing table sized for that
//     query, and at the end of the item merges it into the query's HBM table.
//   * Inside an item every warp pulls chunks of 32 x R rows on its own (a
//     shared cursor), so no barrier runs while rows stream: a warp's lanes
//     load R rows each with 128-bit (or 64-bit) streaming loads issued
//     together before any row is used (about 4 KB in flight per warp), then
//     update the shared table with 32-bit shared atomics.
//   * Rows whose key is not in the shared table and cannot enter it (table
//     full within the probe cap) go to the HBM table: the lane first issues
//     the home-slot loads of all its missed rows, then finishes each insert,
//     so a warp keeps up to 32 x R independent L2 requests in flight.
//   * Input rows are read with evict-first loads so they do not push the HBM
//     tables out of L2.
#include "batch_kernels.h"
#include "gba_internal.cuh"
#include "smem_table.cuh"

namespace {
#include "stream_rows.cuh"

// rows per lane per chunk: fewer when a row carries many accumulators, and
// half as many when two CTAs share an SM (MINB = 2: half the registers)
template <typename Sig, int MINB>
__host__ __device__ constexpr int stream_rows_per_lane() {
  return (Sig::NA <= 2 ? 8 : (Sig::NA <= 4 ? 4 : 2)) / MINB > 0 ? (Sig::NA <= 2 ? 8 : (Sig::NA <= 4 ? 4 : 2)) / MINB
                                                                 : 1;
}

// V consecutive 4-byte / 8-byte elements starting at p (aligned to V * width)
template <int V>
__device__ __forceinline__ void ld_vec4(const unsigned* p, unsigned long long (&o)[V]) {
  if constexpr (V == 1) {
    o[0] = __ldcs(p);
  } else if constexpr (V == 2) {
    const uint2 a = __ldcs(reinterpret_cast<const uint2*>(p));
    o[0] = a.x;
    o[1] = a.y;
  } else {
    const uint4 a = __ldcs(reinterpret_cast<const uint4*>(p));
    o[0] = a.x;
    o[1] = a.y;
    o[2] = a.z;
    o[3] = a.w;
  }
}
template <int V>
__device__ __forceinline__ void ld_vec8(const unsigned long long* p, unsigned long long (&o)[V]) {
  if constexpr (V == 1) {
    o[0] = __ldcs(p);
  } else {
#pragma unroll
    for (int h = 0; h < V / 2; ++h) {
      const uint4 a = __ldcs(reinterpret_cast<const uint4*>(p) + h);
      o[2 * h] = (unsigned long long)a.y << 32 | a.x;
      o[2 * h + 1] = (unsigned long long)a.w << 32 | a.z;
    }
  }
}

template <bool K64, typename Sig, int R, bool HBM>
__device__ __forceinline__ void stream_chunk(const BatchQ& bq, const SmemTable<K64>& st, int nbk, int64_t c0,
                                             int64_t row_end, bool vec) {
  constexpr int NA = Sig::NA;
  constexpr int V = (16 / (K64 ? 8 : 4)) < R ? (16 / (K64 ? 8 : 4)) : R;  // rows per key vector
  constexpr int U = R / V;
  const QDesc& q = bq.q;
  const unsigned lane = lane_id();
  const uint64_t emptyk = K64 ? EMPTY64 : uint64_t(EMPTY32);
  const bool full = vec && c0 + 32 * R <= row_end;

  uint64_t key[R];
  unsigned long long v[R][NA];
  bool live[R];
  {
    unsigned long long raw[R][GBA_MAX_COLS];
#pragma unroll
    for (int i = 0; i < R; ++i) {
#pragma unroll
      for (int c = 0; c < GBA_MAX_COLS; ++c) raw[i][c] = 0ull;
    }
    if (full) {
      // lane's vector u covers rows c0 + (u * 32 + lane) * V + [0, V)
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t r = c0 + (int64_t(u) * 32 + lane) * V;
        unsigned long long kv[V];
        if constexpr (K64) ld_vec8<V>(static_cast<const unsigned long long*>(q.keys) + r, kv);
        else ld_vec4<V>(static_cast<const unsigned*>(q.keys) + r, kv);
#pragma unroll
        for (int e = 0; e < V; ++e) key[u * V + e] = kv[e];
#pragma unroll
        for (int c = 0; c < GBA_MAX_COLS; ++c) {
          if (c < Sig::ncols(q)) {
            unsigned long long cv[V];
            if (gba_type_bytes(Sig::coltype(q, c)) == 8) ld_vec8<V>(static_cast<const unsigned long long*>(q.cols[c]) + r, cv);
            else ld_vec4<V>(static_cast<const unsigned*>(q.cols[c]) + r, cv);
#pragma unroll
            for (int e = 0; e < V; ++e) raw[u * V + e][c] = cv[e];
          }
        }
      }
#pragma unroll
      for (int i = 0; i < R; ++i) live[i] = true;
    } else {
      // ragged or unaligned chunk: row c0 + i * 32 + lane
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const int64_t r = c0 + int64_t(i) * 32 + lane;
        live[i] = r < row_end;
        key[i] = emptyk;
        if (live[i]) {
          key[i] = K64 ? __ldcs(static_cast<const unsigned long long*>(q.keys) + r)
                       : __ldcs(static_cast<const unsigned*>(q.keys) + r);
#pragma unroll
          for (int c = 0; c < GBA_MAX_COLS; ++c)
            if (c < Sig::ncols(q))
              raw[i][c] = gba_type_bytes(Sig::coltype(q, c)) == 8 ? __ldcs(static_cast<const unsigned long long*>(q.cols[c]) + r)
                                                        : __ldcs(static_cast<const unsigned*>(q.cols[c]) + r);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < R; ++i) row_contrib<Sig>(q, raw[i], v[i]);
  }
  if constexpr (HBM) stream_rows_hbm<K64, Sig, R>(bq, key, v, live);
  else stream_rows<K64, Sig, R>(bq, st, nbk, key, v, live);
}
// Persistent streaming aggregation over a work queue of items given as query
// spans (see BatchSpan).
// sprobe: buckets probed before a row goes to the HBM table (BatchQ.pad bits
// 8..15 override it per query when nonzero).
// HBM: a launch of queries without a shared table (BatchQ.S == 0 for all):
// the kernel without the table code, so fewer registers live through the row
// loop (measured: twice the rows per lane instead spilled 60 bytes a thread
// and made the batch step slower, 10.89 against 10.20 ms).
template <bool K64, typename Sig, int MINB, bool HBM>
__global__ void __launch_bounds__(512, MINB) k_stream_agg(const BatchQ* qs, const BatchSpan* spans, int nspans,
                                                          int64_t nitems, unsigned* item_ctr, int sprobe) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned s_item;
  __shared__ unsigned long long s_next;
  __shared__ __align__(16) BatchQ s_q;
  constexpr int R = stream_rows_per_lane<Sig, MINB>();
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(item_ctr, 1u);
    __syncthreads();
    const int64_t it = int64_t(s_item);
    if (it >= nitems) break;
    int lo = 0, hi = nspans - 1;
    while (lo < hi) {  // last span starting at or before item it
      const int mid = (lo + hi + 1) >> 1;
      if (spans[mid].first_item <= it) lo = mid;
      else hi = mid - 1;
    }
    const BatchSpan sp = spans[lo];
    struct {
      int qi;
      int64_t row_begin, row_end;
    } item;
    item.qi = sp.qi;
    item.row_begin = (it - sp.first_item) * sp.item_rows;
    item.row_end = item.row_begin + sp.item_rows < qs[sp.qi].q.n ? item.row_begin + sp.item_rows : qs[sp.qi].q.n;
    {
      const unsigned* src = reinterpret_cast<const unsigned*>(qs + item.qi);
      unsigned* dst = reinterpret_cast<unsigned*>(&s_q);
      for (int w = tid; w < int(sizeof(BatchQ) / 4); w += blockDim.x) dst[w] = src[w];
    }
    if (tid == 0) s_next = (unsigned long long)item.row_begin;
    __syncthreads();
    const SmemTable<K64> st = smem_table_carve<K64>(smem, HBM ? 0 : s_q.S, Sig::nwords(s_q.q));
    if (!HBM && s_q.S > 0) smem_table_init<K64, Sig>(st, s_q.q);
    __syncthreads();
    const bool vec = (s_q.pad & 1) != 0;
    const int nbk = (s_q.pad >> 8) & 255 ? (s_q.pad >> 8) & 255 : sprobe;
    for (;;) {
      unsigned long long c0 = 0;
      if (lane_id() == 0) c0 = atomicAdd(&s_next, (unsigned long long)(32 * R));
      c0 = __shfl_sync(GBA_FULL_MASK, c0, 0);
      if (int64_t(c0) >= item.row_end) break;
      stream_chunk<K64, Sig, R, HBM>(s_q, st, nbk, int64_t(c0), item.row_end, vec);
    }
    __syncthreads();
    if (!HBM && s_q.S > 0) smem_flush_to_gtable<K64, Sig>(s_q.q, s_q.gt, st, s_q.flags);
    __syncthreads();  // s_q and the table are rewritten by the next item
  }
}

}  // namespace

// ---------------------------------------------------------------------------
int gba_stream_rows_per_chunk(const QDesc& q, int minb) {
  int r = 0;
  gba_dispatch_sig(q, [&](auto, auto sig) -> cudaError_t {
    r = 32 * (minb == 4   ? stream_rows_per_lane<decltype(sig), 4>()
              : minb == 3 ? stream_rows_per_lane<decltype(sig), 3>()
              : minb == 2 ? stream_rows_per_lane<decltype(sig), 2>()
                          : stream_rows_per_lane<decltype(sig), 1>());
    return cudaSuccess;
  });
  return r;
}

size_t gba_stream_smem_bytes(const QDesc& q, int S) { return smem_table_bytes(S, q.key64, q.nwords) + 64; }

namespace {
// f(std::integral_constant MINB, std::bool_constant HBM): the HBM-only kernels
// are built for 2 and 3 CTAs per SM; other shapes run the general kernel
template <typename F>
cudaError_t with_shape(int minb, bool hbm, F&& f) {
  using T = std::true_type;
  using Fl = std::false_type;
  if (hbm && minb == 3) return f(std::integral_constant<int, 3>{}, T{});
  if (hbm && minb == 2) return f(std::integral_constant<int, 2>{}, T{});
  return minb == 4   ? f(std::integral_constant<int, 4>{}, Fl{})
         : minb == 3 ? f(std::integral_constant<int, 3>{}, Fl{})
         : minb == 2 ? f(std::integral_constant<int, 2>{}, Fl{})
                     : f(std::integral_constant<int, 1>{}, Fl{});
}
}  // namespace

cudaError_t gba_prepare_stream_agg(const QDesc& proto, int minb, bool hbm) {
  return gba_dispatch_sig(proto, [&](auto K, auto sig) -> cudaError_t {
    constexpr bool k64 = decltype(K)::value;
    using Sig = decltype(sig);
    return with_shape(minb, hbm, [&](auto M, auto H) -> cudaError_t {
      return gba_allow_max_smem(k_stream_agg<k64, Sig, decltype(M)::value, decltype(H)::value>);
    });
  });
}

cudaError_t gba_launch_stream_agg(const QDesc& proto, int minb, bool hbm, const BatchQ* d_qs,
                                  const BatchSpan* d_spans, int nspans, int64_t nitems, unsigned* item_ctr,
                                  size_t smem, int sprobe, int grid, cudaStream_t s) {
  if (nitems <= 0 || nspans <= 0) return cudaSuccess;
  return gba_dispatch_sig(proto, [&](auto K, auto sig) -> cudaError_t {
    constexpr bool k64 = decltype(K)::value;
    using Sig = decltype(sig);
    return with_shape(minb, hbm, [&](auto M, auto H) -> cudaError_t {
      k_stream_agg<k64, Sig, decltype(M)::value, decltype(H)::value>
          <<<grid, 512, smem, s>>>(d_qs, d_spans, nspans, nitems, item_ctr, sprobe);
      return cudaGetLastError();
    });
  });
}
