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

// The shared table is probed by 16-byte buckets (4 32-bit or 2 64-bit keys):
// one vector load compares a whole bucket.  Inside a bucket, slots fill in
// order (a key is only ever claimed in the first empty slot of a complete
// read of its bucket, and slots never empty during an item), so a key found
// absent from a full read with an empty slot is absent from the bucket, and
// it can live in one slot only.
template <bool K64>
struct BucketT {
  static constexpr int SPB = K64 ? 2 : 4;  // slots per bucket
  typedef typename SmemTable<K64>::KeyW KeyW;
};

template <bool K64>
__device__ __forceinline__ void ld_bucket(const typename SmemTable<K64>::KeyW* keys, int b,
                                          typename SmemTable<K64>::KeyW (&o)[BucketT<K64>::SPB]) {
  unsigned x0, x1, x2, x3;
  asm volatile("ld.volatile.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(x0), "=r"(x1), "=r"(x2), "=r"(x3)
               : "r"(smem_u32(keys + b * BucketT<K64>::SPB)));
  if constexpr (K64) {
    o[0] = (unsigned long long)x1 << 32 | x0;
    o[1] = (unsigned long long)x3 << 32 | x2;
  } else {
    o[0] = x0;
    o[1] = x1;
    o[2] = x2;
    o[3] = x3;
  }
}

template <bool K64>
__device__ __forceinline__ int bucket_home(const SmemTable<K64>& t, uint32_t h) {
  return int((uint64_t(h) * unsigned(t.S / BucketT<K64>::SPB)) >> 32);
}

// slot of `key` in the shared table, inserting it if absent; -1 when
// `max_buckets` buckets from its home bucket are full without it
// (out of line: it is the slow path, and inlining it for every row of the
// unrolled chunk overflows the instruction cache)
template <bool K64>
__device__ __noinline__ int bucket_find_or_insert(const SmemTable<K64> t, uint64_t key, uint32_t h,
                                                  int max_buckets) {
  constexpr int SPB = BucketT<K64>::SPB;
  typedef typename SmemTable<K64>::KeyW KeyW;
  const KeyW kk = KeyW(key), empty = smem_empty_key<K64>();
  const int nb = t.S / SPB;
  int b = bucket_home<K64>(t, h);
  for (int p = 0; p < max_buckets; ++p) {
    for (int tries = 0; tries <= SPB; ++tries) {  // a lost claim means one more slot of the bucket is filled
      KeyW k[SPB];
      ld_bucket<K64>(t.keys, b, k);
      int free_e = -1;
#pragma unroll
      for (int e = SPB - 1; e >= 0; --e) {
        if (k[e] == kk) return b * SPB + e;
        if (k[e] == empty) free_e = e;
      }
      if (free_e < 0) break;
      const KeyW prev = atomicCAS(&t.keys[b * SPB + free_e], empty, kk);
      if (prev == empty || prev == kk) return b * SPB + free_e;
    }
    b = b + 1 == nb ? 0 : b + 1;
  }
  return -1;
}

// Accumulator updates of up to R rows (bit i of `rows` set: row i goes to
// shared slot slot[i]).  COUNT and the low word of an integer SUM are issued
// for all rows before any returned value is used; the SUM's carry into its
// high word follows.  Other ops take the generic per-row path.
template <bool K64, typename Sig, int R>
__device__ __forceinline__ void smem_apply_rows(const SmemTable<K64>& t, const QDesc& q, const int (&slot)[R],
                                                const unsigned long long (&v)[R][Sig::NA], unsigned rows) {
#pragma unroll
  for (int a = 0; a < Sig::NA; ++a) {
    const int op = Sig::op(q, a);
    const int w = Sig::woff(q, a);
    // split word: low halves at lo32[slot], high halves at lo32[S + slot]
    unsigned* lo32 = reinterpret_cast<unsigned*>(t.acc + size_t(w) * t.S);
    if (op == ACC_CNT) {
#pragma unroll
      for (int i = 0; i < R; ++i)
        if (rows >> i & 1u) atomicAdd(lo32 + slot[i], unsigned(v[i][a]));
    } else if (op == ACC_ADD_I) {
      unsigned old[R];
#pragma unroll
      for (int i = 0; i < R; ++i) {
        old[i] = 0u;
        if (rows >> i & 1u) old[i] = atomicAdd(lo32 + slot[i], unsigned(v[i][a]));
      }
#pragma unroll
      for (int i = 0; i < R; ++i) {
        if (!(rows >> i & 1u)) continue;
        const unsigned lo = unsigned(v[i][a]), hi = unsigned(v[i][a] >> 32);
        const unsigned add_hi = hi + ((old[i] + lo) < old[i] ? 1u : 0u);
        if (add_hi) atomicAdd(lo32 + t.S + slot[i], add_hi);
      }
    } else {
#pragma unroll
      for (int i = 0; i < R; ++i) {
        if (!(rows >> i & 1u)) continue;
        if (op == ACC_ADD_F)
          smem_fsum(smem_ref<K64>(t, w, slot[i]), smem_ref<K64>(t, w + 1, slot[i]), smem_ref<K64>(t, w + 2, slot[i]),
                    __longlong_as_double(v[i][a]));
        else smem_acc(op, smem_ref<K64>(t, w, slot[i]), v[i][a]);
      }
    }
  }
}

// A row's accumulator contributions, passed by value to the out-of-line slow
// path: a reference to one row of the caller's v[R][NA] would take the array's
// address and move all of it to local memory for the whole chunk.
template <int NA>
struct AccVals {
  unsigned long long x[NA];
};

// HBM-table insert that did not find its key in the home slot (first
// occurrence, or a displaced key): out of line, like bucket_find_or_insert.
template <bool K64, typename Sig>
__device__ __noinline__ void gtable_insert_slow(const GTable gt, const QDesc& q, uint64_t key, uint64_t home,
                                                unsigned long long cur, const AccVals<Sig::NA> v, unsigned* flags) {
  gtable_finish<K64, Sig>(gt, q, key, home, cur, v.x, flags);
}

template <bool K64, typename Sig, int R>
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

  // shared-table pass, phase by phase over the lane's R rows so that their
  // shared-memory round trips overlap: first every row's home-slot key, then
  // the rows that did not find their key there walk the probe sequence, then
  // the accumulator updates of all rows are issued before any result is used
  unsigned miss = 0;
  uint32_t h[R];
#pragma unroll
  for (int i = 0; i < R; ++i) h[i] = table_hash(key[i]);
  if (bq.S > 0) {
    typedef typename SmemTable<K64>::KeyW KeyW;
    constexpr int SPB = BucketT<K64>::SPB;
    int slot[R];
    KeyW kb[R][SPB];
#pragma unroll
    for (int i = 0; i < R; ++i) ld_bucket<K64>(st.keys, bucket_home<K64>(st, h[i]), kb[i]);
    unsigned hit = 0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      slot[i] = -1;
      if (!live[i]) continue;
      if (key[i] == emptyk) {  // the all-ones key has its own slot
        smem_apply_side<K64, Sig>(st, q, v[i]);
        continue;
      }
      bool has_empty = false;
#pragma unroll
      for (int e = 0; e < SPB; ++e) {
        if (kb[i][e] == KeyW(key[i])) slot[i] = bucket_home<K64>(st, h[i]) * SPB + e;
        has_empty = has_empty || kb[i][e] == smem_empty_key<K64>();
      }
      // a home bucket read full without the key settles a one-bucket probe
      if (slot[i] < 0 && (has_empty || nbk > 1)) slot[i] = bucket_find_or_insert<K64>(st, key[i], h[i], nbk);
      if (slot[i] >= 0) hit |= 1u << i;
      else miss |= 1u << i;
    }
    smem_apply_rows<K64, Sig, R>(st, q, slot, v, hit);
  } else {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      if (!live[i]) continue;
      if (key[i] == emptyk) gtable_insert<K64, Sig>(bq.gt, q, key[i], 0u, v[i], bq.flags);
      else miss |= 1u << i;
    }
  }
  if (miss == 0) return;
  // HBM-table pass: every missed row's home-slot load first, then the inserts
  // (measured: also loading the slot after the home slot, to place displaced
  // keys without a second round trip, costs more in L2 requests than it saves)
  constexpr int stride = 1 + NA;
  uint64_t home[R];
  unsigned long long cur[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    home[i] = 0;
    cur[i] = 0;
    if (miss >> i & 1u) {
      home[i] = gtable_home(bq.gt, h[i]);
      cur[i] = __ldcg(bq.gt.base + home[i] * stride);
    }
  }
#pragma unroll
  for (int i = 0; i < R; ++i) {
    if (!(miss >> i & 1u)) continue;
    if (cur[i] == key[i]) {  // the key sits in its home slot: reductions only
      unsigned long long* sp = bq.gt.base + home[i] * stride;
#pragma unroll
      for (int a = 0; a < NA; ++a) global_acc(Sig::op(q, a), sp + 1 + a, v[i][a]);
    } else {
      AccVals<NA> vv;
#pragma unroll
      for (int a = 0; a < NA; ++a) vv.x[a] = v[i][a];
      gtable_insert_slow<K64, Sig>(bq.gt, q, key[i], home[i], cur[i], vv, bq.flags);
    }
  }
}

// Persistent streaming aggregation over a work queue of items given as query
// spans (see BatchSpan).
// sprobe: buckets probed before a row goes to the HBM table (BatchQ.pad bits
// 8..15 override it per query when nonzero).
template <bool K64, typename Sig, int MINB>
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
    const SmemTable<K64> st = smem_table_carve<K64>(smem, s_q.S, Sig::nwords(s_q.q));
    if (s_q.S > 0) smem_table_init<K64, Sig>(st, s_q.q);
    __syncthreads();
    const bool vec = (s_q.pad & 1) != 0;
    const int nbk = (s_q.pad >> 8) & 255 ? (s_q.pad >> 8) & 255 : sprobe;
    for (;;) {
      unsigned long long c0 = 0;
      if (lane_id() == 0) c0 = atomicAdd(&s_next, (unsigned long long)(32 * R));
      c0 = __shfl_sync(GBA_FULL_MASK, c0, 0);
      if (int64_t(c0) >= item.row_end) break;
      stream_chunk<K64, Sig, R>(s_q, st, nbk, int64_t(c0), item.row_end, vec);
    }
    __syncthreads();
    if (s_q.S > 0) smem_flush_to_gtable<K64, Sig>(s_q.q, s_q.gt, st, s_q.flags);
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

cudaError_t gba_prepare_stream_agg(const QDesc& proto, int minb) {
  return gba_dispatch_sig(proto, [&](auto K, auto sig) -> cudaError_t {
    constexpr bool k64 = decltype(K)::value;
    using Sig = decltype(sig);
    return minb == 4   ? gba_allow_max_smem(k_stream_agg<k64, Sig, 4>)
           : minb == 3 ? gba_allow_max_smem(k_stream_agg<k64, Sig, 3>)
           : minb == 2 ? gba_allow_max_smem(k_stream_agg<k64, Sig, 2>)
                       : gba_allow_max_smem(k_stream_agg<k64, Sig, 1>);
  });
}

cudaError_t gba_launch_stream_agg(const QDesc& proto, int minb, const BatchQ* d_qs, const BatchSpan* d_spans,
                                  int nspans, int64_t nitems, unsigned* item_ctr, size_t smem, int sprobe, int grid,
                                  cudaStream_t s) {
  if (nitems <= 0 || nspans <= 0) return cudaSuccess;
  return gba_dispatch_sig(proto, [&](auto K, auto sig) -> cudaError_t {
    constexpr bool k64 = decltype(K)::value;
    using Sig = decltype(sig);
    if (minb == 4) k_stream_agg<k64, Sig, 4><<<grid, 512, smem, s>>>(d_qs, d_spans, nspans, nitems, item_ctr, sprobe);
    else if (minb == 3)
      k_stream_agg<k64, Sig, 3><<<grid, 512, smem, s>>>(d_qs, d_spans, nspans, nitems, item_ctr, sprobe);
    else if (minb == 2)
      k_stream_agg<k64, Sig, 2><<<grid, 512, smem, s>>>(d_qs, d_spans, nspans, nitems, item_ctr, sprobe);
    else k_stream_agg<k64, Sig, 1><<<grid, 512, smem, s>>>(d_qs, d_spans, nspans, nitems, item_ctr, sprobe);
    return cudaGetLastError();
  });
}
