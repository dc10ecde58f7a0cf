// Streaming group-by kernel with bulk-copy staging (sm_100a): the batch
// kernel of the table strategy.
//
// Replaces the reference's per-tile chain (tiled_groupby_agg_partition/src/
// kernel.cu:9-186: a one-probe HBM table, CUB scans, a linear-probe spill
// table) with one persistent launch over a device work queue of
// (query, row range) items, like k_stream.cu, but the rows reach shared memory
// by bulk copies instead of register loads:
//
//   * Every warp runs its own ring of `nstages` slots of 32 x R rows.  Lane 0
//     claims the item's next chunk (a shared cursor) for a free slot and issues
//     one cp.async.bulk per column (keys, then each value column) into it,
//     completing on that slot's mbarrier (1-D bulk copies; no tensor map and no
//     multicast).  The warp then works on its oldest slot while the copies of
//     the others stream in, so up to nstages - 1 chunks per warp are in flight
//     whatever the hash-table work costs.  No barrier joins the warps while an
//     item streams (a CTA-wide barrier per stage, measured, let the slowest
//     warp's L2 misses stall the whole SM: twice the time).
//   * Lane l takes rows l + 32 i of a chunk (conflict-free shared loads) and
//     runs them through the item's shared table, or the query's HBM table for
//     rows that miss it (stream_rows.cuh).
//   * With a query's bit 1 of BatchQ.pad set (skewed keys), lanes of a warp
//     holding equal keys first combine their rows (a log-depth tree over each
//     group of equal keys), so a hot key costs one atomic per warp instead of
//     one per lane, serialised.
//   * Every wait on a copy is bounded (GBA_FLAG_WAIT_TIMEOUT); a warp that gives
//     up waits, again bounded, for its copies in flight before it stops.
//
// Slot layout: keys [32 R] then every value column [32 R], each region a
// multiple of 16 bytes.  A chunk starts at a row that is a multiple of 4
// (items are cut at multiples of 2048 rows, chunks at multiples of 32 R), so
// with 16-byte-aligned columns every copy starts on a 16-byte boundary; the
// rows of a chunk past its last multiple of 4 (only at the end of a query) are
// read from global memory, and so is every row of a query whose columns are
// not 16-byte aligned.
#include "batch_kernels.h"
#include "gba_internal.cuh"
#include "smem_table.cuh"

namespace {
#include "stream_rows.cuh"

constexpr int kTmaMaxStages = 4;

// CTA shapes (template MINB): 1 or 2 CTAs of 512 threads per SM (MINB = 1,
// 2), or MINB = 0: one CTA of 1024 threads per SM, which holds as many warps
// as two 512-thread CTAs with one shared table of twice the slots.
template <int MINB>
__host__ __device__ constexpr int tma_threads() {
  return MINB == 0 ? 1024 : 512;
}
template <int MINB>
__host__ __device__ constexpr int tma_ctas_per_sm() {
  return MINB == 0 ? 1 : MINB;
}

// rows per lane per chunk: fewer with more accumulators, and fewer when an
// SM holds 32 warps (their registers are split).  With 16-byte rows a slot
// holds 2 KB (16 warps per SM) or 1 KB (32), so two or three slots per warp
// keep 64-96 KB of copies in flight per SM and leave the rest of the shared
// memory to the tables.
template <typename Sig, int MINB>
__host__ __device__ constexpr int tma_rows_per_lane() {
  return MINB == 1 ? (Sig::NA <= 2 ? 4 : (Sig::NA <= 4 ? 2 : 1)) : (Sig::NA <= 2 ? 2 : 1);
}

__host__ __device__ inline int col_bytes_of(int t) { return (t == GBA_I64 || t == GBA_F64) ? 8 : 4; }

// bytes of one stage of `sr` rows of query q, and each column's offset in it
__host__ __device__ inline size_t tma_stage_layout(const QDesc& q, int sr, size_t (&coff)[GBA_MAX_COLS]) {
  size_t o = size_t(sr) * (q.key64 ? 8 : 4);
#pragma unroll
  for (int c = 0; c < GBA_MAX_COLS; ++c) {
    coff[c] = o;
    if (c < q.ncols) o += size_t(sr) * col_bytes_of(q.col_type[c]);
  }
  return o;
}

// Lanes of a warp whose keys are equal combine their contributions; the lowest
// lane of each such group keeps the combined row (returns true), the others
// drop theirs.  All 32 lanes call it.  The combination is a tree over each
// group: in round d every remaining lane adds the value of the nearest
// remaining lane of its group above it, then the lanes at odd positions of the
// round (already added into their neighbour below) leave; ceil(log2(largest
// group)) rounds.  This is the segmented warp reduction of the published
// warp-aggregated-atomics technique (Lin and Grover, "Using CUDA Warp-Level
// Primitives", 2018), written here for this library's accumulator types.
template <bool K64, typename Sig>
__device__ __forceinline__ bool warp_combine_equal_keys(const QDesc& q, bool live, uint64_t key,
                                                        unsigned long long (&v)[Sig::NA]) {
  constexpr int NA = Sig::NA;
  const unsigned lane = lane_id();
  const unsigned live_mask = __ballot_sync(GBA_FULL_MASK, live);
  unsigned group;
  if constexpr (K64) group = __match_any_sync(GBA_FULL_MASK, (unsigned long long)key);
  else group = __match_any_sync(GBA_FULL_MASK, unsigned(key));
  group = live ? (group & live_mask) : (1u << lane);
  if (__reduce_max_sync(GBA_FULL_MASK, unsigned(__popc(group))) <= 1u) return live;
  // position among the group's lanes, and the group's lanes above this one
  unsigned pos = __popc(group & ((1u << lane) - 1u));
  unsigned above = group & ~((2u << lane) - 1u);  // lane 31: 2u << 31 == 0, so none
  while (__any_sync(GBA_FULL_MASK, above != 0u)) {
    const int nxt = __ffs(above);  // 0 when none
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      const unsigned long long x = __shfl_sync(GBA_FULL_MASK, v[a], nxt ? nxt - 1 : int(lane));
      if (nxt) v[a] = acc_combine(Sig::op(q, a), v[a], x);
    }
    const unsigned gone = __ballot_sync(GBA_FULL_MASK, (pos & 1u) != 0u);
    above &= ~gone;
    pos >>= 1;
  }
  return live && (group & ((1u << lane) - 1u)) == 0u;
}

// CL = 1: every CTA takes its own items.  CL > 1 (a thread-block cluster of CL
// CTAs, integer SUM/COUNT signatures): the cluster takes an item together, CTA
// rank r streaming the r-th of CL equal parts of it; the item's shared table
// is the CL CTAs' tables together (stream_rows_cluster), cleared by every CTA
// before any row of the item is applied and merged into HBM by every CTA
// after all rows are, with a cluster barrier between the phases.  A CTA
// with a warp whose copy wait gave up stops working but keeps taking part in
// the cluster's barriers until the queue is empty, so no CTA waits for it.
template <bool K64, typename Sig, int CL, int MINB>
__global__ void __launch_bounds__(tma_threads<MINB>(), tma_ctas_per_sm<MINB>())
    k_stream_tma(const BatchQ* qs, const BatchSpan* spans, int nspans, int64_t nitems, unsigned* item_ctr,
                 int sprobe, int nstages, unsigned slot_bytes) {
  constexpr int R = tma_rows_per_lane<Sig, MINB>();
  constexpr int CR = 32 * R;  // rows per chunk
  constexpr int NA = Sig::NA;
  constexpr int NW = tma_threads<MINB>() / 32;  // warps
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bars[NW * kTmaMaxStages];
  __shared__ unsigned s_item;
  __shared__ int s_abort;
  __shared__ unsigned long long s_next;
  __shared__ long long s_chunk[NW][kTmaMaxStages];  // warp w's slot s holds rows from s_chunk[w][s]
  __shared__ __align__(16) BatchQ s_q;
  const int tid = threadIdx.x;
  const unsigned lane = lane_id(), warp = unsigned(tid) >> 5;
  const size_t ring = size_t(NW) * nstages * slot_bytes;
  unsigned char* const wring = smem + size_t(warp) * nstages * slot_bytes;  // this warp's slots
  uint64_t* const wbar = bars + warp * kTmaMaxStages;
  const unsigned rank = CL > 1 ? cluster_ctarank() : 0u;
  if (lane == 0) {
    for (int s = 0; s < nstages; ++s) mbar_init(&wbar[s], 1);
    mbar_fence_init();
  }
  if (tid == 0) s_abort = 0;
  __syncthreads();
  unsigned phase = 0;    // bit s: parity of the next completion to wait for on slot s
  unsigned pending = 0;  // (lane 0) bit s: slot s has a copy in flight
  bool dead = false;     // (CL > 1) this CTA gave up on a copy; it only keeps the barriers
  for (;;) {
    if constexpr (CL > 1) {
      if (rank == 0 && tid == 0) {
        const unsigned v = atomicAdd(item_ctr, 1u);
        for (unsigned r = 0; r < unsigned(CL); ++r) dsmem_st_u32(dsmem_map(smem_u32(&s_item), r), v);
      }
      cluster_sync_all();
    } else {
      if (tid == 0) s_item = atomicAdd(item_ctr, 1u);
      __syncthreads();
    }
    const int64_t it = int64_t(s_item);
    if (it >= nitems) break;
    int lo = 0, hi = nspans - 1;
    while (lo < hi) {  // last span starting at or before item it
      const int mid = (lo + hi + 1) >> 1;
      if (spans[mid].first_item <= it) lo = mid;
      else hi = mid - 1;
    }
    const BatchSpan sp = spans[lo];
    const int64_t ib = (it - sp.first_item) * sp.item_rows;
    const int64_t qn = qs[sp.qi].q.n;
    const int64_t ie = ib + sp.item_rows < qn ? ib + sp.item_rows : qn;
    // this CTA's rows of the item: all of them, or its part of CL chunk-aligned parts
    int64_t pb = ib, pe = ie;
    if constexpr (CL > 1) {
      const int64_t part = ((ie - ib + CL - 1) / CL + CR - 1) / CR * CR;
      pb = ib + part * rank < ie ? ib + part * rank : ie;
      pe = pb + part < ie ? pb + part : ie;
    }
    {
      const unsigned* src = reinterpret_cast<const unsigned*>(qs + sp.qi);
      unsigned* dst = reinterpret_cast<unsigned*>(&s_q);
      for (int w = tid; w < int(sizeof(BatchQ) / 4); w += blockDim.x) dst[w] = src[w];
    }
    if (tid == 0) s_next = (unsigned long long)pb;
    __syncthreads();
    const QDesc& q = s_q.q;
    const SmemTable<K64> st = smem_table_carve<K64>(smem + ring, s_q.S, Sig::nwords(q));
    if (s_q.S > 0) smem_table_init<K64, Sig>(st, q);
    const bool tma = (s_q.pad & 1) != 0;
    const bool comb = (s_q.pad & 2) != 0;
    const int nbk = (s_q.pad >> 8) & 255 ? (s_q.pad >> 8) & 255 : sprobe;
    size_t coff[GBA_MAX_COLS];
    tma_stage_layout(q, CR, coff);
    const int kb = K64 ? 8 : 4;
    auto issue = [&](int64_t c0, int s) {  // lane 0
      const int64_t left = pe - c0;
      const uint32_t rows = uint32_t(left < CR ? left : CR) & ~3u;
      unsigned char* dst = wring + size_t(s) * slot_bytes;
      uint32_t bytes = rows * kb;
#pragma unroll
      for (int c = 0; c < GBA_MAX_COLS; ++c)
        if (c < Sig::ncols(q)) bytes += rows * col_bytes_of(Sig::coltype(q, c));
      mbar_arrive_expect_tx(&wbar[s], bytes);
      bulk_g2s(dst, static_cast<const unsigned char*>(q.keys) + c0 * kb, rows * kb, &wbar[s]);
#pragma unroll
      for (int c = 0; c < GBA_MAX_COLS; ++c) {
        if (c < Sig::ncols(q)) {
          const int cb = col_bytes_of(Sig::coltype(q, c));
          bulk_g2s(dst + coff[c], static_cast<const unsigned char*>(q.cols[c]) + c0 * cb, rows * cb, &wbar[s]);
        }
      }
    };
    // a chunk goes through a slot by bulk copy when it holds at least 4 rows
    auto via_copy = [&](int64_t c0) { return tma && c0 < pe && pe - c0 >= 4; };
    if constexpr (CL > 1) cluster_sync_all();  // every CTA's table part cleared before any row lands in it
    else __syncthreads();                      // table initialised

    // this warp's ring: slot s holds the chunk starting at s_chunk[warp][s]
    // (chunks are claimed in slot order)
    long long* const cs = s_chunk[warp];
    if (lane == 0) {
      for (int s = 0; s < nstages; ++s) {
        const unsigned long long c = atomicAdd(&s_next, (unsigned long long)CR);
        cs[s] = (long long)c;
        if (!dead && via_copy(int64_t(c))) {
          issue(int64_t(c), s);
          pending |= 1u << s;
        }
      }
    }
    __syncwarp();
    for (int s = 0; !dead;) {
      const int64_t c0 = cs[s];
      if (c0 >= pe) break;  // later slots hold later chunks: all past the end
      const int rows = pe - c0 < CR ? int(pe - c0) : CR;
      const bool copied = via_copy(c0);
      const int rows_tma = copied ? (rows & ~3) : 0;
      if (copied) {
        // the warp goes on only if every lane saw the copy land (the lanes
        // stay together for the warp-wide steps below)
        const bool landed = mbar_wait_bounded(&wbar[s], (phase >> s) & 1u, s_q.flags);
        if (__all_sync(GBA_FULL_MASK, landed)) {
          phase ^= 1u << s;
          if (lane == 0) pending &= ~(1u << s);
        } else {
          // give up: drain this warp's copies in flight, stop the CTA
          s_abort = 1;
          if (lane == 0) {
            for (int x = 0; x < nstages; ++x) {
              if (!(pending >> x & 1u)) continue;
              bool landed = false;
              for (unsigned n = 0; n < (1u << 22) && !landed; ++n) landed = mbar_try_wait(&wbar[x], (phase >> x) & 1u);
              if (!landed) atomicOr(s_q.flags, GBA_FLAG_DRAIN_TIMEOUT);
            }
            pending = 0;
          }
          __syncwarp();
          break;
        }
      }
      {
        const unsigned char* sb = wring + size_t(s) * slot_bytes;
        uint64_t key[R];
        unsigned long long v[R][NA];
        bool live[R];
#pragma unroll
        for (int i = 0; i < R; ++i) {
          const int r = int(lane) + 32 * i;
          live[i] = r < rows;
          key[i] = K64 ? EMPTY64 : uint64_t(EMPTY32);
          unsigned long long raw[GBA_MAX_COLS] = {0ull, 0ull, 0ull, 0ull};
          if (r < rows_tma) {
            key[i] = K64 ? reinterpret_cast<const unsigned long long*>(sb)[r] : reinterpret_cast<const unsigned*>(sb)[r];
#pragma unroll
            for (int c = 0; c < GBA_MAX_COLS; ++c)
              if (c < Sig::ncols(q))
                raw[c] = col_bytes_of(Sig::coltype(q, c)) == 8
                             ? reinterpret_cast<const unsigned long long*>(sb + coff[c])[r]
                             : reinterpret_cast<const unsigned*>(sb + coff[c])[r];
          } else if (r < rows) {
            const int64_t g = c0 + r;
            key[i] = K64 ? __ldcs(static_cast<const unsigned long long*>(q.keys) + g)
                         : __ldcs(static_cast<const unsigned*>(q.keys) + g);
#pragma unroll
            for (int c = 0; c < GBA_MAX_COLS; ++c)
              if (c < Sig::ncols(q))
                raw[c] = col_bytes_of(Sig::coltype(q, c)) == 8
                             ? __ldcs(static_cast<const unsigned long long*>(q.cols[c]) + g)
                             : __ldcs(static_cast<const unsigned*>(q.cols[c]) + g);
          }
          row_contrib<Sig>(q, raw, v[i]);
        }
        __syncwarp();  // the slot's rows are in registers: lane 0 may refill it
        if (lane == 0) {
          const unsigned long long c = atomicAdd(&s_next, (unsigned long long)CR);
          cs[s] = (long long)c;
          if (via_copy(int64_t(c))) {
            fence_proxy_async_smem();
            issue(int64_t(c), s);
            pending |= 1u << s;
          }
        }
        __syncwarp();
        if (comb) {
#pragma unroll
          for (int i = 0; i < R; ++i) live[i] = warp_combine_equal_keys<K64, Sig>(q, live[i], key[i], v[i]);
        }
        if constexpr (CL > 1) {
          if (s_q.S > 0) stream_rows_cluster<K64, Sig, R>(s_q, st, nbk, CL, key, v, live);
          else stream_rows<K64, Sig, R>(s_q, st, nbk, key, v, live);
        } else {
          stream_rows<K64, Sig, R>(s_q, st, nbk, key, v, live);
        }
      }
      s = s + 1 == nstages ? 0 : s + 1;
    }
    __syncthreads();  // every warp done with the item (and s_abort visible)
    if (s_abort) dead = true;
    if constexpr (CL > 1) {
      cluster_sync_all();  // every row of the item applied, in every CTA's table part
      if (!dead && s_q.S > 0) smem_flush_to_gtable<K64, Sig>(q, s_q.gt, st, s_q.flags);
      __syncthreads();  // s_q and the table are rewritten by the next item
    } else {
      if (dead) return;
      if (s_q.S > 0) smem_flush_to_gtable<K64, Sig>(q, s_q.gt, st, s_q.flags);
      __syncthreads();  // s_q and the table are rewritten by the next item
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
namespace {
template <typename F>
cudaError_t with_minb(int minb, F&& f) {
  return minb == 2   ? f(std::integral_constant<int, 2>{})
         : minb == 0 ? f(std::integral_constant<int, 0>{})
                     : f(std::integral_constant<int, 1>{});
}
}  // namespace

size_t gba_stream_tma_slot_bytes(const QDesc& q, int minb) {
  size_t b = 0;
  gba_dispatch_sig(q, [&](auto, auto sig) -> cudaError_t {
    return with_minb(minb, [&](auto M) -> cudaError_t {
      size_t coff[GBA_MAX_COLS];
      b = tma_stage_layout(q, 32 * tma_rows_per_lane<decltype(sig), decltype(M)::value>(), coff);
      return cudaSuccess;
    });
  });
  return (b + 127) / 128 * 128;
}

size_t gba_stream_tma_smem_bytes(const QDesc& q, int S, int nstages, size_t slot_bytes, int minb) {
  const size_t warps = size_t(minb == 0 ? tma_threads<0>() : tma_threads<1>()) / 32;
  return warps * nstages * slot_bytes + smem_table_bytes(S, q.key64, q.nwords) + 64;
}

bool gba_stream_tma_cluster_ok(const QDesc& q) {
  bool ok = false;
  gba_dispatch_sig(q, [&](auto, auto sig) -> cudaError_t {
    ok = ClusterSig<decltype(sig)>::ok;
    return cudaSuccess;
  });
  return ok;
}

namespace {
template <bool K64, typename Sig, int CL, int MINB>
cudaError_t prepare_one() {
  auto* f = k_stream_tma<K64, Sig, CL, MINB>;
  cudaError_t e = gba_allow_max_smem(f);
  if (e == cudaSuccess && CL > 8) e = cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

template <int CL>
void cluster_cfg(cudaLaunchConfig_t& cfg, cudaLaunchAttribute (&attr)[1], int grid, size_t smem, cudaStream_t s) {
  cfg = {};
  cfg.gridDim = dim3(unsigned(grid / CL * CL));
  cfg.blockDim = dim3(tma_threads<1>());
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
}

template <bool K64, typename Sig, int CL, int MINB>
cudaError_t launch_one(const BatchQ* d_qs, const BatchSpan* d_spans, int nspans, int64_t nitems, unsigned* item_ctr,
                       size_t smem, int sprobe, int grid, int nstages, size_t slot_bytes, cudaStream_t s) {
  if constexpr (CL == 1) {
    k_stream_tma<K64, Sig, 1, MINB><<<grid, tma_threads<MINB>(), smem, s>>>(d_qs, d_spans, nspans, nitems, item_ctr,
                                                                            sprobe, nstages, unsigned(slot_bytes));
    return cudaGetLastError();
  } else {
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr[1];
    cluster_cfg<CL>(cfg, attr, grid, smem, s);
    return cudaLaunchKernelEx(&cfg, k_stream_tma<K64, Sig, CL, MINB>, d_qs, d_spans, nspans, nitems, item_ctr,
                              sprobe, nstages, unsigned(slot_bytes));
  }
}

template <bool K64, typename Sig, int CL>
int max_clusters(size_t smem, int sms) {
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute attr[1];
  cluster_cfg<CL>(cfg, attr, sms, smem, nullptr);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_stream_tma<K64, Sig, CL, 1>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}
}  // namespace

cudaError_t gba_prepare_stream_tma(const QDesc& proto, int cluster, int minb) {
  return gba_dispatch_sig(proto, [&](auto K, auto sig) -> cudaError_t {
    constexpr bool k64 = decltype(K)::value;
    using Sig = decltype(sig);
    if constexpr (ClusterSig<Sig>::ok) {
      if (cluster == 16) return prepare_one<k64, Sig, 16, 1>();
      if (cluster == 8) return prepare_one<k64, Sig, 8, 1>();
      if (cluster == 4) return prepare_one<k64, Sig, 4, 1>();
      if (cluster == 2) return prepare_one<k64, Sig, 2, 1>();
    }
    if (cluster != 1) return cudaErrorInvalidValue;
    return with_minb(minb, [&](auto M) -> cudaError_t { return prepare_one<k64, Sig, 1, decltype(M)::value>(); });
  });
}

int gba_stream_tma_cluster_grid(const QDesc& proto, int cluster, size_t smem, int sms) {
  int n = 0;
  gba_dispatch_sig(proto, [&](auto K, auto sig) -> cudaError_t {
    constexpr bool k64 = decltype(K)::value;
    using Sig = decltype(sig);
    if constexpr (ClusterSig<Sig>::ok) {
      if (cluster == 16) n = max_clusters<k64, Sig, 16>(smem, sms);
      else if (cluster == 8) n = max_clusters<k64, Sig, 8>(smem, sms);
      else if (cluster == 4) n = max_clusters<k64, Sig, 4>(smem, sms);
      else if (cluster == 2) n = max_clusters<k64, Sig, 2>(smem, sms);
    }
    return cudaSuccess;
  });
  return n * cluster;
}

cudaError_t gba_launch_stream_tma(const QDesc& proto, int cluster, int minb, const BatchQ* d_qs,
                                  const BatchSpan* d_spans, int nspans, int64_t nitems, unsigned* item_ctr,
                                  size_t smem, int sprobe, int grid, int nstages, size_t slot_bytes, cudaStream_t s) {
  if (nitems <= 0 || nspans <= 0) return cudaSuccess;
  if (nstages < 1 || nstages > kTmaMaxStages || slot_bytes == 0 || slot_bytes % 16) return cudaErrorInvalidValue;
  return gba_dispatch_sig(proto, [&](auto K, auto sig) -> cudaError_t {
    constexpr bool k64 = decltype(K)::value;
    using Sig = decltype(sig);
    if constexpr (ClusterSig<Sig>::ok) {
      if (cluster == 16)
        return launch_one<k64, Sig, 16, 1>(d_qs, d_spans, nspans, nitems, item_ctr, smem, sprobe, grid, nstages,
                                           slot_bytes, s);
      if (cluster == 8)
        return launch_one<k64, Sig, 8, 1>(d_qs, d_spans, nspans, nitems, item_ctr, smem, sprobe, grid, nstages,
                                          slot_bytes, s);
      if (cluster == 4)
        return launch_one<k64, Sig, 4, 1>(d_qs, d_spans, nspans, nitems, item_ctr, smem, sprobe, grid, nstages,
                                          slot_bytes, s);
      if (cluster == 2)
        return launch_one<k64, Sig, 2, 1>(d_qs, d_spans, nspans, nitems, item_ctr, smem, sprobe, grid, nstages,
                                          slot_bytes, s);
    }
    if (cluster != 1) return cudaErrorInvalidValue;
    return with_minb(minb, [&](auto M) -> cudaError_t {
      return launch_one<k64, Sig, 1, decltype(M)::value>(d_qs, d_spans, nspans, nitems, item_ctr, smem, sprobe, grid,
                                                         nstages, slot_bytes, s);
    });
  });
}
