// Tiled hash pre-aggregation + HBM table + final compaction (sm_100a).
//
// Replaces the reference's per-tile aggregation chain (tiled_groupby_agg_partition/
// src/kernel.cu:9-186 driven by group_then_partition.cu:24-246: a one-probe
// "one-third" table in HBM, three CUB scans, a linear-probe spill table and two
// compaction kernels, with three host round-trips per tile) by:
//
//   k_table_init   - fills the HBM table with the empty key and identities.
//   k_preagg       - persistent CTAs stream row tiles into shared memory with
//                    TMA bulk copies (cp.async.bulk + mbarrier, no multicast),
//                    coalesce equal keys inside each warp with __match_any_sync,
//                    aggregate into a shared-memory open-addressing table with a
//                    capped probe count, send rows that do not fit to the HBM
//                    table, and flush the shared table to HBM at the end.
//   k_compact      - the final reduce: writes every occupied slot once to the
//                    caller's output columns (warp-aggregated output cursor).
#include "gba_internal.cuh"
#include "smem_table.cuh"
#include "batch_kernels.h"

namespace {

struct PreaggParams {
  QDesc q;
  GTable gt;
  int S;          // shared-memory table slots (0 = no pre-aggregation)
  int sprobe;     // probe cap in the shared table
  int T;          // rows per tile (multiple of blockDim.x and of 4)
  int nstages;    // TMA pipeline depth (1..4)
  int use_tma;    // 1: full tiles arrive by cp.async.bulk
  int coalesce;   // 1: __match_any_sync pre-combining
  unsigned* flags;
};

constexpr int kMaxStages = 4;

__host__ __device__ inline int key_bytes(const QDesc& q) { return q.key64 ? 8 : 4; }
__host__ __device__ inline int col_bytes(int t) { return gba_type_bytes(t); }
__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline size_t stage_bytes(const QDesc& q, int T) {
  size_t b = align16(size_t(T) * key_bytes(q));
#pragma unroll
  for (int c = 0; c < GBA_MAX_COLS; ++c)
    if (c < q.ncols) b += align16(size_t(T) * col_bytes(q.col_type[c]));
  return b;
}

// Row j of the current tile: from the TMA stage or straight from HBM.  The
// column count and types come from the signature (constants when compiled in).
template <bool K64, typename Sig>
__device__ __forceinline__ void load_row(const QDesc& q, bool via_tma, const unsigned char* sbase,
                                         const size_t (&coff)[GBA_MAX_COLS], int64_t r0, int j, uint64_t& key,
                                         unsigned long long (&r)[GBA_MAX_COLS]) {
#pragma unroll
  for (int c = 0; c < GBA_MAX_COLS; ++c) r[c] = 0ull;
  if (via_tma) {
    key = K64 ? reinterpret_cast<const unsigned long long*>(sbase)[j] : reinterpret_cast<const unsigned*>(sbase)[j];
#pragma unroll
    for (int c = 0; c < GBA_MAX_COLS; ++c)
      if (c < Sig::ncols(q))
        r[c] = col_bytes(Sig::coltype(q, c)) == 8 ? reinterpret_cast<const unsigned long long*>(sbase + coff[c])[j]
                                                  : reinterpret_cast<const unsigned*>(sbase + coff[c])[j];
  } else {
    key = K64 ? __ldg(static_cast<const unsigned long long*>(q.keys) + r0 + j)
              : __ldg(static_cast<const unsigned*>(q.keys) + r0 + j);
#pragma unroll
    for (int c = 0; c < GBA_MAX_COLS; ++c)
      if (c < Sig::ncols(q))
        r[c] = col_bytes(Sig::coltype(q, c)) == 8 ? __ldg(static_cast<const unsigned long long*>(q.cols[c]) + r0 + j)
                                                  : __ldg(static_cast<const unsigned*>(q.cols[c]) + r0 + j);
  }
}

// Phases A and B of one tile (every thread of the CTA calls it; it syncs
// between the phases, the caller syncs after it).
template <bool K64, typename Sig>
__device__ __forceinline__ void tile_two_phase(const QDesc& q, const GTable& gt, const SmemTable<K64>& st, int S,
                                               int sprobe, int coalesce, bool via_tma, const unsigned char* sbase,
                                               const size_t (&coff)[GBA_MAX_COLS], int64_t r0, int rows, int T,
                                               unsigned short* miss, unsigned* s_nmiss, unsigned* flags) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  const unsigned lane = lane_id();
  const uint64_t emptyk = K64 ? EMPTY64 : uint64_t(EMPTY32);
    // ---- phase A: shared-table pass (two rows per thread loaded up front) ----
    constexpr int R = 2;
    for (int j0 = 0; j0 < T; j0 += R * nthr) {
      uint64_t key[R];
      unsigned long long r[R][GBA_MAX_COLS];
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int j = j0 + u * nthr + tid;
        key[u] = emptyk;
        if (j < rows) load_row<K64, Sig>(q, via_tma, sbase, coff, r0, j, key[u], r[u]);
        else {
#pragma unroll
          for (int c = 0; c < GBA_MAX_COLS; ++c) r[u][c] = 0ull;
        }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int j = j0 + u * nthr + tid;
        const bool valid = j < rows;
        unsigned long long v[Sig::NA];
        row_contrib<Sig>(q, r[u], v);
        uint64_t k = key[u];
        const bool sent = valid && k == emptyk;
        if (sent) {
          if (S > 0) smem_apply_side<K64, Sig>(st, q, v);
          else gtable_insert<K64, Sig>(gt, q, k, 0u, v, flags);
        }
        bool live = valid && !sent;
        if (coalesce) {  // warp-synchronous: every lane of the warp is here
          if (!live) k = emptyk;
          live = warp_coalesce<K64, Sig>(q, live, k, v);
        }
        bool missed = false;
        if (live) {
          int slot = -1;
          const uint32_t h = table_hash(k);
          if (S > 0) slot = smem_find_or_insert<K64>(st, k, h, sprobe);
          if (slot >= 0) smem_apply<K64, Sig>(st, q, slot, v);
          else if (coalesce) gtable_insert<K64, Sig>(gt, q, k, h, v, flags);
          else missed = true;
        }
        // warp-aggregated append of the misses to the tile's miss list
        const unsigned mm = __ballot_sync(GBA_FULL_MASK, missed);
        if (mm) {
          unsigned base = 0;
          if (lane == 0) base = atomicAdd(s_nmiss, unsigned(__popc(mm)));
          base = __shfl_sync(GBA_FULL_MASK, base, 0);
          if (missed) miss[base + __popc(mm & ((1u << lane) - 1u))] = (unsigned short)j;
        }
      }
    }
    __syncthreads();

    // ---- phase B: HBM-table inserts of the misses, two in flight per thread ----
    const int nm = int(*s_nmiss);
    for (int i0 = 0; i0 < nm; i0 += 2 * nthr) {
      uint64_t k[2];
      uint64_t slot[2];
      unsigned long long cur[2];
      unsigned long long v[2][Sig::NA];
      bool act[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int i = i0 + u * nthr + tid;
        act[u] = i < nm;
        k[u] = 0;
        slot[u] = 0;
        unsigned long long rr[GBA_MAX_COLS] = {0ull, 0ull, 0ull, 0ull};
        if (act[u]) {
          load_row<K64, Sig>(q, via_tma, sbase, coff, r0, int(miss[i]), k[u], rr);
          slot[u] = gtable_home(gt, table_hash(k[u]));
        }
        row_contrib<Sig>(q, rr, v[u]);
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) cur[u] = act[u] ? __ldcg(gt.base + slot[u] * gba_gt_stride(Sig::NA)) : 0ull;
#pragma unroll
      for (int u = 0; u < 2; ++u)
        if (act[u]) gtable_finish<K64, Sig>(gt, q, k[u], slot[u], cur[u], v[u], flags);
    }
}

// Merges a CTA's shared table into the HBM table (caller synced first).
// Each tile is processed in two phases.
//  A: every row probes the CTA's shared table (capped probes) and updates it
//     with 32-bit atomics; a row whose key is not there and cannot enter only
//     records its index in the tile's miss list (warp-aggregated append).
//  B: the CTA walks the miss list with two independent HBM-table inserts per
//     thread in flight, so their L2 round trips overlap (the reference's
//     kernels do one dependent probe chain per thread,
//     kernel.cu:116-158).
// With warp coalescing enabled the leaders' combined contributions cannot be
// re-read from the tile, so their misses are inserted in phase A instead.
template <bool K64, typename Sig>
__global__ void __launch_bounds__(1024, 1) k_preagg(PreaggParams P) {
  extern __shared__ __align__(128) unsigned char smem[];
  const QDesc& q = P.q;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int T = P.T;
  const int64_t n = q.n;
  const int64_t ntiles = (n + T - 1) / T;
  const int64_t nfull = n / T;
  const int kb = K64 ? 8 : 4;
  const uint64_t emptyk = K64 ? EMPTY64 : uint64_t(EMPTY32);

  // ---- carve shared memory ------------------------------------------------------
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  size_t off = 128;
  const size_t sb = stage_bytes(q, T);
  unsigned char* stage0 = smem + off;
  if (P.use_tma) off += sb * P.nstages;
  unsigned short* miss = reinterpret_cast<unsigned short*>(smem + off);
  off += align16(size_t(T) * 2);
  const SmemTable<K64> st = smem_table_carve<K64>(smem + off, P.S, q.nwords);
  __shared__ int s_abort;
  __shared__ unsigned s_nmiss;

  // column offsets inside a stage
  size_t coff[GBA_MAX_COLS];
  {
    size_t o = align16(size_t(T) * kb);
#pragma unroll
    for (int c = 0; c < GBA_MAX_COLS; ++c) {
      coff[c] = o;
      if (c < q.ncols) o += align16(size_t(T) * col_bytes(q.col_type[c]));
    }
  }

  smem_table_init<K64, Sig>(st, q);
  if (tid == 0) {
    s_abort = 0;
    s_nmiss = 0;
    if (P.use_tma) {
      for (int s = 0; s < P.nstages; ++s) mbar_init(&bars[s], 1);
      mbar_fence_init();
    }
  }
  __syncthreads();

  auto issue = [&](int64_t tile, int s) {
    unsigned char* dst = stage0 + size_t(s) * sb;
    const int64_t r0 = tile * T;
    uint32_t bytes = uint32_t(size_t(T) * kb);
#pragma unroll
    for (int c = 0; c < GBA_MAX_COLS; ++c)
      if (c < q.ncols) bytes += uint32_t(size_t(T) * col_bytes(q.col_type[c]));
    mbar_arrive_expect_tx(&bars[s], bytes);
    bulk_g2s(dst, static_cast<const unsigned char*>(q.keys) + r0 * kb, uint32_t(size_t(T) * kb), &bars[s]);
#pragma unroll
    for (int c = 0; c < GBA_MAX_COLS; ++c) {
      if (c < q.ncols) {
        const int cb = col_bytes(q.col_type[c]);
        bulk_g2s(dst + coff[c], static_cast<const unsigned char*>(q.cols[c]) + r0 * cb,
                 uint32_t(size_t(T) * cb), &bars[s]);
      }
    }
  };

  // prologue: fill the pipeline
  unsigned pending = 0;  // (thread 0) bit s: stage s has a copy in flight
  if (P.use_tma && tid == 0) {
    for (int s = 0; s < P.nstages; ++s) {
      const int64_t tile = blockIdx.x + int64_t(s) * gridDim.x;
      if (tile < nfull) {
        issue(tile, s);
        pending |= 1u << s;
      }
    }
  }

  const unsigned lane = lane_id();
  unsigned phase = 0;  // bit s = parity to wait for on stage s (flipped only once that phase completed)
  int64_t it = 0;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
    const int s = int(it % P.nstages);
    const int64_t r0 = tile * T;
    const int rows = int(n - r0 < int64_t(T) ? n - r0 : int64_t(T));
    const bool via_tma = P.use_tma && tile < nfull;
    if (via_tma) {
      if (mbar_wait_bounded(&bars[s], (phase >> s) & 1u, P.flags)) {
        phase ^= 1u << s;
        pending &= ~(1u << s);
      } else {
        s_abort = 1;
      }
    }
    __syncthreads();
    if (s_abort) break;
    const unsigned char* sbase = stage0 + size_t(s) * sb;

    tile_two_phase<K64, Sig>(q, P.gt, st, P.S, P.sprobe, P.coalesce, via_tma, sbase, coff, r0, rows, T, miss,
                             &s_nmiss, P.flags);
    __syncthreads();  // stage s and the miss list fully consumed
    if (tid == 0) {
      s_nmiss = 0;
      if (via_tma) {
        const int64_t nxt = tile + int64_t(P.nstages) * gridDim.x;
        if (nxt < nfull) {
          fence_proxy_async_smem();
          issue(nxt, s);
          pending |= 1u << s;
        }
      }
    }
  }

  if (s_abort) {
    // drain: wait (bounded) for every copy this CTA still has in flight, the
    // one whose wait gave up included (its phase bit was not flipped, so the
    // wait is for the same phase), before the CTA's shared memory is released
    if (tid == 0 && P.use_tma) {
      for (int s = 0; s < P.nstages; ++s) {
        if (!(pending >> s & 1u)) continue;
        bool landed = false;
        for (unsigned k = 0; k < (1u << 22) && !landed; ++k) landed = mbar_try_wait(&bars[s], (phase >> s) & 1u);
        if (!landed) atomicOr(P.flags, GBA_FLAG_DRAIN_TIMEOUT);
      }
    }
    return;
  }

  __syncthreads();
  smem_flush_to_gtable<K64, Sig>(q, P.gt, st, P.flags);
}

// Slots first, first + step, ... <= cap (cap is the all-ones key's side slot,
// whose key word is its presence flag) get their key word and identities, one
// slot per iteration (no division of a word index by the slot stride).
__device__ __forceinline__ void init_slots(const GTable& t, int naccs, const unsigned long long (&id)[GBA_MAX_AGGS],
                                           uint64_t first, uint64_t step) {
  const int stride = gba_gt_stride(naccs);
  for (uint64_t slot = first; slot <= t.cap; slot += step) {
    unsigned long long* p = t.base + slot * stride;
    p[0] = slot == t.cap ? 0ull : EMPTY64;
#pragma unroll
    for (int a = 0; a < GBA_MAX_AGGS; ++a)
      if (a < naccs) p[1 + a] = id[a];
  }
}

__global__ void k_table_init(GTable t, int naccs, QDesc q) {
  unsigned long long id[GBA_MAX_AGGS];
#pragma unroll
  for (int a = 0; a < GBA_MAX_AGGS; ++a) id[a] = a < naccs ? acc_identity(q.acc_op[a]) : 0ull;
  init_slots(t, naccs, id, blockIdx.x * uint64_t(blockDim.x) + threadIdx.x, uint64_t(gridDim.x) * blockDim.x);
}

// Compaction of table slots [lo, hi) (hi - lo <= 2048) by a whole CTA of 256
// threads: every thread takes 8 slots, the CTA counts its occupied ones with
// a block scan and reserves their output rows with ONE atomic on the output
// counter, then each thread writes its slots in order.  (Reserving per warp
// put millions of atomics on one counter per query, which serialised in L2.)
constexpr int kCompactThreads = 256, kCompactPer = 8, kCompactSlots = kCompactThreads * kCompactPer;
__device__ __forceinline__ void compact_range(const GTable& t, const QDesc& q, const OutDesc& o, uint64_t lo,
                                              uint64_t hi) {
  __shared__ unsigned s_warp[kCompactThreads / 32];
  __shared__ unsigned long long s_base;
  const int stride = gba_gt_stride(q.naccs);
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  unsigned long long k[kCompactPer];
  unsigned cnt = 0;
#pragma unroll
  for (int j = 0; j < kCompactPer; ++j) {
    const uint64_t i = lo + uint64_t(j) * kCompactThreads + threadIdx.x;
    k[j] = i < hi ? t.base[i * stride] : EMPTY64;
    cnt += k[j] != EMPTY64;
  }
  unsigned x = cnt;  // inclusive warp scan
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned y = __shfl_up_sync(GBA_FULL_MASK, x, d);
    if (int(lane) >= d) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned run = 0;
    for (int w = 0; w < kCompactThreads / 32; ++w) {
      const unsigned c = s_warp[w];
      s_warp[w] = run;
      run += c;
    }
    s_base = run ? atomicAdd(o.count, (unsigned long long)run) : 0ull;
  }
  __syncthreads();
  unsigned long long pos = s_base + s_warp[warp] + (x - cnt);
  const bool K64 = q.key64 != 0;
#pragma unroll
  for (int j = 0; j < kCompactPer; ++j) {
    if (k[j] == EMPTY64) continue;
    const uint64_t i = lo + uint64_t(j) * kCompactThreads + threadIdx.x;
    if (pos < (unsigned long long)o.capacity) {
      if (K64) static_cast<unsigned long long*>(o.keys)[pos] = k[j];
      else static_cast<unsigned*>(o.keys)[pos] = unsigned(k[j]);
#pragma unroll
      for (int a = 0; a < GBA_MAX_AGGS; ++a)
        if (a < q.naccs) o.accs[a][pos] = t.base[i * stride + 1 + a];
    }
    ++pos;
  }
  __syncthreads();  // s_warp / s_base are reused by the next range
}

// the all-ones key's side slot, if present (one thread)
__device__ __forceinline__ void compact_side(const GTable& t, const QDesc& q, const OutDesc& o) {
  const int stride = gba_gt_stride(q.naccs);
  const unsigned long long* side = t.base + t.cap * stride;
  if (side[0] == 0ull) return;
  const unsigned long long pos = atomicAdd(o.count, 1ull);
  if (pos >= (unsigned long long)o.capacity) return;
  if (q.key64) static_cast<unsigned long long*>(o.keys)[pos] = EMPTY64;
  else static_cast<unsigned*>(o.keys)[pos] = EMPTY32;
#pragma unroll
  for (int a = 0; a < GBA_MAX_AGGS; ++a)
    if (a < q.naccs) o.accs[a][pos] = side[1 + a];
}

__global__ void __launch_bounds__(kCompactThreads) k_compact(GTable t, QDesc q, OutDesc o) {
  for (uint64_t lo = uint64_t(blockIdx.x) * kCompactSlots; lo < t.cap; lo += uint64_t(gridDim.x) * kCompactSlots)
    compact_range(t, q, o, lo, lo + kCompactSlots < t.cap ? lo + kCompactSlots : t.cap);
  if (blockIdx.x == 0 && threadIdx.x == 0) compact_side(t, q, o);
}

// ---- batched queries: table init and compaction (the aggregation itself is
// k_stream.cu's streaming kernel) ----
// table init for every query of a batch: blocks are dealt to queries in
// proportion to their table sizes (blk_prefix[i] = first block of query i)
__device__ __forceinline__ int batch_query_of_block(const int64_t* blk_prefix, int nq, int64_t b) {
  int lo = 0, hi = nq - 1;
  while (lo < hi) {  // largest i with blk_prefix[i] <= b
    const int mid = (lo + hi + 1) >> 1;
    if (blk_prefix[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(256) k_batch_init(const BatchQ* qs, const int64_t* blk_prefix, int nq,
                                                    int64_t block0) {
  const int64_t blk = block0 + int64_t(blockIdx.x);
  const int qi = batch_query_of_block(blk_prefix, nq, blk);
  const int64_t b = blk - blk_prefix[qi];
  const int64_t nb = blk_prefix[qi + 1] - blk_prefix[qi];
  const GTable t = qs[qi].gt;
  const QDesc& q = qs[qi].q;
  unsigned long long id[GBA_MAX_AGGS];
#pragma unroll
  for (int a = 0; a < GBA_MAX_AGGS; ++a) id[a] = a < q.naccs ? acc_identity(q.acc_op[a]) : 0ull;
  init_slots(t, q.naccs, id, uint64_t(b) * blockDim.x + threadIdx.x, uint64_t(nb) * blockDim.x);
}

// compaction of every query of a batch into its own output (blocks dealt as
// in k_batch_init, one block per 2048 slots; block 0 of a query also emits
// its all-ones-key side slot)
__global__ void __launch_bounds__(kCompactThreads) k_batch_compact(const BatchQ* qs, const int64_t* blk_prefix,
                                                                   int nq, int64_t block0) {
  const int64_t blk = block0 + int64_t(blockIdx.x);
  const int qi = batch_query_of_block(blk_prefix, nq, blk);
  const int64_t b = blk - blk_prefix[qi];
  const int64_t nb = blk_prefix[qi + 1] - blk_prefix[qi];
  const GTable t = qs[qi].gt;
  const QDesc q = qs[qi].q;
  const OutDesc o = qs[qi].out;
  for (uint64_t lo = uint64_t(b) * kCompactSlots; lo < t.cap; lo += uint64_t(nb) * kCompactSlots)
    compact_range(t, q, o, lo, lo + kCompactSlots < t.cap ? lo + kCompactSlots : t.cap);
  if (b == 0 && threadIdx.x == 0) compact_side(t, q, o);
}

__global__ void k_avg_finish(AvgDesc d, int64_t rows) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < rows; r += int64_t(gridDim.x) * blockDim.x) {
    const double c = double(d.count[r]);
#pragma unroll
    for (int i = 0; i < GBA_MAX_AGGS; ++i) {
      if (i >= d.n) break;
      const unsigned long long x = d.col[i][r];
      const double sum = d.fp[i] ? __longlong_as_double(x) : double((long long)x);
      d.col[i][r] = __double_as_longlong(sum / c);
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Host launchers.
cudaError_t gba_launch_avg_finish(const AvgDesc& d, int64_t rows, int sms, cudaStream_t s) {
  const int64_t want = (rows + 255) / 256;
  k_avg_finish<<<int(want < int64_t(sms) * 8 ? want : int64_t(sms) * 8), 256, 0, s>>>(d, rows);
  return cudaGetLastError();
}

size_t gba_preagg_smem_bytes(const QDesc& q, int S, int T, int nstages, int use_tma) {
  size_t b = 128;
  if (use_tma) b += stage_bytes(q, T) * nstages;
  b += align16(size_t(T) * 2);  // miss list
  b += smem_table_bytes(S, q.key64, q.nwords);
  return b;
}

cudaError_t gba_launch_table_init(const GTable& t, const QDesc& q, int grid, cudaStream_t s) {
  k_table_init<<<grid, 256, 0, s>>>(t, q.naccs, q);
  return cudaGetLastError();
}

cudaError_t gba_launch_preagg(const QDesc& q, const GTable& t, const PreaggCfg& c, unsigned* flags,
                              cudaStream_t s) {
  PreaggParams P;
  P.q = q;
  P.gt = t;
  P.S = c.smem_slots;
  P.sprobe = c.smem_probe_cap;
  P.T = c.tile_rows;
  P.nstages = c.nstages < 1 ? 1 : (c.nstages > kMaxStages ? kMaxStages : c.nstages);
  P.use_tma = c.use_tma;
  P.coalesce = c.coalesce;
  P.flags = flags;
  const size_t smem = gba_preagg_smem_bytes(q, P.S, P.T, P.nstages, P.use_tma);
  return gba_dispatch_sig(q, [&](auto K, auto sig) -> cudaError_t {
    constexpr bool k64 = decltype(K)::value;
    using Sig = decltype(sig);
    cudaError_t e = gba_allow_max_smem(k_preagg<k64, Sig>);
    if (e != cudaSuccess) return e;
    k_preagg<k64, Sig><<<c.grid, c.block, smem, s>>>(P);
    return cudaGetLastError();
  });
}

cudaError_t gba_launch_compact(const GTable& t, const QDesc& q, const OutDesc& o, int grid, cudaStream_t s) {
  k_compact<<<grid, kCompactThreads, 0, s>>>(t, q, o);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
size_t gba_batch_static_smem() { return sizeof(BatchQ) + 64; }

int gba_batch_sig_id(const QDesc& q) {
  int id = -1;
  gba_dispatch_sig(q, [&](auto, auto sig) -> cudaError_t {
    id = gba_sig_index(decltype(sig){});
    return cudaSuccess;
  });
  return id;
}

cudaError_t gba_launch_batch_init(const BatchQ* d_qs, const int64_t* blk_prefix, int nq, int64_t nblocks,
                                  int64_t block0, cudaStream_t s) {
  if (nq <= 0 || nblocks <= 0) return cudaSuccess;
  k_batch_init<<<unsigned(nblocks), 256, 0, s>>>(d_qs, blk_prefix, nq, block0);
  return cudaGetLastError();
}

cudaError_t gba_launch_batch_compact(const BatchQ* d_qs, const int64_t* blk_prefix, int nq, int64_t nblocks,
                                     int64_t block0, cudaStream_t s) {
  if (nq <= 0 || nblocks <= 0) return cudaSuccess;
  k_batch_compact<<<unsigned(nblocks), kCompactThreads, 0, s>>>(d_qs, blk_prefix, nq, block0);
  return cudaGetLastError();
}
