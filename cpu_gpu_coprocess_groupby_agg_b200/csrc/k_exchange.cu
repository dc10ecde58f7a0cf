// Owner-exchange aggregation (sm_100a): the batch kernel for queries whose
// groups outgrow one CTA's shared table but fit the shared tables of all SMs
// together.
//
// Replaces, for those queries, the reference's spill of a tile's leftover rows
// to an unbounded global linear-probe table (tiled_groupby_agg_partition/src/
// kernel.cu:116-158) and the per-partition global table of phase 2
// (kernel.cu:294-351): here no row's aggregate goes through an HBM table.
//
// One cooperative launch, one CTA of 512 threads per SM.  CTA c owns the keys
// whose owner hash falls in the c-th of grid equal ranges, and holds their
// groups in its shared-memory table for the whole query.  A query's rows are
// taken in windows of `win` rows:
//   A  (route)  every CTA reads its slice of the window (coalesced streaming
//               loads), counts its rows per owner in shared memory, reserves
//               each owner's run with one global atomic per owner and tile,
//               and writes every row, as a record (key, then each value
//               column, 8 bytes each), into its owner's region of the
//               window's exchange buffer;
//   (a grid barrier: every record of the window written)
//   B  (reduce) every CTA reads the records of its own region and applies
//               them to its shared table (stream_rows.cuh: the same probe and
//               32-bit atomics as the streaming kernels; a key whose probe
//               window is full goes to the query's HBM table).
// Two exchange buffers of buf_words words each alternate between windows
// (buf_words holds grid regions of `region` records of the widest record any
// phase writes: a buffer's rows of one window and the other buffer's partial
// records never overlap), so the records of one
// window are read while the next window's are written; a buffer of
// win x record bytes stays in L2 between its writes and its reads, so the
// rows cross HBM once.  After a query's last window every CTA writes the
// groups of its table straight to the query's output (one atomic per CTA
// reserves its rows); keys that went to the HBM table are written by the
// batch's compaction kernel after the launch, so a group is written once.
//
// Skewed keys: a query with bits 16..27 of BatchQ.pad set gives every CTA a
// small "hot" table of 4 x that many slots beside its owner table.  In A a
// row whose key is in the CTA's hot table, or can enter its home bucket there,
// is aggregated on the spot instead of routed, so a key that takes a large
// share of the rows does not load its owner alone.  After the query's last
// window every CTA routes its hot table's groups as partial records (key and
// accumulator values) to their owners, which merge them like rows.
//
// The grid barrier is a counter and a generation word in global memory with
// a bounded wait (GBA_FLAG_WAIT_TIMEOUT; a CTA that gives up returns, and the
// others give up at their next barrier).  The launch is cooperative, so all
// CTAs are resident together.
#include "batch_kernels.h"
#include "gba_internal.cuh"
#include "smem_table.cuh"

namespace {
#include "stream_rows.cuh"

constexpr int kXThreads = 512;
constexpr int kXRows = 4;                       // rows per thread per tile
constexpr int kXTile = kXThreads * kXRows;      // rows per tile
constexpr int kXMaxGrid = 1024;

// Grid-wide barrier of a cooperative launch, bounded: false when the wait
// gave up (the timeout flag is raised).
__device__ bool grid_barrier(unsigned* count, unsigned* gen, unsigned nblocks, unsigned* flags, int* s_fail) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned g = *(volatile unsigned*)gen;
    __threadfence();  // this CTA's writes before its arrival
    if (atomicAdd(count, 1u) == nblocks - 1) {
      *(volatile unsigned*)count = 0u;
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      bool ok = false;
      for (unsigned it = 0; it < (1u << 24) && !ok; ++it) {
        ok = *(volatile unsigned*)gen != g;
        if (!ok) __nanosleep(64);
      }
      if (!ok) {
        atomicOr(flags, GBA_FLAG_WAIT_TIMEOUT);
        *s_fail = 1;
      }
    }
    __threadfence();  // the other CTAs' writes before this CTA's next reads
  }
  __syncthreads();
  return *s_fail == 0;
}

template <bool K64, typename Sig>
__global__ void __launch_bounds__(kXThreads, 1)
    k_exchange_agg(const BatchQ* qs, const int* xq, int nxq, int64_t win, unsigned long long* xbuf, int64_t region,
                   int64_t buf_words, unsigned* cursors, unsigned* bar, unsigned* bar_flags, int sprobe) {
  constexpr int NA = Sig::NA;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned s_cnt[kXMaxGrid];
  __shared__ unsigned s_base[kXMaxGrid];
  __shared__ unsigned s_warp[kXThreads / 32];
  __shared__ unsigned long long s_out;
  __shared__ int s_fail;
  __shared__ __align__(16) BatchQ s_q;
  const int tid = threadIdx.x;
  const unsigned lane = lane_id(), warp = unsigned(tid) >> 5;
  const unsigned G = gridDim.x, me = blockIdx.x;
  for (unsigned o = tid; o < G; o += blockDim.x) s_cnt[o] = 0u;
  if (tid == 0) s_fail = 0;
  __syncthreads();
  int64_t wglob = 0;  // windows done by the launch (selects the exchange buffer)
  for (int x = 0; x < nxq; ++x) {
    {
      const unsigned* src = reinterpret_cast<const unsigned*>(qs + xq[x]);
      unsigned* dst = reinterpret_cast<unsigned*>(&s_q);
      for (int w = tid; w < int(sizeof(BatchQ) / 4); w += blockDim.x) dst[w] = src[w];
    }
    __syncthreads();
    const QDesc& q = s_q.q;
    const int ncols = Sig::ncols(q);
    const int stride = 1 + ncols;  // record words
    const SmemTable<K64> st = smem_table_carve<K64>(smem, s_q.S, Sig::nwords(q));
    smem_table_init<K64, Sig>(st, q);
    const int hot = ((s_q.pad >> 16) & 4095) * 4;  // hot-table slots (0: none)
    const SmemTable<K64> ht = smem_table_carve<K64>(
        smem + ((smem_table_bytes(s_q.S, K64, Sig::nwords(q)) + 127) & ~size_t(127)), hot, Sig::nwords(q));
    if (hot > 0) smem_table_init<K64, Sig>(ht, q);
    const int nbk = (s_q.pad >> 8) & 255 ? (s_q.pad >> 8) & 255 : sprobe;
    __syncthreads();
    const int64_t n = q.n;
    for (int64_t w0 = 0; w0 < n; w0 += win, ++wglob) {
      const int b = int(wglob & 1);
      unsigned long long* buf = xbuf + size_t(b) * size_t(buf_words);
      unsigned* cur = cursors + size_t(b) * G;
      // ---- A: route this CTA's slice of the window to the owners ----
      const int64_t we = w0 + win < n ? w0 + win : n;
      const int64_t slice = ((we - w0 + G - 1) / G + kXTile - 1) / kXTile * kXTile;
      const int64_t sb = w0 + slice * me < we ? w0 + slice * me : we;
      const int64_t se = sb + slice < we ? sb + slice : we;
      for (int64_t t0 = sb; t0 < se; t0 += kXTile) {
        uint64_t key[kXRows];
        unsigned long long raw[kXRows][GBA_MAX_COLS];
        unsigned own[kXRows], rank[kXRows];
        bool live[kXRows];
#pragma unroll
        for (int i = 0; i < kXRows; ++i) {
          const int64_t r = t0 + tid + int64_t(kXThreads) * i;
          live[i] = r < se;
          key[i] = K64 ? EMPTY64 : uint64_t(EMPTY32);
#pragma unroll
          for (int c = 0; c < GBA_MAX_COLS; ++c) raw[i][c] = 0ull;
          if (live[i]) {
            key[i] = K64 ? __ldcs(static_cast<const unsigned long long*>(q.keys) + r)
                         : __ldcs(static_cast<const unsigned*>(q.keys) + r);
#pragma unroll
            for (int c = 0; c < GBA_MAX_COLS; ++c)
              if (c < ncols)
                raw[i][c] = gba_type_bytes(Sig::coltype(q, c)) == 8
                                ? __ldcs(static_cast<const unsigned long long*>(q.cols[c]) + r)
                                : __ldcs(static_cast<const unsigned*>(q.cols[c]) + r);
          }
        }
        if (hot > 0) {  // keys of the hot table are aggregated here, the rest routed
          unsigned long long v[kXRows][NA];
#pragma unroll
          for (int i = 0; i < kXRows; ++i) row_contrib<Sig>(q, raw[i], v[i]);
          uint32_t hh[kXRows];
#pragma unroll
          for (int i = 0; i < kXRows; ++i) hh[i] = table_hash(key[i]);
          const unsigned miss = smem_rows<K64, Sig, kXRows>(ht, q, 1, key, v, live, hh);
#pragma unroll
          for (int i = 0; i < kXRows; ++i) live[i] = (miss >> i) & 1u;
        }
#pragma unroll
        for (int i = 0; i < kXRows; ++i) {
          own[i] = ~0u;
          if (live[i]) {
            own[i] = unsigned((uint64_t(part_hash(key[i])) * G) >> 32);
            rank[i] = atomicAdd(&s_cnt[own[i]], 1u);
          }
        }
        __syncthreads();
        for (unsigned o = tid; o < G; o += blockDim.x) {
          const unsigned c = s_cnt[o];
          s_base[o] = c ? atomicAdd(&cur[o], c) : 0u;
          s_cnt[o] = 0u;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kXRows; ++i) {
          if (own[i] == ~0u) continue;
          const uint64_t pos = uint64_t(s_base[own[i]]) + rank[i];  // < region: a window has win <= region rows
          unsigned long long* rec = buf + (uint64_t(own[i]) * uint64_t(region) + pos) * stride;
          if (stride == 2) {  // one 16-byte store (records of an even word count are 16-byte aligned)
            *reinterpret_cast<ulonglong2*>(rec) = make_ulonglong2(key[i], raw[i][0]);
          } else {
            rec[0] = key[i];
#pragma unroll
            for (int c = 0; c < GBA_MAX_COLS; ++c)
              if (c < ncols) rec[1 + c] = raw[i][c];
          }
        }
      }
      if (!grid_barrier(bar, bar + 1, G, bar_flags, &s_fail)) return;
      // ---- B: this CTA's records into its shared table ----
      const unsigned cnt = __ldcg(&cur[me]);
      const unsigned long long* mine = buf + uint64_t(me) * uint64_t(region) * stride;
      for (unsigned r0 = 0; r0 < cnt; r0 += kXTile) {
        uint64_t k2[kXRows];
        unsigned long long v[kXRows][NA];
        bool live[kXRows];
#pragma unroll
        for (int i = 0; i < kXRows; ++i) {
          const unsigned r = r0 + tid + kXThreads * i;
          live[i] = r < cnt;
          k2[i] = K64 ? EMPTY64 : uint64_t(EMPTY32);
          unsigned long long raw[GBA_MAX_COLS] = {0ull, 0ull, 0ull, 0ull};
          if (live[i]) {
            const unsigned long long* rec = mine + uint64_t(r) * stride;
            if (stride == 2) {
              const ulonglong2 x = __ldcg(reinterpret_cast<const ulonglong2*>(rec));
              k2[i] = x.x;
              raw[0] = x.y;
            } else {
              k2[i] = __ldcg(rec);
#pragma unroll
              for (int c = 0; c < GBA_MAX_COLS; ++c)
                if (c < ncols) raw[c] = __ldcg(rec + 1 + c);
            }
          }
          row_contrib<Sig>(q, raw, v[i]);
        }
        stream_rows<K64, Sig, kXRows>(s_q, st, nbk, k2, v, live);
      }
      __syncthreads();
      if (tid == 0) cur[me] = 0u;  // the buffer's next writers start after the next barrier
    }
    if (hot > 0) {
      // ---- the hot tables' groups to their owners, as partial records ----
      const int b = int(wglob & 1);
      const int pstride = 1 + NA;
      unsigned long long* buf = xbuf + size_t(b) * size_t(buf_words);
      unsigned* cur = cursors + size_t(b) * G;
      for (int i = tid; i <= hot; i += kXThreads) {
        uint64_t k;
        if (i < hot) {
          k = uint64_t(ht.keys[i]);
          if (k == uint64_t(smem_empty_key<K64>())) continue;
        } else {
          if (!*ht.side_present()) continue;
          k = K64 ? EMPTY64 : uint64_t(EMPTY32);
        }
        const unsigned o = unsigned((uint64_t(part_hash(k)) * G) >> 32);
        const unsigned pos = atomicAdd(&cur[o], 1u);  // < hot + 1 per CTA: within the region
        unsigned long long* rec = buf + (uint64_t(o) * uint64_t(region) + pos) * pstride;
        rec[0] = k;
#pragma unroll
        for (int a = 0; a < NA; ++a) rec[1 + a] = smem_acc_read<K64, Sig>(ht, q, a, i < hot ? i : -1);
      }
      if (!grid_barrier(bar, bar + 1, G, bar_flags, &s_fail)) return;
      const unsigned cnt = __ldcg(&cur[me]);
      const unsigned long long* mine = buf + uint64_t(me) * uint64_t(region) * pstride;
      for (unsigned r0 = 0; r0 < cnt; r0 += kXTile) {
        uint64_t k2[kXRows];
        unsigned long long v[kXRows][NA];
        bool live[kXRows];
#pragma unroll
        for (int i = 0; i < kXRows; ++i) {
          const unsigned r = r0 + tid + kXThreads * i;
          live[i] = r < cnt;
          k2[i] = K64 ? EMPTY64 : uint64_t(EMPTY32);
#pragma unroll
          for (int a = 0; a < NA; ++a) v[i][a] = acc_identity(Sig::op(q, a));
          if (live[i]) {
            const unsigned long long* rec = mine + uint64_t(r) * pstride;
            k2[i] = __ldcg(rec);
#pragma unroll
            for (int a = 0; a < NA; ++a) v[i][a] = __ldcg(rec + 1 + a);  // partial values merge as contributions
          }
        }
        stream_rows<K64, Sig, kXRows>(s_q, st, nbk, k2, v, live);
      }
      __syncthreads();
      if (tid == 0) cur[me] = 0u;
      ++wglob;
    }
    // ---- the query's groups of this CTA's table, straight to its output ----
    __syncthreads();
    {
      const OutDesc& o = s_q.out;
      const int per = (st.S + kXThreads - 1) / kXThreads;
      unsigned cnt = 0;
      for (int j = 0; j < per; ++j) {
        const int i = tid * per + j;
        if (i < st.S && uint64_t(st.keys[i]) != uint64_t(smem_empty_key<K64>())) ++cnt;
      }
      unsigned xs = cnt;  // inclusive warp scan
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const unsigned y = __shfl_up_sync(GBA_FULL_MASK, xs, d);
        if (int(lane) >= d) xs += y;
      }
      if (lane == 31) s_warp[warp] = xs;
      __syncthreads();
      if (tid == 0) {
        unsigned run = 0;
        for (int w = 0; w < kXThreads / 32; ++w) {
          const unsigned c = s_warp[w];
          s_warp[w] = run;
          run += c;
        }
        const unsigned side = *st.side_present() ? 1u : 0u;
        s_out = run + side ? atomicAdd(o.count, (unsigned long long)(run + side)) : 0ull;
        if (side) {  // the all-ones key's group, after this CTA's others
          const unsigned long long pos = s_out + run;
          if (pos < (unsigned long long)o.capacity) {
            if (K64) static_cast<unsigned long long*>(o.keys)[pos] = EMPTY64;
            else static_cast<unsigned*>(o.keys)[pos] = EMPTY32;
#pragma unroll
            for (int a = 0; a < NA; ++a) o.accs[a][pos] = smem_acc_read<K64, Sig>(st, q, a, -1);
          }
        }
      }
      __syncthreads();
      unsigned long long pos = s_out + s_warp[warp] + (xs - cnt);
      for (int j = 0; j < per; ++j) {
        const int i = tid * per + j;
        if (i >= st.S || uint64_t(st.keys[i]) == uint64_t(smem_empty_key<K64>())) continue;
        if (pos < (unsigned long long)o.capacity) {
          if (K64) static_cast<unsigned long long*>(o.keys)[pos] = st.keys[i];
          else static_cast<unsigned*>(o.keys)[pos] = unsigned(st.keys[i]);
#pragma unroll
          for (int a = 0; a < NA; ++a) o.accs[a][pos] = smem_acc_read<K64, Sig>(st, q, a, i);
        }
        ++pos;
      }
    }
    __syncthreads();  // s_q and the table are rewritten by the next query
  }
}

}  // namespace

// ---------------------------------------------------------------------------
size_t gba_exchange_smem_bytes(const QDesc& q, int S, int hot) {
  return ((smem_table_bytes(S, q.key64, q.nwords) + 127) & ~size_t(127)) +
         (hot > 0 ? smem_table_bytes(hot, q.key64, q.nwords) : 0) + 64;
}

size_t gba_exchange_static_smem() { return 2 * kXMaxGrid * 4 + sizeof(BatchQ) + 256; }

cudaError_t gba_prepare_exchange(const QDesc& proto) {
  return gba_dispatch_sig(proto, [&](auto K, auto sig) -> cudaError_t {
    return gba_allow_max_smem(k_exchange_agg<decltype(K)::value, decltype(sig)>);
  });
}

int gba_exchange_grid(const QDesc& proto, size_t smem, int sms) {
  int per_sm = 0;
  gba_dispatch_sig(proto, [&](auto K, auto sig) -> cudaError_t {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_exchange_agg<decltype(K)::value, decltype(sig)>,
                                                      kXThreads, smem) != cudaSuccess) {
      cudaGetLastError();
      per_sm = 0;
    }
    return cudaSuccess;
  });
  return per_sm >= 1 ? std::min(sms, kXMaxGrid) : 0;
}

cudaError_t gba_launch_exchange(const QDesc& proto, const BatchQ* d_qs, const int* d_xq, int nxq, int64_t win,
                                unsigned long long* xbuf, int64_t region, int64_t buf_words, unsigned* cursors,
                                unsigned* bar, unsigned* bar_flags, size_t smem, int sprobe, int grid, cudaStream_t s) {
  if (nxq <= 0) return cudaSuccess;
  if (grid < 1 || grid > kXMaxGrid || win > region) return cudaErrorInvalidValue;
  return gba_dispatch_sig(proto, [&](auto K, auto sig) -> cudaError_t {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(kXThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_exchange_agg<decltype(K)::value, decltype(sig)>, d_qs, d_xq, nxq, win, xbuf,
                              region, buf_words, cursors, bar, bar_flags, sprobe);
  });
}
