// Row processing shared by the streaming aggregation kernels (k_stream.cu:
// rows loaded into registers by each warp; k_stream_tma.cu: rows staged in
// shared memory by bulk copies).  Included inside each kernel file's
// anonymous namespace, after batch_kernels.h, gba_internal.cuh and
// smem_table.cuh.
#pragma once

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
    // column w: low halves (a COUNT's only column) at lo32[slot], high halves
    // in the next column, lo32[SS + slot]
    unsigned* lo32 = reinterpret_cast<unsigned*>(t.acc) + size_t(w) * t.SS;
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
        if (add_hi) atomicAdd(lo32 + t.SS + slot[i], add_hi);
      }
    } else {
#pragma unroll
      for (int i = 0; i < R; ++i) {
        if (!(rows >> i & 1u)) continue;
        if (op == ACC_ADD_F)
          smem_fsum(smem_ref<K64>(t, w, slot[i]), smem_ref<K64>(t, w + 2, slot[i]), smem_ref<K64>(t, w + 4, slot[i]),
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


// HBM-table pass over the rows of `miss` (h: their table hashes): every such
// row's home-slot load first, then the inserts, so a thread keeps R
// independent L2 requests in flight (measured: also loading the slot after the
// home slot, to place displaced keys without a second round trip, costs more
// in L2 requests than it saves).
template <bool K64, typename Sig, int R>
__device__ __forceinline__ void hbm_rows(const BatchQ& bq, const uint64_t (&key)[R],
                                         const unsigned long long (&v)[R][Sig::NA], const uint32_t (&h)[R],
                                         unsigned miss) {
  constexpr int NA = Sig::NA;
  constexpr int stride = gba_gt_stride(NA);
  const QDesc& q = bq.q;
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

// The shared-table pass over a thread's R rows (key[i], accumulator
// contributions v[i], table hashes h[i]; rows whose bit in `live` is clear
// are skipped), phase by phase so that their shared-memory round trips
// overlap: first every row's home bucket, then the rows that did not find
// their key there walk the probe sequence (nbk buckets), then the
// accumulator updates of all rows are issued before any result is used.
// Returns the rows whose key is not in the table and cannot enter it.
template <bool K64, typename Sig, int R>
__device__ __forceinline__ unsigned smem_rows(const SmemTable<K64>& st, const QDesc& q, int nbk,
                                              const uint64_t (&key)[R], const unsigned long long (&v)[R][Sig::NA],
                                              const bool (&live)[R], const uint32_t (&h)[R]) {
  typedef typename SmemTable<K64>::KeyW KeyW;
  constexpr int SPB = BucketT<K64>::SPB;
  const uint64_t emptyk = K64 ? EMPTY64 : uint64_t(EMPTY32);
  unsigned miss = 0;
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
  return miss;
}

// A thread's R rows into the item's shared table, or, for rows whose key is
// not in it and cannot enter it, into the query's HBM table.
template <bool K64, typename Sig, int R>
__device__ __forceinline__ void stream_rows(const BatchQ& bq, const SmemTable<K64>& st, int nbk, const uint64_t (&key)[R],
                                            const unsigned long long (&v)[R][Sig::NA], const bool (&live)[R]) {
  const QDesc& q = bq.q;
  const uint64_t emptyk = K64 ? EMPTY64 : uint64_t(EMPTY32);
  unsigned miss = 0;
  uint32_t h[R];
#pragma unroll
  for (int i = 0; i < R; ++i) h[i] = table_hash(key[i]);
  if (bq.S > 0) {
    miss = smem_rows<K64, Sig, R>(st, q, nbk, key, v, live, h);
  } else {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      if (!live[i]) continue;
      if (key[i] == emptyk) gtable_insert<K64, Sig>(bq.gt, q, key[i], 0u, v[i], bq.flags);
      else miss |= 1u << i;
    }
  }
  if (miss == 0) return;
  hbm_rows<K64, Sig, R>(bq, key, v, h, miss);
}

// A thread's R rows straight into the query's HBM table (a query without a
// shared table: BatchQ.S == 0).
template <bool K64, typename Sig, int R>
__device__ __forceinline__ void stream_rows_hbm(const BatchQ& bq, const uint64_t (&key)[R],
                                                const unsigned long long (&v)[R][Sig::NA], const bool (&live)[R]) {
  const uint64_t emptyk = K64 ? EMPTY64 : uint64_t(EMPTY32);
  uint32_t h[R];
  unsigned miss = 0;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    h[i] = table_hash(key[i]);
    if (!live[i]) continue;
    if (key[i] == emptyk) gtable_insert<K64, Sig>(bq.gt, bq.q, key[i], 0u, v[i], bq.flags);
    else miss |= 1u << i;
  }
  if (miss) hbm_rows<K64, Sig, R>(bq, key, v, h, miss);
}

// ---------------------------------------------------------------------------
// A table spread over the CL CTAs of a thread-block cluster (distributed
// shared memory): each CTA's shared table holds nb = S / SPB buckets of the
// whole table's CL * nb; a row's hash picks a bucket of the whole table,
// which lives in CTA owner = bucket / nb, and its probes stay inside that
// CTA's buckets.  Every access goes through the shared::cluster window
// (bucket loads, claims by compare-and-swap, accumulator atomics).  Integer
// SUM and COUNT only: the signatures a cluster launch is made for.
template <typename Sig>
struct ClusterSig {
  static constexpr bool ok = false;
};
template <int... C>
struct ClusterSig<SigCT<C...>> {
  static constexpr bool ok = ((((C & 15) == ACC_CNT) || ((C & 15) == ACC_ADD_I)) && ...);
};

template <bool K64>
__device__ __forceinline__ void dsmem_ld_bucket(uint32_t addr, typename SmemTable<K64>::KeyW (&o)[BucketT<K64>::SPB]) {
  unsigned x0, x1, x2, x3;
  dsmem_ld_v4(addr, x0, x1, x2, x3);
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

// slot (inside the owner's table) of `key`, inserting it if absent, walking at
// most max_buckets of the owner's buckets from bucket b; -1 when all are full
// without it.  keys_addr: the owner's key array in the shared::cluster window.
template <bool K64>
__device__ __noinline__ int cluster_find_or_insert(uint32_t keys_addr, int nb, int b, uint64_t key, int max_buckets) {
  constexpr int SPB = BucketT<K64>::SPB;
  constexpr int kb = K64 ? 8 : 4;
  typedef typename SmemTable<K64>::KeyW KeyW;
  const KeyW kk = KeyW(key), empty = smem_empty_key<K64>();
  for (int p = 0; p < max_buckets; ++p) {
    for (int tries = 0; tries <= SPB; ++tries) {
      KeyW k[SPB];
      dsmem_ld_bucket<K64>(keys_addr + uint32_t(b) * 16u, k);
      int free_e = -1;
#pragma unroll
      for (int e = SPB - 1; e >= 0; --e) {
        if (k[e] == kk) return b * SPB + e;
        if (k[e] == empty) free_e = e;
      }
      if (free_e < 0) break;
      const uint32_t a = keys_addr + uint32_t(b * SPB + free_e) * kb;
      KeyW prev;
      if constexpr (K64) prev = dsmem_cas_b64(a, empty, kk);
      else prev = dsmem_cas_b32(a, empty, kk);
      if (prev == empty || prev == kk) return b * SPB + free_e;
    }
    b = b + 1 == nb ? 0 : b + 1;
  }
  return -1;
}

template <bool K64, typename Sig, int R>
__device__ __forceinline__ void stream_rows_cluster(const BatchQ& bq, const SmemTable<K64>& st, int nbk, int CL,
                                                    const uint64_t (&key)[R], const unsigned long long (&v)[R][Sig::NA],
                                                    const bool (&live)[R]) {
  static_assert(ClusterSig<Sig>::ok, "cluster tables take integer SUM and COUNT only");
  constexpr int NA = Sig::NA;
  constexpr int SPB = BucketT<K64>::SPB;
  typedef typename SmemTable<K64>::KeyW KeyW;
  const QDesc& q = bq.q;
  const uint64_t emptyk = K64 ? EMPTY64 : uint64_t(EMPTY32);
  const int nb = st.S / SPB;
  const uint32_t keys_local = smem_u32(st.keys), acc_local = smem_u32(st.acc);
  uint32_t h[R];
  unsigned owner[R];
  int b[R];
  KeyW kb[R][SPB];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    h[i] = table_hash(key[i]);
    const unsigned gb = unsigned((uint64_t(h[i]) * unsigned(nb * CL)) >> 32);
    owner[i] = gb / unsigned(nb);
    b[i] = int(gb - owner[i] * unsigned(nb));
    if (live[i]) dsmem_ld_bucket<K64>(dsmem_map(keys_local, owner[i]) + uint32_t(b[i]) * 16u, kb[i]);
  }
  int slot[R];
  unsigned hit = 0, miss = 0;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    slot[i] = -1;
    if (!live[i]) continue;
    if (key[i] == emptyk) {  // the all-ones key: this CTA's own side slot
      smem_apply_side<K64, Sig>(st, q, v[i]);
      continue;
    }
    bool has_empty = false;
#pragma unroll
    for (int e = 0; e < SPB; ++e) {
      if (kb[i][e] == KeyW(key[i])) slot[i] = b[i] * SPB + e;
      has_empty = has_empty || kb[i][e] == smem_empty_key<K64>();
    }
    if (slot[i] < 0 && (has_empty || nbk > 1))
      slot[i] = cluster_find_or_insert<K64>(dsmem_map(keys_local, owner[i]), nb, b[i], key[i], nbk);
    if (slot[i] >= 0) hit |= 1u << i;
    else miss |= 1u << i;
  }
#pragma unroll
  for (int a = 0; a < NA; ++a) {
    const uint32_t lo_local = acc_local + uint32_t(Sig::woff(q, a)) * uint32_t(st.SS) * 4u;
    if (Sig::op(q, a) == ACC_CNT) {
#pragma unroll
      for (int i = 0; i < R; ++i)
        if (hit >> i & 1u) dsmem_red_add_u32(dsmem_map(lo_local, owner[i]) + uint32_t(slot[i]) * 4u, unsigned(v[i][a]));
    } else {
      unsigned old[R];
#pragma unroll
      for (int i = 0; i < R; ++i) {
        old[i] = 0u;
        if (hit >> i & 1u)
          old[i] = dsmem_atom_add_u32(dsmem_map(lo_local, owner[i]) + uint32_t(slot[i]) * 4u, unsigned(v[i][a]));
      }
#pragma unroll
      for (int i = 0; i < R; ++i) {
        if (!(hit >> i & 1u)) continue;
        const unsigned lo = unsigned(v[i][a]), hi = unsigned(v[i][a] >> 32);
        const unsigned add_hi = hi + ((old[i] + lo) < old[i] ? 1u : 0u);
        if (add_hi)
          dsmem_red_add_u32(dsmem_map(lo_local, owner[i]) + uint32_t(st.SS + slot[i]) * 4u, add_hi);
      }
    }
  }
  if (miss) hbm_rows<K64, Sig, R>(bq, key, v, h, miss);
}
