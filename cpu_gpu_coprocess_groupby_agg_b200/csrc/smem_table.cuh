// Shared-memory open-addressing aggregation table, shared by the
// pre-aggregation kernel and the per-partition aggregation kernel.
//
// Measured on B200 (sm_100a): shared-memory 32-bit atomicAdd runs at about
// 3.4 T ops/s, 64-bit atomicAdd at about 0.5 T ops/s.  Accumulators are
// therefore updated with 32-bit atomics wherever that stays exact:
//   COUNT      32-bit add on the low word (a table lives for fewer than 2^32
//              rows of one CTA)
//   SUM int64  32-bit add on the low word; the add's own carry out of the
//              low word is added to the high word with a second 32-bit add,
//              issued only when nonzero.  The final 64-bit value is exactly
//              the sum mod 2^64 because each carry is produced and accounted
//              by the add that caused it.
//   MIN / MAX  read first; the 64-bit atomic is issued only when the row
//              improves on the value read (values only move one way, so a
//              stale read can only cause an extra atomic, never a wrong skip).
//   SUM fp32   fp64 atomicAdd.
// Sig (template) is the query's aggregate signature (sig.cuh).
#pragma once
#include <type_traits>

#include "gba_internal.cuh"
#include "sig.cuh"

template <bool K64>
struct SmemTable {
  typedef typename std::conditional<K64, unsigned long long, unsigned>::type KeyW;
  KeyW* keys;
  unsigned long long* acc;  // nw columns of SS 4-byte words
  int S;
  int SS;  // column length: S rounded up to even, so every column starts 8-byte aligned
  int nw;  // 4-byte words per slot
  // after the columns: one 8-byte word per column index for the all-ones
  // key's accumulators (6 per accumulator at most), then its presence flag
  // (computed where used: fewer registers live through the row loops)
  __device__ __forceinline__ unsigned long long* side() const {
    return reinterpret_cast<unsigned long long*>(reinterpret_cast<unsigned*>(acc) + size_t(SS) * nw);
  }
  __device__ __forceinline__ unsigned* side_present() const {
    return reinterpret_cast<unsigned*>(side() + 6 * GBA_MAX_AGGS);
  }
};

template <bool K64>
__device__ __forceinline__ typename SmemTable<K64>::KeyW smem_empty_key() {
  return typename SmemTable<K64>::KeyW(K64 ? EMPTY64 : EMPTY32);
}

template <bool K64>
__device__ __forceinline__ int smem_find_or_insert(const SmemTable<K64>& t, uint64_t key, uint32_t h, int cap) {
  typedef typename SmemTable<K64>::KeyW KeyW;
  const KeyW kk = KeyW(key);
  const KeyW empty = smem_empty_key<K64>();
  int s = int((uint64_t(h) * unsigned(t.S)) >> 32);
  for (int p = 0; p < cap; ++p) {
    KeyW cur = *(volatile KeyW*)&t.keys[s];
    if (cur == kk) return s;
    if (cur == empty) {
      KeyW prev = atomicCAS(&t.keys[s], empty, kk);
      if (prev == empty || prev == kk) return s;
    }
    s = (s + 1 == t.S) ? 0 : s + 1;
  }
  return -1;
}

// Where an accumulator of a slot lives.  The table's accumulators are
// columns of SS 32-bit words, column c of slot i at C[c * SS + i] (C the
// accumulator area read as 32-bit words).  A COUNT takes one column.  An
// 8-byte accumulator starting at column w takes columns w and w + 1, split in
// two 32-bit halves: the low half at column w, the high half at column w + 1.
// The 32-bit atomics of lanes updating different slots then hit consecutive
// banks (as whole 8-byte words, slot i's low half sat in bank 2i mod 32, half
// the banks went unused and 78% of the partition kernel's atomic wavefronts
// conflicted; measured end to end the change is small: +2% on the skewed and
// serving queries, -2% on high cardinality).  MIN and MAX words, updated by
// 64-bit atomics, and the fp64 residual of an fp32 SUM stay whole: the two
// columns read as one array of SS 8-byte words, (8-byte words)[i].
// The side slot keeps one whole 8-byte word per column index, halves in place.
struct AccRef {
  unsigned* lo;             // low 32 bits (split words)
  unsigned* hi;             // high 32 bits (split words)
  unsigned long long* w64;  // the word itself (whole words)
};

template <bool K64>
__device__ __forceinline__ AccRef smem_ref(const SmemTable<K64>& t, int w, int i) {
  AccRef r;
  if (i < 0) {
    r.w64 = t.side() + w;
    r.lo = reinterpret_cast<unsigned*>(r.w64);
    r.hi = r.lo + 1;
  } else {
    unsigned* region = reinterpret_cast<unsigned*>(t.acc) + size_t(w) * t.SS;
    r.w64 = reinterpret_cast<unsigned long long*>(region) + i;
    r.lo = region + i;
    r.hi = region + t.SS + i;
  }
  return r;
}

// update one shared-memory accumulator (not ACC_ADD_F: see smem_fsum)
__device__ __forceinline__ void smem_acc(int op, const AccRef& r, unsigned long long v) {
  switch (op) {
    case ACC_CNT: atomicAdd(r.lo, unsigned(v)); break;
    case ACC_ADD_I: {
      const unsigned lo = unsigned(v), hi = unsigned(v >> 32);
      const unsigned old = atomicAdd(r.lo, lo);
      const unsigned add_hi = hi + ((old + lo) < old ? 1u : 0u);
      if (add_hi) atomicAdd(r.hi, add_hi);
      break;
    }
    case ACC_MIN_I:
      if ((long long)v < *(volatile long long*)r.w64) atomicMin(reinterpret_cast<long long*>(r.w64), (long long)v);
      break;
    case ACC_MAX_I:
      if ((long long)v > *(volatile long long*)r.w64) atomicMax(reinterpret_cast<long long*>(r.w64), (long long)v);
      break;
    default: break;
  }
}

// fp32 SUM in shared memory: an exact 128-bit two's-complement fixed-point
// accumulator with 64 fraction bits, held as four 32-bit limbs (the halves of
// its first two words), plus an fp64 residual in its third.  A contribution d (an fp32 value,
// or an fp64 sum of a few of them after warp coalescing) is added exactly when
// its binary expansion lies in [2^-64, 2^30): it is written as m * 2^shift with
// a 53-bit integer m and added limb by limb with 32-bit atomics, each carry
// forwarded by the add that produced it (so the limbs hold the exact sum mod
// 2^128; sums of fewer than 2^32 such values stay below 2^62 in magnitude).
// Anything else (NaN, infinities, |d| >= 2^30, bits below 2^-64) is added to
// the fp64 residual.  32-bit shared atomics keep their rate when many threads
// hit one hot key (measured 4.3 T/s on 8 slots, against 48 G/s for fp64
// atomicAdd, which contends like a compare-and-swap loop).
// The accumulator's three words: limbs 0-1 in split word r0, limbs 2-3 in
// split word r1, the residual in whole word r2.
__device__ __forceinline__ void smem_fsum(const AccRef& r0, const AccRef& r1, const AccRef& r2, double d) {
  const unsigned long long bits = __double_as_longlong(d);
  const int ex = int((bits >> 52) & 0x7ff);
  unsigned long long m = bits & ((1ull << 52) - 1);
  if (ex == 0 && m == 0) return;  // +-0
  bool exact = ex != 0 && ex != 0x7ff;
  int shift = ex - 1075 + 64;  // d = (m | 2^52) * 2^(ex-1075)
  if (exact) {
    m |= 1ull << 52;
    if (shift < 0) {
      const int r = -shift;
      if (r >= 53 || (m & ((1ull << r) - 1))) exact = false;
      else {
        m >>= r;
        shift = 0;
      }
    }
    if (shift > 41) exact = false;  // |d| >= 2^30
  }
  if (!exact) {
    atomicAdd(reinterpret_cast<double*>(r2.w64), d);
    return;
  }
  unsigned long long vlo = shift ? (m << shift) : m;
  unsigned long long vhi = shift ? (m >> (64 - shift)) : 0ull;
  if (bits >> 63) {  // negate (two's complement, 128 bits)
    vlo = ~vlo + 1ull;
    vhi = ~vhi + (vlo == 0ull ? 1ull : 0ull);
  }
  unsigned* const limb[4] = {r0.lo, r0.hi, r1.lo, r1.hi};
  const unsigned v[4] = {unsigned(vlo), unsigned(vlo >> 32), unsigned(vhi), unsigned(vhi >> 32)};
  unsigned carry = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const unsigned long long t = (unsigned long long)v[i] + carry;
    const unsigned add = unsigned(t);
    const unsigned k = unsigned(t >> 32);
    if (add == 0u) {
      carry = k;
    } else if (i < 3) {
      const unsigned old = atomicAdd(limb[i], add);
      carry = k + ((old + add) < old ? 1u : 0u);
    } else {
      atomicAdd(limb[3], add);  // carries out of bit 127 are discarded (mod 2^128)
    }
  }
}

// accumulator a of slot i (or of the side slot when i < 0) as its 8-byte
// result value; an fp32 SUM is one rounding of the exact fixed-point sum plus
// the residual, as fp64 bits
template <bool K64, typename Sig>
__device__ __forceinline__ unsigned long long smem_acc_read(const SmemTable<K64>& t, const QDesc& q, int a, int i) {
  const int w = Sig::woff(q, a);
  const int op = Sig::op(q, a);
  const AccRef r = smem_ref<K64>(t, w, i);
  if (op == ACC_MIN_I || op == ACC_MAX_I) return *r.w64;
  if (op == ACC_CNT) return *r.lo;
  const unsigned long long x = (unsigned long long)*r.hi << 32 | *r.lo;
  if (op != ACC_ADD_F) return x;
  const AccRef r1 = smem_ref<K64>(t, w + 2, i), r2 = smem_ref<K64>(t, w + 4, i);
  const long long hi = (long long)((unsigned long long)*r1.hi << 32 | *r1.lo);
  const double d = double(hi) + double(x) * 0x1p-64 + __longlong_as_double(*r2.w64);
  return __double_as_longlong(d);
}

// init all slots (called by the whole CTA; caller syncs): every accumulator
// word starts at its op's identity (fixed-point words and residual at 0)
// Merges every group of a shared table into an HBM table (all threads of the
// block; the caller syncs before and after).
template <bool K64, typename Sig>
__device__ __forceinline__ void smem_flush_to_gtable(const QDesc& q, const GTable& gt, const SmemTable<K64>& st,
                                                     unsigned* flags) {
  for (int i = threadIdx.x; i < st.S; i += blockDim.x) {
    const uint64_t k = st.keys[i];
    if (k == uint64_t(smem_empty_key<K64>())) continue;
    unsigned long long v[Sig::NA];
#pragma unroll
    for (int a = 0; a < Sig::NA; ++a) v[a] = smem_acc_read<K64, Sig>(st, q, a, i);
    gtable_insert<K64, Sig>(gt, q, k, table_hash(k), v, flags);
  }
  if (threadIdx.x == 0 && *st.side_present()) {
    unsigned long long v[Sig::NA];
#pragma unroll
    for (int a = 0; a < Sig::NA; ++a) v[a] = smem_acc_read<K64, Sig>(st, q, a, -1);
    gtable_insert<K64, Sig>(gt, q, K64 ? EMPTY64 : uint64_t(EMPTY32), 0u, v, flags);
  }
}

template <bool K64, typename Sig>
__device__ __forceinline__ void smem_table_init(const SmemTable<K64>& t, const QDesc& q) {
  for (int i = threadIdx.x; i < t.S; i += blockDim.x) {
    t.keys[i] = smem_empty_key<K64>();
#pragma unroll
    for (int a = 0; a < Sig::NA; ++a) {
      const int op = Sig::op(q, a), w = Sig::woff(q, a);
      const AccRef r = smem_ref<K64>(t, w, i);
      if (op == ACC_MIN_I || op == ACC_MAX_I) {
        *r.w64 = acc_identity(op);
      } else if (op == ACC_CNT) {
        *r.lo = 0u;
      } else {
        *r.lo = 0u;
        *r.hi = 0u;
        if (op == ACC_ADD_F) {
          const AccRef r1 = smem_ref<K64>(t, w + 2, i);
          *r1.lo = 0u;
          *r1.hi = 0u;
          *smem_ref<K64>(t, w + 4, i).w64 = 0ull;
        }
      }
    }
  }
  if (threadIdx.x == 0) {
    for (int w = 0; w < Sig::nwords(q); ++w) t.side()[w] = 0ull;
#pragma unroll
    for (int a = 0; a < Sig::NA; ++a)
      if (Sig::op(q, a) != ACC_ADD_F) t.side()[Sig::woff(q, a)] = acc_identity(Sig::op(q, a));
    *t.side_present() = 0u;
  }
}

// Warp-cooperative coalescing of equal keys (all 32 lanes call it).  Lanes
// holding the same key combine their contributions and only the group's
// lowest lane (returned true) applies the combined update:
//   - every live lane holds the same key (the hot-key case): xor-butterfly
//     reduction, 5 shuffle rounds per accumulator;
//   - largest group <= 4 lanes: each lane walks its (small) group;
//   - otherwise: no combining; each lane applies its own row (atomics to the
//     same address are serialised by the hardware, but the walk would cost
//     more than that).
template <bool K64, typename Sig>
__device__ __forceinline__ bool warp_coalesce(const QDesc& q, bool live, uint64_t key,
                                              unsigned long long (&v)[Sig::NA]) {
  constexpr int NA = Sig::NA;
  const unsigned lane = lane_id();
  const unsigned live_mask = __ballot_sync(GBA_FULL_MASK, live);
  unsigned peers;
  if constexpr (K64) peers = __match_any_sync(GBA_FULL_MASK, (unsigned long long)key);
  else peers = __match_any_sync(GBA_FULL_MASK, unsigned(key));
  peers &= live_mask;
  const unsigned gsize = live ? __popc(peers) : 0u;
  const unsigned maxg = __reduce_max_sync(GBA_FULL_MASK, gsize);
  if (maxg <= 1) return live;
  if (maxg == unsigned(__popc(live_mask))) {
    // one key across all live lanes: dead lanes contribute identities
    if (!live) {
#pragma unroll
      for (int a = 0; a < NA; ++a) v[a] = acc_identity(Sig::op(q, a));
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
#pragma unroll
      for (int a = 0; a < NA; ++a) v[a] = acc_combine(Sig::op(q, a), v[a], __shfl_xor_sync(GBA_FULL_MASK, v[a], o));
    }
    return live && lane == unsigned(__ffs(live_mask) - 1);
  }
  if (maxg > 4) return live;
  // small groups: each lane sums its own peer group from the peers' ORIGINAL values
  unsigned long long own[NA];
#pragma unroll
  for (int a = 0; a < NA; ++a) own[a] = v[a];
  unsigned rem = live ? (peers & ~(1u << lane)) : 0u;
#pragma unroll 1
  for (unsigned i = 1; i < maxg; ++i) {
    const int src = rem ? __ffs(rem) - 1 : int(lane);
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      unsigned long long x = __shfl_sync(GBA_FULL_MASK, own[a], src);
      if (rem) v[a] = acc_combine(Sig::op(q, a), v[a], x);
    }
    rem &= rem - 1u;
  }
  return live && ((peers & ((1u << lane) - 1u)) == 0u);
}

// apply a row (or coalesced partial) to shared slot `slot`
template <bool K64, typename Sig>
__device__ __forceinline__ void smem_apply(const SmemTable<K64>& t, const QDesc& q, int slot,
                                           const unsigned long long (&v)[Sig::NA]) {
#pragma unroll
  for (int a = 0; a < Sig::NA; ++a) {
    const int w = Sig::woff(q, a);
    if (Sig::op(q, a) == ACC_ADD_F)
      smem_fsum(smem_ref<K64>(t, w, slot), smem_ref<K64>(t, w + 2, slot), smem_ref<K64>(t, w + 4, slot),
                __longlong_as_double(v[a]));
    else smem_acc(Sig::op(q, a), smem_ref<K64>(t, w, slot), v[a]);
  }
}

template <bool K64, typename Sig>
__device__ __forceinline__ void smem_apply_side(const SmemTable<K64>& t, const QDesc& q,
                                                const unsigned long long (&v)[Sig::NA]) {
  if (*(volatile unsigned*)t.side_present() == 0u) atomicExch(t.side_present(), 1u);
#pragma unroll
  for (int a = 0; a < Sig::NA; ++a) {
    const int w = Sig::woff(q, a);
    if (Sig::op(q, a) == ACC_ADD_F)
      smem_fsum(smem_ref<K64>(t, w, -1), smem_ref<K64>(t, w + 2, -1), smem_ref<K64>(t, w + 4, -1),
                __longlong_as_double(v[a]));
    else smem_acc(Sig::op(q, a), smem_ref<K64>(t, w, -1), v[a]);
  }
}

// smem bytes of a table with S slots of `nwords` 4-byte accumulator words
// (side slot: one 8-byte word per column, at most 6 columns per accumulator)
__host__ __device__ inline size_t smem_table_bytes(int S, int key64, int nwords) {
  const size_t kb = key64 ? 8 : 4;
  return ((size_t(S) * kb + 15) & ~size_t(15)) + size_t((S + 1) & ~1) * nwords * 4 + 6 * GBA_MAX_AGGS * 8 + 16;
}

// carve a table at `base` (16-byte aligned)
template <bool K64>
__device__ __forceinline__ SmemTable<K64> smem_table_carve(unsigned char* base, int S, int nwords) {
  SmemTable<K64> t;
  t.S = S;
  t.SS = (S + 1) & ~1;
  size_t off = 0;
  t.keys = reinterpret_cast<typename SmemTable<K64>::KeyW*>(base + off);
  off += (size_t(S) * (K64 ? 8 : 4) + 15) & ~size_t(15);
  t.acc = reinterpret_cast<unsigned long long*>(base + off);
  t.nw = nwords;
  return t;
}

// contribution of a row's raw column bits to each accumulator
__device__ __forceinline__ unsigned long long pick_col(int c, const unsigned long long (&r)[GBA_MAX_COLS]) {
  return c == 0 ? r[0] : c == 1 ? r[1] : c == 2 ? r[2] : r[3];
}
template <typename Sig>
__device__ __forceinline__ void row_contrib(const QDesc& q, const unsigned long long (&raw)[GBA_MAX_COLS],
                                            unsigned long long (&v)[Sig::NA]) {
#pragma unroll
  for (int a = 0; a < Sig::NA; ++a)
    v[a] = acc_contrib(Sig::op(q, a), Sig::ctype(q, a), pick_col(Sig::col(q, a), raw));
}
