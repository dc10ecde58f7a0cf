// Device-side building blocks shared by the group-by kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "gba_kernels.h"

#define GBA_FULL_MASK 0xffffffffu

static constexpr unsigned long long EMPTY64 = ~0ull;
static constexpr unsigned EMPTY32 = ~0u;

// ---------------------------------------------------------------------------
// MurmurHash3_x86_32 of a 4-byte or 8-byte little-endian key (the hash the
// reference uses through cuco::detail::MurmurHash3_32, kernel.cu:22).
__device__ __forceinline__ uint32_t mm3_round(uint32_t h, uint32_t k) {
  k *= 0xcc9e2d51u;
  k = __funnelshift_l(k, k, 15);
  k *= 0x1b873593u;
  h ^= k;
  h = __funnelshift_l(h, h, 13);
  return h * 5u + 0xe6546b64u;
}
__device__ __forceinline__ uint32_t mm3_fmix(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}
__device__ __forceinline__ uint32_t murmur3_32(uint32_t key, uint32_t seed) {
  return mm3_fmix(mm3_round(seed, key) ^ 4u);
}
__device__ __forceinline__ uint32_t murmur3_64(uint64_t key, uint32_t seed) {
  uint32_t h = mm3_round(seed, uint32_t(key));
  h = mm3_round(h, uint32_t(key >> 32));
  return mm3_fmix(h ^ 8u);
}
template <bool K64>
__device__ __forceinline__ uint32_t key_hash(uint64_t k, uint32_t seed) {
  if constexpr (K64) return murmur3_64(k, seed);
  else return murmur3_32(uint32_t(k), seed);
}

// Engine hashes.  MurmurHash3 (above) is kept for the reference-compatible
// partition layout of the drop-in API; the engine's own tables and radix
// digits only need a well-mixed 32-bit value, and the kernels are
// instruction-bound (measured: ~100 G rows/s for a COUNT in shared memory with
// murmur), so they use one 64-bit multiply after a xor-fold (5 instructions).
// Two different odd multipliers keep the partition digit (top bits of one
// hash) independent of the slot inside the partition's table (top bits of the
// other).
static constexpr uint32_t GBA_TABLE_SEED = 0x9747b28cu;
static constexpr uint32_t GBA_PART_SEED = 0x2545f491u;
__device__ __forceinline__ uint32_t fast_hash(uint64_t k, uint64_t mul) {
  k ^= k >> 29;
  return uint32_t((k * mul) >> 32);
}
__device__ __forceinline__ uint32_t table_hash(uint64_t k) { return fast_hash(k, 0x9e3779b97f4a7c15ull); }
__device__ __forceinline__ uint32_t part_hash(uint64_t k) { return fast_hash(k, 0xd6e8feb86659fd93ull); }

// ---------------------------------------------------------------------------
// Row access.
__device__ __forceinline__ uint64_t load_key_g(const QDesc& q, int64_t r) {
  if (q.key64) return __ldg(static_cast<const unsigned long long*>(q.keys) + r);
  return __ldg(static_cast<const unsigned*>(q.keys) + r);
}

// Contribution of row value `raw` (8 raw bytes as loaded) to accumulator a.
// raw holds the column value bits: i32/u32 in the low word, f32 bits in the low
// word, i64 and f64 in full.
__device__ __forceinline__ unsigned long long acc_contrib(int op, int ctype, unsigned long long raw) {
  switch (op) {
    case ACC_CNT: return 1ull;
    case ACC_ADD_F: {
      if (ctype == GBA_F64) return raw;
      return __double_as_longlong(double(__uint_as_float(unsigned(raw))));
    }
    default: {
      long long v;
      if (ctype == GBA_I32) v = (long long)(int)(unsigned)raw;
      else if (ctype == GBA_U32) v = (long long)(unsigned)raw;
      else v = (long long)raw;
      return (unsigned long long)v;
    }
  }
}

__device__ __forceinline__ unsigned long long acc_identity(int op) {
  switch (op) {
    case ACC_MIN_I: return 0x7fffffffffffffffull;
    case ACC_MAX_I: return 0x8000000000000000ull;
    default: return 0ull;  // integer 0 and +0.0 share the bit pattern
  }
}

// combine two partial accumulators (register arithmetic)
__device__ __forceinline__ unsigned long long acc_combine(int op, unsigned long long a, unsigned long long b) {
  switch (op) {
    case ACC_MIN_I: return (long long)a < (long long)b ? a : b;
    case ACC_MAX_I: return (long long)a > (long long)b ? a : b;
    case ACC_ADD_F: return __double_as_longlong(__longlong_as_double(a) + __longlong_as_double(b));
    default: return a + b;
  }
}

// atomic combine into shared or global memory (generic address)
__device__ __forceinline__ void acc_atomic(int op, unsigned long long* p, unsigned long long v) {
  switch (op) {
    case ACC_MIN_I: atomicMin(reinterpret_cast<long long*>(p), (long long)v); break;
    case ACC_MAX_I: atomicMax(reinterpret_cast<long long*>(p), (long long)v); break;
    case ACC_ADD_F: atomicAdd(reinterpret_cast<double*>(p), __longlong_as_double(v)); break;
    default: atomicAdd(p, v);
  }
}

// Fire-and-forget reductions into global memory.  The address space is
// stated explicitly: a table pointer read from shared memory (a batch kernel's
// query descriptor) is a generic pointer to the compiler, and a generic
// atomicAdd whose result is unused still compiles to a returning atomic, which
// the warp then waits for.
__device__ __forceinline__ void red_add_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}
__device__ __forceinline__ void red_min_s64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.min.s64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}
__device__ __forceinline__ void red_max_s64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.max.s64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}
__device__ __forceinline__ void red_add_f64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "d"(__longlong_as_double(v))
               : "memory");
}
__device__ __forceinline__ unsigned long long cas_global_u64(unsigned long long* p, unsigned long long cmp,
                                                             unsigned long long val) {
  unsigned long long old;
  asm volatile("atom.relaxed.gpu.global.cas.b64 %0, [%1], %2, %3;"
               : "=l"(old)
               : "l"(__cvta_generic_to_global(p)), "l"(cmp), "l"(val)
               : "memory");
  return old;
}

// HBM/L2 accumulator update: 64-bit reductions (L2 runs 64- and 32-bit
// atomics at the same rate); MIN/MAX read first and skip rows that cannot
// improve.
__device__ __forceinline__ void global_acc(int op, unsigned long long* p, unsigned long long v) {
  switch (op) {
    case ACC_MIN_I:
      if ((long long)v < (long long)__ldcg(p)) red_min_s64(p, v);
      break;
    case ACC_MAX_I:
      if ((long long)v > (long long)__ldcg(p)) red_max_s64(p, v);
      break;
    case ACC_ADD_F: red_add_f64(p, v); break;
    default: red_add_u64(p, v);
  }
}

// ---------------------------------------------------------------------------
// Global table insert of one (key, partial accumulators) pair.  Linear probing
// from the hashed slot, capped at t.probe_cap probes; on failure the overflow
// flag is raised and the pair is dropped (the host re-runs the query with a
// larger table, so a result is never reported from an overflowed table).
// NA is the number of accumulators of the query (the table's slot stride is
// gba_gt_stride(NA) words); kernels are instantiated per NA so no dead
// accumulator code is emitted.
template <bool K64, typename Sig>
__device__ __forceinline__ void gtable_insert(const GTable& t, const QDesc& q, uint64_t key, uint32_t h,
                                              const unsigned long long* vals, unsigned* flags) {
  constexpr int NA = Sig::NA;
  constexpr int stride = gba_gt_stride(NA);
  unsigned long long* slotp;
  if (key == (K64 ? EMPTY64 : uint64_t(EMPTY32))) {
    slotp = t.base + t.cap * stride;
    if (slotp[0] == 0ull) atomicExch(slotp, 1ull);
  } else {
    uint64_t s = (uint64_t(h) * t.cap) >> 32;  // cap <= 2^32
    int p = 0;
    for (;;) {
      slotp = t.base + s * stride;
      unsigned long long cur = __ldcg(slotp);  // L2 (coherent point), no L1
      if (cur == key) break;
      if (cur == EMPTY64) {
        unsigned long long prev = cas_global_u64(slotp, EMPTY64, key);
        if (prev == EMPTY64 || prev == key) break;
      }
      if (++p >= t.probe_cap) {
        atomicOr(flags, GBA_FLAG_TABLE_OVERFLOW);
        return;
      }
      s = (s + 1 == t.cap) ? 0 : s + 1;
    }
  }
#pragma unroll
  for (int a = 0; a < NA; ++a) global_acc(Sig::op(q, a), slotp + 1 + a, vals[a]);
}

// The same insert split in two so a thread can have several first probes in
// flight: gtable_first_slot() gives the home slot; the caller loads its key
// word with __ldcg for each pending insert, then finishes each one.
__device__ __forceinline__ uint64_t gtable_home(const GTable& t, uint32_t h) { return (uint64_t(h) * t.cap) >> 32; }

template <bool K64, typename Sig>
__device__ __forceinline__ void gtable_finish(const GTable& t, const QDesc& q, uint64_t key, uint64_t s,
                                              unsigned long long cur, const unsigned long long* vals,
                                              unsigned* flags) {
  constexpr int NA = Sig::NA;
  constexpr int stride = gba_gt_stride(NA);
  unsigned long long* slotp = t.base + s * stride;
  int p = 0;
  for (;;) {
    if (cur == key) break;
    if (cur == EMPTY64) {
      unsigned long long prev = cas_global_u64(slotp, EMPTY64, key);
      if (prev == EMPTY64 || prev == key) break;
    }
    if (++p >= t.probe_cap) {
      atomicOr(flags, GBA_FLAG_TABLE_OVERFLOW);
      return;
    }
    s = (s + 1 == t.cap) ? 0 : s + 1;
    slotp = t.base + s * stride;
    cur = __ldcg(slotp);
  }
#pragma unroll
  for (int a = 0; a < NA; ++a) global_acc(Sig::op(q, a), slotp + 1 + a, vals[a]);
}

// Compile-time dispatch over (key width, accumulator count): f(K64, NA) is
// called with std::integral_constant arguments.
#include <type_traits>
template <typename F>
inline cudaError_t gba_dispatch(bool key64, int na, F&& f) {
  using T = std::true_type;
  using Fl = std::false_type;
#define GBA_NA_CASE(N)                                                                   \
  case N:                                                                                \
    return key64 ? f(T{}, std::integral_constant<int, N>{}) : f(Fl{}, std::integral_constant<int, N>{});
  switch (na) {
    GBA_NA_CASE(1)
    GBA_NA_CASE(2)
    GBA_NA_CASE(3)
    GBA_NA_CASE(4)
    GBA_NA_CASE(5)
    GBA_NA_CASE(6)
    GBA_NA_CASE(7)
    GBA_NA_CASE(8)
  }
#undef GBA_NA_CASE
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// TMA bulk copy + mbarrier helpers (no multicast anywhere in this library).
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: returns false (and raises the timeout flag) after max_iter
// unsuccessful polls.  try_wait itself suspends for a hardware-chosen interval,
// so max_iter = 1<<22 bounds the wait to well under a few seconds.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, unsigned* flags) {
  for (unsigned it = 0; it < (1u << 22); ++it)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(flags, GBA_FLAG_WAIT_TIMEOUT);
  return false;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
// Dynamic shared-memory limit for a kernel: always the most the device allows
// beside the kernel's static shared memory.  The attribute is process-wide per
// kernel, so setting it to each launch's own size would race between host
// threads launching the same kernel with different sizes (one thread's
// smaller limit failing the other's launch); this value is the same for every
// caller and does not change a launch's occupancy, which follows the shared
// memory the launch asks for.
template <typename K>
inline cudaError_t gba_allow_max_smem(K* kernel) {
  static const int optin = [] {
    int d = 0, v = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, d);
    return v;
  }();
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, kernel);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - int(a.sharedSizeBytes));
}


// ---------------------------------------------------------------------------
// Thread-block-cluster distributed shared memory (sm_90+): addresses in the
// shared::cluster window, mapped from this CTA's shared address to the same
// offset in CTA `rank` of the cluster.
__device__ __forceinline__ unsigned cluster_ctarank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t dsmem_map(uint32_t local_addr, unsigned rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local_addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void dsmem_ld_v4(uint32_t addr, unsigned& x0, unsigned& x1, unsigned& x2, unsigned& x3) {
  asm volatile("ld.volatile.shared::cluster.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(x0), "=r"(x1), "=r"(x2), "=r"(x3)
               : "r"(addr));
}
__device__ __forceinline__ unsigned dsmem_atom_add_u32(uint32_t addr, unsigned v) {
  unsigned old;
  asm volatile("atom.shared::cluster.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(addr), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ void dsmem_red_add_u32(uint32_t addr, unsigned v) {
  asm volatile("red.shared::cluster.add.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned dsmem_cas_b32(uint32_t addr, unsigned cmp, unsigned val) {
  unsigned old;
  asm volatile("atom.shared::cluster.cas.b32 %0, [%1], %2, %3;" : "=r"(old) : "r"(addr), "r"(cmp), "r"(val) : "memory");
  return old;
}
__device__ __forceinline__ unsigned long long dsmem_cas_b64(uint32_t addr, unsigned long long cmp,
                                                            unsigned long long val) {
  unsigned long long old;
  asm volatile("atom.shared::cluster.cas.b64 %0, [%1], %2, %3;" : "=l"(old) : "r"(addr), "l"(cmp), "l"(val) : "memory");
  return old;
}
__device__ __forceinline__ void dsmem_st_u32(uint32_t addr, unsigned v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
// All threads of every CTA of the cluster: release this CTA's shared-memory
// writes, wait for every other CTA's (a hardware barrier; it completes once
// all threads of the cluster have arrived).
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
