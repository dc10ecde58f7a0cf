// CPU oracle for the hash GROUP BY aggregation path.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker: only tests/, the smoke
// check in __graft_entry__.py and the CPU-baseline leg of bench.py may load it.
// The product library never links, loads or falls back to it.
//
// It restates, on the CPU, what the reference computes on the GPU
// (PneNPproof/cpu_gpu_coprocess_groupby_agg):
//
//  * orc_murmur3_32      MurmurHash3_x86_32, the hash the reference calls through
//                        cuco::detail::MurmurHash3_32 (tiled_groupby_agg_partition/
//                        src/kernel.cu:22,127,196,261,309).  Written from the published
//                        public-domain algorithm; pinned by known answers.
//  * orc_groupby         exact GROUP BY: one output row per distinct key with the
//                        aggregate of every input row carrying that key.  This is the
//                        result of phase 1 + phase 2 together: kernel.cu:9-186 (per tile)
//                        and kernel.cu:294-406 (per partition) both compute an exact
//                        per-key SUM; the reference accumulates u32 (wrapping), this
//                        oracle accumulates int64 (and fp64 for fp32 and fp64 columns) so nothing
//                        overflows, which is the contract of the new implementation.
//  * orc_tile_partition_counts
//                        the reference's phase-1 partition layout: each tile of
//                        tile_len rows (group_then_partition.cu:342-348) is reduced to its
//                        distinct keys, which are placed in partition murmur(key, 0) % P
//                        (kernel.cu:196,225,261,285).
//  * orc_merge_partitions
//                        the greedy min-heap merge of small partitions
//                        (groupby_agg_intra_partition.cu:13-48) and the resulting
//                        par_kv_begin prefix (groupby_agg_intra_partition.cu:303-311).
//  * orc_gen             the benchmark's seeded input columns, from the same
//                        generator header the library's own generator uses
//                        (datagen.h), so the CPU arm of the benchmark produces
//                        the GPU arm's inputs without loading the library.
//
// Parity with the reference itself is pinned by tests/golden/ fixtures produced by
// running the unmodified reference (built by oracle/Makefile into oracle/_ref).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <queue>
#include <thread>
#include <vector>

#include "datagen.h"

extern "C" {

enum { ORC_I32 = 0, ORC_I64 = 1, ORC_F32 = 2, ORC_U32 = 3, ORC_F64 = 4 };
enum { ORC_SUM = 0, ORC_COUNT = 1, ORC_MIN = 2, ORC_MAX = 3, ORC_SUMABS = 4 };

// ---------------------------------------------------------------------------
// MurmurHash3_x86_32 (Appleby, public domain), restated from its description.
static inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

uint32_t orc_murmur3_32(const void* data, uint64_t len, uint32_t seed) {
  const uint8_t* p = static_cast<const uint8_t*>(data);
  const uint32_t c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
  uint32_t h = seed;
  const uint64_t nblocks = len / 4;
  for (uint64_t i = 0; i < nblocks; ++i) {
    uint32_t k;
    std::memcpy(&k, p + 4 * i, 4);
    k *= c1;
    k = rotl32(k, 15);
    k *= c2;
    h ^= k;
    h = rotl32(h, 13);
    h = h * 5u + 0xe6546b64u;
  }
  const uint8_t* tail = p + 4 * nblocks;
  uint32_t k = 0;
  switch (len & 3) {
    case 3: k ^= uint32_t(tail[2]) << 16; [[fallthrough]];
    case 2: k ^= uint32_t(tail[1]) << 8; [[fallthrough]];
    case 1:
      k ^= tail[0];
      k *= c1;
      k = rotl32(k, 15);
      k *= c2;
      h ^= k;
  }
  h ^= uint32_t(len);
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

}  // extern "C"

namespace {

inline int key_bytes(int t) { return t == ORC_I64 ? 8 : 4; }

// Keys are carried as int64 internally: I32 sign-extended, U32 zero-extended.
inline int64_t load_key(int t, const void* keys, int64_t i) {
  switch (t) {
    case ORC_I32: return static_cast<const int32_t*>(keys)[i];
    case ORC_U32: return static_cast<const uint32_t*>(keys)[i];
    default: return static_cast<const int64_t*>(keys)[i];
  }
}
inline void store_key(int t, void* keys, int64_t i, int64_t k) {
  switch (t) {
    case ORC_I32: static_cast<int32_t*>(keys)[i] = int32_t(k); break;
    case ORC_U32: static_cast<uint32_t*>(keys)[i] = uint32_t(k); break;
    default: static_cast<int64_t*>(keys)[i] = k;
  }
}
inline uint32_t key_hash(int t, int64_t k, uint32_t seed) {
  if (t == ORC_I64) return orc_murmur3_32(&k, 8, seed);
  uint32_t k32 = uint32_t(k);
  return orc_murmur3_32(&k32, 4, seed);
}

struct AggSpec {
  int naggs;
  const int* ops;
  const int* cols;
  const int* col_types;
  const void* const* cols_data;
};

inline bool agg_is_fp(const AggSpec& s, int a) {
  const int op = s.ops[a];
  if (op == ORC_COUNT) return false;
  const int t = s.col_types[s.cols[a]];
  return (t == ORC_F32 || t == ORC_F64) && (op == ORC_SUM || op == ORC_SUMABS);
}

union Acc {
  int64_t i;
  double f;
};

inline Acc agg_init(const AggSpec& s, int a) {
  Acc v;
  switch (s.ops[a]) {
    case ORC_MIN:
      if (agg_is_fp(s, a)) v.f = INFINITY; else v.i = INT64_MAX;
      break;
    case ORC_MAX:
      if (agg_is_fp(s, a)) v.f = -INFINITY; else v.i = INT64_MIN;
      break;
    default:
      if (agg_is_fp(s, a)) v.f = 0.0; else v.i = 0;
  }
  return v;
}

inline void agg_update(const AggSpec& s, int a, Acc& acc, int64_t row) {
  const int op = s.ops[a];
  if (op == ORC_COUNT) { acc.i += 1; return; }
  const int c = s.cols[a];
  const void* col = s.cols_data[c];
  switch (s.col_types[c]) {
    case ORC_F32:
    case ORC_F64: {
      const double x = s.col_types[c] == ORC_F64 ? static_cast<const double*>(col)[row]
                                                 : double(static_cast<const float*>(col)[row]);
      if (op == ORC_SUM) acc.f += x;
      else if (op == ORC_SUMABS) acc.f += std::fabs(x);
      else if (op == ORC_MIN) { /* fp MIN/MAX are not part of the contract */ }
      return;
    }
    default: {
      int64_t x;
      switch (s.col_types[c]) {
        case ORC_I32: x = static_cast<const int32_t*>(col)[row]; break;
        case ORC_U32: x = static_cast<const uint32_t*>(col)[row]; break;
        default: x = static_cast<const int64_t*>(col)[row];
      }
      if (op == ORC_SUM) acc.i = int64_t(uint64_t(acc.i) + uint64_t(x));  // wraps mod 2^64 like the GPU
      else if (op == ORC_MIN) acc.i = std::min(acc.i, x);
      else if (op == ORC_MAX) acc.i = std::max(acc.i, x);
      else if (op == ORC_SUMABS) acc.i = int64_t(uint64_t(acc.i) + uint64_t(x < 0 ? -x : x));
    }
  }
}

// Open-addressing table of (key -> index into a dense group array).  Keys are
// compared in full, so the result never depends on the hash.
struct GroupTable {
  std::vector<int64_t> slot_key;
  std::vector<int64_t> slot_grp;  // -1 = empty
  uint64_t mask = 0;
  void reset(uint64_t expect) {
    uint64_t cap = 16;
    while (cap < expect * 2) cap <<= 1;
    slot_key.assign(cap, 0);
    slot_grp.assign(cap, -1);
    mask = cap - 1;
  }
  // returns group index, creating it (as ngroups) when absent
  int64_t find_or_insert(int64_t k, uint32_t h, int64_t ngroups, bool* created) {
    uint64_t s = h & mask;
    while (true) {
      if (slot_grp[s] < 0) {
        slot_key[s] = k;
        slot_grp[s] = ngroups;
        *created = true;
        return ngroups;
      }
      if (slot_key[s] == k) { *created = false; return slot_grp[s]; }
      s = (s + 1) & mask;
    }
  }
};

// Aggregate rows idx[0..m) (or rows [lo,hi) when idx == nullptr) into dense
// group arrays: out_key[g], acc[g*naggs + a].  Returns the group count.
int64_t aggregate_rows(int key_type, const void* keys, const AggSpec& s, const uint32_t* idx, int64_t lo,
                       int64_t hi, std::vector<int64_t>& out_key, std::vector<Acc>& acc) {
  const int64_t m = hi - lo;
  GroupTable t;
  t.reset(uint64_t(std::max<int64_t>(m, 1)));
  out_key.clear();
  acc.clear();
  int64_t ng = 0;
  for (int64_t j = lo; j < hi; ++j) {
    const int64_t row = idx ? int64_t(idx[j]) : j;
    const int64_t k = load_key(key_type, keys, row);
    bool created;
    const int64_t g = t.find_or_insert(k, key_hash(key_type, k, 0x9747b28cu), ng, &created);
    if (created) {
      ++ng;
      out_key.push_back(k);
      for (int a = 0; a < s.naggs; ++a) acc.push_back(agg_init(s, a));
    }
    for (int a = 0; a < s.naggs; ++a) agg_update(s, a, acc[size_t(g) * s.naggs + a], row);
  }
  return ng;
}

}  // namespace

extern "C" {

// Exact GROUP BY over n rows.  keys: n keys of key_type.  cols: ncols value
// columns of col_types.  Aggregate a is ops[a] over column agg_cols[a]
// (ignored for COUNT).  Output (capacity n rows): out_keys in key_type,
// out_accs[a] an array of int64 (integer aggregates, COUNT) or double (SUM /
// SUMABS over fp32 or fp64).  Rows are written sorted by key when sort_output != 0.
// nthreads <= 1 runs single-threaded; more threads run a partitioned
// aggregation (radix partition on hash bits, then one table per partition).
// Returns the number of groups.
int64_t orc_groupby(int key_type, const void* keys, int64_t n, int ncols, const int* col_types,
                    const void* const* cols, int naggs, const int* agg_ops, const int* agg_cols,
                    void* out_keys, void* const* out_accs, int nthreads, int sort_output) {
  (void)ncols;
  AggSpec s{naggs, agg_ops, agg_cols, col_types, cols};
  std::vector<int64_t> gk;
  std::vector<Acc> ga;
  int64_t ng = 0;

  if (nthreads <= 1 || n < (1 << 16)) {
    ng = aggregate_rows(key_type, keys, s, nullptr, 0, n, gk, ga);
  } else {
    const int T = nthreads;
    const int PB = 10;
    const int P = 1 << PB;
    std::vector<uint32_t> hist(size_t(T) * P, 0);
    std::vector<uint32_t> idx(static_cast<size_t>(n));
    auto pid_of = [&](int64_t row) {
      return key_hash(key_type, load_key(key_type, keys, row), 0x2545f491u) >> (32 - PB);
    };
    auto chunk = [&](int t, int64_t* lo, int64_t* hi) {
      *lo = n * t / T;
      *hi = n * (t + 1) / T;
    };
    {
      std::vector<std::thread> th;
      for (int t = 0; t < T; ++t)
        th.emplace_back([&, t] {
          int64_t lo, hi;
          chunk(t, &lo, &hi);
          uint32_t* h = &hist[size_t(t) * P];
          for (int64_t r = lo; r < hi; ++r) h[pid_of(r)]++;
        });
      for (auto& x : th) x.join();
    }
    std::vector<uint64_t> off(size_t(T) * P), pbeg(P + 1);
    uint64_t run = 0;
    for (int p = 0; p < P; ++p) {
      pbeg[p] = run;
      for (int t = 0; t < T; ++t) {
        off[size_t(t) * P + p] = run;
        run += hist[size_t(t) * P + p];
      }
    }
    pbeg[P] = run;
    {
      std::vector<std::thread> th;
      for (int t = 0; t < T; ++t)
        th.emplace_back([&, t] {
          int64_t lo, hi;
          chunk(t, &lo, &hi);
          uint64_t* o = &off[size_t(t) * P];
          for (int64_t r = lo; r < hi; ++r) idx[o[pid_of(r)]++] = uint32_t(r);
        });
      for (auto& x : th) x.join();
    }
    std::vector<std::vector<int64_t>> pk(P);
    std::vector<std::vector<Acc>> pa(P);
    std::atomic<int> next{0};
    {
      std::vector<std::thread> th;
      for (int t = 0; t < T; ++t)
        th.emplace_back([&] {
          for (int p = next++; p < P; p = next++)
            aggregate_rows(key_type, keys, s, idx.data(), int64_t(pbeg[p]), int64_t(pbeg[p + 1]), pk[p], pa[p]);
        });
      for (auto& x : th) x.join();
    }
    for (int p = 0; p < P; ++p) {
      gk.insert(gk.end(), pk[p].begin(), pk[p].end());
      ga.insert(ga.end(), pa[p].begin(), pa[p].end());
    }
    ng = int64_t(gk.size());
  }

  std::vector<int64_t> order(static_cast<size_t>(ng));
  for (int64_t g = 0; g < ng; ++g) order[g] = g;
  if (sort_output) {
    if (key_type == ORC_U32)
      std::sort(order.begin(), order.end(),
                [&](int64_t a, int64_t b) { return uint64_t(gk[a]) < uint64_t(gk[b]); });
    else
      std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return gk[a] < gk[b]; });
  }
  for (int64_t j = 0; j < ng; ++j) {
    const int64_t g = order[j];
    store_key(key_type, out_keys, j, gk[g]);
    for (int a = 0; a < naggs; ++a) {
      const Acc v = ga[size_t(g) * naggs + a];
      if (agg_is_fp(s, a)) static_cast<double*>(out_accs[a])[j] = v.f;
      else static_cast<int64_t*>(out_accs[a])[j] = v.i;
    }
  }
  return ng;
}

// Reference phase-1 layout for u32 keys: for every tile of tile_len rows, the
// number of distinct keys of the tile that land in partition murmur(key,0) % P.
// out_counts has ntiles * P entries (tile-major).
void orc_tile_partition_counts(const uint32_t* keys, int64_t n, int64_t tile_len, int64_t P,
                               uint32_t* out_counts) {
  const int64_t ntiles = (n + tile_len - 1) / tile_len;
  std::memset(out_counts, 0, sizeof(uint32_t) * size_t(ntiles * P));
  for (int64_t t = 0; t < ntiles; ++t) {
    const int64_t lo = t * tile_len, hi = std::min(n, lo + tile_len);
    std::vector<uint32_t> ks(keys + lo, keys + hi);
    std::sort(ks.begin(), ks.end());
    ks.erase(std::unique(ks.begin(), ks.end()), ks.end());
    for (uint32_t k : ks) out_counts[t * P + orc_murmur3_32(&k, 4, 0) % uint32_t(P)]++;
  }
}

// Partition of u32 keys as the reference's partitioner places them (seed 0).
uint32_t orc_partition_of_u32(uint32_t key, uint32_t P) { return orc_murmur3_32(&key, 4, 0) % P; }
void orc_partition_u32_array(const uint32_t* keys, int64_t n, uint32_t P, uint32_t* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = orc_murmur3_32(&keys[i], 4, 0) % P;
}

// Greedy merge of partitions (min-heap by size, merge while the sum stays <= K),
// restating groupby_agg_intra_partition.cu:13-48 with the same container
// (std::priority_queue, same comparator, same push/pop sequence) so equal-size
// ties resolve identically.  sizes[P] are partition row counts.  Output:
// merged_of[p] = index of the merged partition that original partition p joined;
// merged_sizes[i]; returns the merged partition count.  Segment order inside a
// merged partition does not affect any observable result.
int64_t orc_merge_partitions(const uint32_t* sizes, int64_t P, uint64_t K, int64_t* merged_of,
                             uint64_t* merged_sizes) {
  struct Part {
    uint64_t size;
    std::vector<int64_t> members;
  };
  auto cmp = [](const Part& l, const Part& r) { return l.size > r.size; };
  std::vector<Part> init;
  for (int64_t p = 0; p < P; ++p) init.push_back(Part{sizes[p], {p}});
  std::priority_queue<Part, std::vector<Part>, decltype(cmp)> H(init.begin(), init.end(), cmp);
  while (true) {
    if (H.size() == 1) break;
    Part tmp = H.top();
    H.pop();
    Part top = H.top();
    if (tmp.size + top.size > K) {
      H.push(tmp);
      break;
    }
    do {
      tmp.size += top.size;
      tmp.members.insert(tmp.members.end(), top.members.begin(), top.members.end());
      H.pop();
      if (H.size() == 0) break;
      top = H.top();
    } while (top.size + tmp.size <= K);
    H.push(tmp);
  }
  int64_t m = 0;
  while (!H.empty()) {
    const Part& q = H.top();
    for (int64_t p : q.members) merged_of[p] = m;
    merged_sizes[m] = q.size;
    ++m;
    H.pop();
  }
  return m;
}

// ---------------------------------------------------------------------------
// Input generator: rows [row0, row0 + n) of a seeded spec, on nthreads threads
// (every row is an independent PCG32 stream, so any split gives the same
// columns).  keys: 4- or 8-byte column; cols[c]: int32, int64 or fp32 as the
// spec's column kind says.  Returns 0, or -1 for a bad spec.
int orc_gen(const gba_gen_spec* sp, int64_t row0, int64_t n, void* keys, void* const* cols, int nthreads) {
  if (!sp || (sp->key_bits != 32 && sp->key_bits != 64) || sp->ndv < 1 || sp->ncols < 0 ||
      sp->ncols > GBA_GEN_MAX_COLS || sp->zipf_s < 0 || n < 0)
    return -1;
  const gba_zipf z = gba_zipf_make(sp->ndv, sp->zipf_s > 0 ? sp->zipf_s : 1.0);
  auto work = [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; ++i) {
      uint64_t key;
      int64_t iv[GBA_GEN_MAX_COLS];
      float fv[GBA_GEN_MAX_COLS];
      gba_gen_row(sp, &z, uint64_t(row0 + i), &key, iv, fv);
      if (sp->key_bits == 64) static_cast<uint64_t*>(keys)[i] = key;
      else static_cast<uint32_t*>(keys)[i] = uint32_t(key);
      for (int c = 0; c < sp->ncols; ++c) {
        if (sp->col_kind[c] == GBA_GEN_UNIFORM_I64) static_cast<int64_t*>(cols[c])[i] = iv[c];
        else if (sp->col_kind[c] == GBA_GEN_NORMAL_F32) static_cast<float*>(cols[c])[i] = fv[c];
        else static_cast<int32_t*>(cols[c])[i] = int32_t(iv[c]);
      }
    }
  };
  const int T = std::max(1, std::min(nthreads, 256));
  if (T == 1 || n < 65536) {
    work(0, n);
  } else {
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) th.emplace_back(work, n * t / T, n * (t + 1) / T);
    for (auto& x : th) x.join();
  }
  return 0;
}

}  // extern "C"
