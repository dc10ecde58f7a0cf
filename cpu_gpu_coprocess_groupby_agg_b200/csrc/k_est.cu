// Learned cardinality estimator: sampling/feature kernels and a 3x64 MLP with
// hand-written forward, backward and Adam kernels (fp32).
//
// No counterpart in the reference: it sizes every table from the tile length
// (Capacity = tile_len, test/test.cu:104) and never estimates group counts.
//
// Features of one query (32 floats), from a sample of up to 1024 rows (128
// evenly spaced runs of 8 rows) in each of up to 256 evenly spaced tiles of
// `tile_rows` rows:
//   0 log2(n+1)/32          1 log2(s+1)/32 (s = sampled rows)
//   2 d/s (d = distinct sampled keys)   3..6 f1/s, f2/s, f3/s, f4+/s
//   7 log2(d+1)/32          8 log2(GEE+1)/32, GEE = sqrt(n/s) f1 + (d - f1)
//   9 log2(Chao1+1)/32, Chao1 = d + f1^2 / (2 max(f2, 1))
//  10 log2(HLL+1)/32 (64-register HyperLogLog of the sample)
//  11 max key frequency / s  12 key bits / 64   13 s/n
//  14..29 histogram of the 64 HLL register values 0..15 (fraction)
//  30 log2(n/s)/32          31 1
// The network predicts t = log2(groups)/32; the caller clamps 2^(32 t) to
// [d, n].
#include <math.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "est_kernels.h"
#include "gba_context.h"
#include "gba_internal.cuh"
#include "gba_plan.h"

namespace {

constexpr int F = GBA_EST_FEATURES;  // 32
constexpr int H = GBA_EST_HIDDEN;    // 64
// parameter layout
constexpr int OW1 = 0, OB1 = OW1 + H * F, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + H * H,
              OW4 = OB3 + H, OB4 = OW4 + H, NPARAM = OB4 + 1;

__device__ __forceinline__ uint64_t sample_row(const EstQuery& e, int64_t item) {
  // item = sampled tile * 1024 + j: the tile's 1024 sampled rows are 128 runs
  // of 8 consecutive rows at evenly spaced positions (run j / 8 starts at
  // (j / 8) * len / 128).  A run of 8 keys fills whole 32-byte sectors (one
  // row per position had spent a sector on every 4- or 8-byte key), and 128
  // positions still spread the sample over the tile: a column that repeats
  // with a period shows its every value (runs of 32 at 32 positions did not)
  const int64_t st = item >> 10, j = item & 1023;
  const int64_t tile = st * e.tile_step;
  const int64_t tb = tile * e.tile_rows;
  const int64_t te = tb + e.tile_rows < e.n ? tb + e.tile_rows : e.n;
  const int64_t len = te - tb;
  if (len <= 0) return ~0ull;
  if (len <= 1024) return j < len ? uint64_t(tb + j) : ~0ull;
  return uint64_t(tb + (j >> 3) * (len / 128) + (j & 7));
}

// every query's count table to {empty key, 0} (blockIdx.y = query)
__global__ void k_est_init(const EstQuery* qs, int nq) {
  for (int qi = blockIdx.y; qi < nq; qi += gridDim.y) {
    const EstQuery e = qs[qi];
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < e.cap;
         i += uint64_t(gridDim.x) * blockDim.x) {
      e.table[2 * i] = EMPTY64;
      e.table[2 * i + 1] = 0ull;
    }
  }
}

// Frequency-class bookkeeping: a key's count moving from c to c + m leaves
// class min(c, 4) and enters class min(c + m, 4) (classes 1, 2, 3, 4+), and
// c == 0 makes it a new distinct key.  Whatever order the increments run in,
// the totals end exact, so the sample's frequency profile needs no scan of
// the count table afterwards.  A thread keeps its own signed deltas
// (d[0] distinct, d[1..4] f1..f4+) and maximum; they are summed per warp and
// per block before they reach the query's counters.
struct FreqAcc {
  int d[5];
  unsigned mx;
  unsigned rows;
};

__device__ __forceinline__ void freq_step(FreqAcc& f, unsigned long long old, unsigned m) {
  const unsigned long long nw = old + m;
  const int co = old < 4 ? int(old) : 4, cn = nw < 4 ? int(nw) : 4;
  if (old == 0) f.d[0] += 1;
#pragma unroll
  for (int c = 1; c <= 4; ++c) f.d[c] += (c == cn) - (c == co);
  const unsigned nw32 = nw < 0xffffffffull ? unsigned(nw) : 0xffffffffu;
  f.mx = f.mx > nw32 ? f.mx : nw32;
  f.rows += m;
}

// First insert of a sampled key into its query's count table (linear
// probing from slot s); returns the key's count before this one's m rows.
__device__ __noinline__ unsigned long long est_count_insert(unsigned long long* table, uint64_t cap, uint64_t k,
                                                            uint64_t s, unsigned m) {
  for (uint64_t p = 0; p < cap; ++p) {
    unsigned long long* slot = table + 2 * s;
    const unsigned long long cur = __ldcg(slot);
    if (cur == k) return atomicAdd(slot + 1, (unsigned long long)m);
    if (cur == EMPTY64) {
      const unsigned long long prev = atomicCAS(slot, EMPTY64, k);
      if (prev == EMPTY64 || prev == k) return atomicAdd(slot + 1, (unsigned long long)m);
    }
    s = s + 1 == cap ? 0 : s + 1;
  }
  return 0ull;  // unreachable: the table holds 1.5x the sample
}

// One block per chunk of GBA_EST_CHUNK_TILES sampled tiles of one query (a
// flat grid over every query's chunks).  Per sampled row: the 64 HLL
// registers (block-local, merged once), and the query's count table (keys +
// counts, linear probing, capacity 1.5x the sample).  Lanes of a warp
// holding the same key add their rows with one atomic from the lowest of
// them (a skewed column's hot key would otherwise serialise thousands of
// atomics on one counter).  A thread works on kEstU rows at a time, each
// step's loads and atomics issued before any result is used.
constexpr int kEstThreads = 256;
constexpr int kEstU = 4;
__global__ void __launch_bounds__(kEstThreads) k_est_sample(const EstQuery* qs, int nq) {
  __shared__ unsigned long long sf[7];
  __shared__ unsigned s_hll[64];
  int lo = 0, hi = nq - 1;
  while (lo < hi) {  // last query whose first block is at or before this one
    const int mid = (lo + hi + 1) >> 1;
    if (qs[mid].chunk_base <= int64_t(blockIdx.x)) lo = mid;
    else hi = mid - 1;
  }
  const EstQuery e = qs[lo];
  const int64_t chunk = int64_t(blockIdx.x) - e.chunk_base;
  if (chunk >= e.nchunks) return;  // past the last query's blocks (block-uniform)
  if (threadIdx.x < 7) sf[threadIdx.x] = 0ull;
  if (threadIdx.x < 64) s_hll[threadIdx.x] = 0u;
  __syncthreads();
  const int64_t items = int64_t(e.sampled_tiles) << 10;
  const int64_t c0 = chunk * (int64_t(GBA_EST_CHUNK_TILES) << 10);
  const int64_t c1 = c0 + (int64_t(GBA_EST_CHUNK_TILES) << 10) < items ? c0 + (int64_t(GBA_EST_CHUNK_TILES) << 10) : items;
  FreqAcc f;
#pragma unroll
  for (int c = 0; c < 5; ++c) f.d[c] = 0;
  f.mx = 0u;
  f.rows = 0u;
  unsigned long long ones = 0ull;  // rows of the all-ones key (64-bit keys only)
  // every thread runs the same number of steps (whole warps, for __match_any_sync)
  for (int64_t base = c0; base < c1; base += int64_t(kEstThreads) * kEstU) {
    uint64_t k[kEstU];
    bool live[kEstU];
#pragma unroll
    for (int u = 0; u < kEstU; ++u) {
      const int64_t it = base + int64_t(u) * kEstThreads + threadIdx.x;
      const uint64_t r = it < c1 ? sample_row(e, it) : ~0ull;
      live[u] = r != ~0ull;
      k[u] = 0;
      if (live[u])
        k[u] = e.key64 ? __ldcs(static_cast<const unsigned long long*>(e.keys) + r)
                       : __ldcs(static_cast<const unsigned*>(e.keys) + r);
    }
    unsigned m[kEstU];
    uint64_t s[kEstU];
    unsigned long long cur[kEstU];
#pragma unroll
    for (int u = 0; u < kEstU; ++u) {
      if (live[u]) {
        const uint32_t h = e.key64 ? murmur3_64(k[u], 0x5bd1e995u) : murmur3_32(uint32_t(k[u]), 0x5bd1e995u);
        // HLL: the top 6 bits select the register, the rank of the first set
        // bit among the remaining 26 is its candidate value
        atomicMax(&s_hll[h >> 26], unsigned(__clz((h << 6) | (1u << 5)) + 1));
      }
      const unsigned live_mask = __ballot_sync(GBA_FULL_MASK, live[u]);
      const unsigned peers = __match_any_sync(GBA_FULL_MASK, live[u] ? k[u] : ~0ull) & live_mask;
      // the group's lowest lane carries its m rows; the others drop out
      m[u] = (live[u] && !(peers & ((1u << lane_id()) - 1u))) ? unsigned(__popc(peers)) : 0u;
      s[u] = 0;
      cur[u] = EMPTY64;
      if (m[u] && k[u] != EMPTY64) {
        s[u] = (uint64_t(table_hash(k[u])) * e.cap) >> 32;
        cur[u] = __ldcg(e.table + 2 * s[u]);
      }
    }
    unsigned long long old[kEstU];
#pragma unroll
    for (int u = 0; u < kEstU; ++u) {
      old[u] = 0ull;
      if (m[u] && k[u] != EMPTY64 && cur[u] == k[u]) old[u] = atomicAdd(e.table + 2 * s[u] + 1, (unsigned long long)m[u]);
    }
#pragma unroll
    for (int u = 0; u < kEstU; ++u) {
      if (!m[u]) continue;
      if (k[u] == EMPTY64) {  // the table's empty marker (only a 64-bit key can equal it)
        ones += m[u];
        continue;
      }
      if (cur[u] != k[u]) old[u] = est_count_insert(e.table, e.cap, k[u], s[u], m[u]);
      freq_step(f, old[u], m[u]);
    }
  }
  // the all-ones key's count: its old value decides its frequency class, so it
  // takes one atomic per thread that saw it
  if (ones) freq_step(f, atomicAdd(&e.stats[3], ones), unsigned(ones));
  // warp sums, then one shared update per warp
#pragma unroll
  for (int c = 0; c < 5; ++c) f.d[c] = __reduce_add_sync(GBA_FULL_MASK, f.d[c]);
  f.mx = __reduce_max_sync(GBA_FULL_MASK, f.mx);
  f.rows = __reduce_add_sync(GBA_FULL_MASK, f.rows);
  if (lane_id() == 0) {
#pragma unroll
    for (int c = 0; c < 5; ++c)
      if (f.d[c]) atomicAdd(&sf[c], (unsigned long long)(long long)f.d[c]);
    if (f.mx) atomicMax(&sf[5], (unsigned long long)f.mx);
    if (f.rows) atomicAdd(&sf[6], (unsigned long long)f.rows);
  }
  __syncthreads();
  if (threadIdx.x < 7 && sf[threadIdx.x] != 0ull) {
    if (threadIdx.x == 5) atomicMax(&e.freq[5], sf[5]);
    else atomicAdd(&e.freq[threadIdx.x], sf[threadIdx.x]);
  }
  if (threadIdx.x < 64 && s_hll[threadIdx.x] > __ldcg(&e.hll[threadIdx.x])) atomicMax(&e.hll[threadIdx.x], s_hll[threadIdx.x]);
}

// per query (one thread each): frequency profile and HLL registers -> the 32
// features
__global__ void k_est_reduce(const EstQuery* qs, int nq) {
  for (int qi = blockIdx.x * blockDim.x + threadIdx.x; qi < nq; qi += gridDim.x * blockDim.x) {
    const EstQuery e = qs[qi];
    unsigned long long acc[7];
#pragma unroll
    for (int i = 0; i < 7; ++i) acc[i] = e.freq[i];
    float* f = e.feat;
    const double n = double(e.n), s = double(acc[6] > 0 ? acc[6] : 1);
    const double dd = double(acc[0]), a1 = double(acc[1]), a2 = double(acc[2]);
    const double gee = sqrt(n / s) * a1 + (dd - a1);
    const double chao = dd + a1 * a1 / (2.0 * (a2 > 1 ? a2 : 1.0));
    // HLL estimate (m = 64, alpha_64 = 0.709) with the small-range correction
    double z = 0;
    int zeros = 0;
    int hist[16] = {0};
    for (int r = 0; r < 64; ++r) {
      const unsigned v = e.hll[r];
      z += ldexp(1.0, -int(v));
      zeros += v == 0;
      hist[v < 15 ? v : 15]++;
    }
    double hll = 0.709 * 64 * 64 / z;
    if (hll <= 2.5 * 64 && zeros > 0) hll = 64 * log(64.0 / zeros);
    f[0] = float(log2(n + 1) / 32);
    f[1] = float(log2(s + 1) / 32);
    f[2] = float(dd / s);
    f[3] = float(a1 / s);
    f[4] = float(a2 / s);
    f[5] = float(double(acc[3]) / s);
    f[6] = float(double(acc[4]) / s);
    f[7] = float(log2(dd + 1) / 32);
    f[8] = float(log2(gee + 1) / 32);
    f[9] = float(log2(chao + 1) / 32);
    f[10] = float(log2(hll + 1) / 32);
    f[11] = float(double(acc[5]) / s);
    f[12] = e.key64 ? 1.0f : 0.5f;
    f[13] = float(s / (n > 0 ? n : 1));
    for (int i = 0; i < 16; ++i) f[14 + i] = float(hist[i]) / 64.0f;
    f[30] = float(log2(n / s > 1 ? n / s : 1) / 32);
    f[31] = 1.0f;
    e.stats[0] = acc[0];
    e.stats[1] = acc[5];
    e.stats[2] = acc[6];
  }
}

// ---- MLP ------------------------------------------------------------------------
__device__ __forceinline__ float relu(float x) { return x > 0.f ? x : 0.f; }

// Inference: a CTA of H threads takes kFwdRows samples; thread j computes
// hidden unit j of every sample of the CTA, activations stay in shared memory
// and the output unit is a warp-shuffle sum over the hidden units.
constexpr int kFwdRows = 8;
__global__ void __launch_bounds__(H) k_mlp_forward(const float* __restrict__ W, const float* __restrict__ X, int n,
                                                   float* __restrict__ out) {
  __shared__ float xs[kFwdRows][F];
  __shared__ float ha[kFwdRows][H];
  __shared__ float hb[kFwdRows][H];
  __shared__ float part[kFwdRows][H / 32];
  const int j = threadIdx.x;
  for (int b0 = blockIdx.x * kFwdRows; b0 < n; b0 += gridDim.x * kFwdRows) {
    const int rows = n - b0 < kFwdRows ? n - b0 : kFwdRows;
    for (int i = j; i < kFwdRows * F; i += H) xs[i / F][i % F] = i / F < rows ? X[size_t(b0) * F + i] : 0.f;
    __syncthreads();
    float acc[kFwdRows];
#pragma unroll
    for (int r = 0; r < kFwdRows; ++r) acc[r] = __ldg(W + OB1 + j);
    for (int i = 0; i < F; ++i) {
      const float w = __ldg(W + OW1 + j * F + i);
#pragma unroll
      for (int r = 0; r < kFwdRows; ++r) acc[r] = fmaf(w, xs[r][i], acc[r]);
    }
#pragma unroll
    for (int r = 0; r < kFwdRows; ++r) ha[r][j] = relu(acc[r]);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kFwdRows; ++r) acc[r] = __ldg(W + OB2 + j);
    for (int i = 0; i < H; ++i) {
      const float w = __ldg(W + OW2 + j * H + i);
#pragma unroll
      for (int r = 0; r < kFwdRows; ++r) acc[r] = fmaf(w, ha[r][i], acc[r]);
    }
#pragma unroll
    for (int r = 0; r < kFwdRows; ++r) hb[r][j] = relu(acc[r]);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kFwdRows; ++r) acc[r] = __ldg(W + OB3 + j);
    for (int i = 0; i < H; ++i) {
      const float w = __ldg(W + OW3 + j * H + i);
#pragma unroll
      for (int r = 0; r < kFwdRows; ++r) acc[r] = fmaf(w, hb[r][i], acc[r]);
    }
    const float w4 = __ldg(W + OW4 + j);
#pragma unroll
    for (int r = 0; r < kFwdRows; ++r) {
      float v = w4 * relu(acc[r]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(GBA_FULL_MASK, v, o);
      if ((j & 31) == 0) part[r][j >> 5] = v;
    }
    __syncthreads();
    if (j < rows) {
      float y = __ldg(W + OB4);
#pragma unroll
      for (int w = 0; w < H / 32; ++w) y += part[j][w];
      out[b0 + j] = y;
    }
    __syncthreads();
  }
}

// One training step on a batch (single CTA): forward, MSE loss, backward;
// writes the gradient of every parameter (no atomics: each gradient element is
// one thread's sum over the batch) and the batch loss.
constexpr int kTrainB = 128;
__global__ void __launch_bounds__(1024) k_mlp_fwd_bwd(const float* __restrict__ W, const float* __restrict__ X,
                                                      const float* __restrict__ T, const int* __restrict__ idx,
                                                      int B, float* __restrict__ G, float* __restrict__ loss) {
  extern __shared__ float sm[];
  float* x = sm;                  // [B][F]
  float* a1 = x + kTrainB * F;    // [B][H]  (post-ReLU)
  float* a2 = a1 + kTrainB * H;
  float* a3 = a2 + kTrainB * H;
  float* d = a3 + kTrainB * H;    // [B][H] delta buffer
  float* d2 = d + kTrainB * H;    // [B][H]
  float* dy = d2 + kTrainB * H;   // [B]
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < B * F; i += nt) {
    const int b = i / F, f = i % F;
    x[i] = X[size_t(idx ? idx[b] : b) * F + f];
  }
  __syncthreads();
  auto dense = [&](const float* in, int nin, float* outp, int wofs, int bofs) {
    for (int o = tid; o < B * H; o += nt) {
      const int b = o / H, j = o % H;
      float a = W[bofs + j];
      for (int i = 0; i < nin; ++i) a = fmaf(W[wofs + j * nin + i], in[b * nin + i], a);
      outp[o] = relu(a);
    }
    __syncthreads();
  };
  dense(x, F, a1, OW1, OB1);
  dense(a1, H, a2, OW2, OB2);
  dense(a2, H, a3, OW3, OB3);
  __shared__ float s_loss;
  if (tid == 0) s_loss = 0.f;
  __syncthreads();
  for (int b = tid; b < B; b += nt) {
    float y = W[OB4];
    for (int j = 0; j < H; ++j) y = fmaf(W[OW4 + j], a3[b * H + j], y);
    const float t = T[idx ? idx[b] : b];
    const float e = y - t;
    dy[b] = 2.f * e / float(B);
    atomicAdd(&s_loss, e * e / float(B));
  }
  __syncthreads();
  // output layer
  for (int j = tid; j < H + 1; j += nt) {
    float g = 0.f;
    if (j < H)
      for (int b = 0; b < B; ++b) g = fmaf(dy[b], a3[b * H + j], g);
    else
      for (int b = 0; b < B; ++b) g += dy[b];
    G[j < H ? OW4 + j : OB4] = g;
  }
  for (int o = tid; o < B * H; o += nt) {
    const int b = o / H, j = o % H;
    d[o] = a3[o] > 0.f ? dy[b] * W[OW4 + j] : 0.f;
  }
  __syncthreads();
  // hidden layers: given delta d at layer L's output (post-ReLU mask applied),
  // gW[j][i] = sum_b d[b][j] in[b][i], gb[j] = sum_b d[b][j],
  // d_in[b][i] = (sum_j d[b][j] W[j][i]) * (in[b][i] > 0)
  auto back = [&](const float* in, int nin, int wofs, int bofs, float* dnext, bool mask) {
    for (int w = tid; w < H * nin + H; w += nt) {
      float g = 0.f;
      if (w < H * nin) {
        const int j = w / nin, i = w % nin;
        for (int b = 0; b < B; ++b) g = fmaf(d[b * H + j], in[b * nin + i], g);
        G[wofs + w] = g;
      } else {
        const int j = w - H * nin;
        for (int b = 0; b < B; ++b) g += d[b * H + j];
        G[bofs + j] = g;
      }
    }
    if (dnext) {
      for (int o = tid; o < B * nin; o += nt) {
        const int b = o / nin, i = o % nin;
        float s = 0.f;
        for (int j = 0; j < H; ++j) s = fmaf(d[b * H + j], W[wofs + j * nin + i], s);
        dnext[o] = (mask && in[o] <= 0.f) ? 0.f : s;
      }
    }
    __syncthreads();
  };
  back(a2, H, OW3, OB3, d2, true);
  for (int o = tid; o < B * H; o += nt) d[o] = d2[o];
  __syncthreads();
  back(a1, H, OW2, OB2, d2, true);
  for (int o = tid; o < B * H; o += nt) d[o] = d2[o];
  __syncthreads();
  back(x, F, OW1, OB1, nullptr, false);
  if (tid == 0 && loss) *loss = s_loss;
}

__global__ void k_adam(float* W, const float* G, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = G[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    W[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

size_t train_smem() { return sizeof(float) * (size_t(kTrainB) * (F + 5 * H) + kTrainB); }

}  // namespace

// ---------------------------------------------------------------------------
// launchers
cudaError_t gba_launch_est_sample(const EstQuery* d_qs, int nq, int64_t total_chunks, cudaStream_t s) {
  // a flat grid: one block per chunk of GBA_EST_CHUNK_TILES sampled tiles of
  // a query, so every query gets as many blocks as its sample needs (a grid
  // of queries x the largest query's blocks left most blocks empty)
  if (nq <= 0 || total_chunks <= 0) return cudaSuccess;
  if (total_chunks > int64_t(0x7fffffff)) return cudaErrorInvalidValue;
  k_est_sample<<<unsigned(total_chunks), kEstThreads, 0, s>>>(d_qs, nq);
  return cudaGetLastError();
}
cudaError_t gba_launch_est_init(const EstQuery* d_qs, int nq, cudaStream_t s) {
  if (nq <= 0) return cudaSuccess;
  k_est_init<<<dim3(64, std::min(nq, 65535)), 256, 0, s>>>(d_qs, nq);
  return cudaGetLastError();
}
cudaError_t gba_launch_est_reduce(const EstQuery* d_qs, int nq, cudaStream_t s) {
  if (nq <= 0) return cudaSuccess;
  k_est_reduce<<<(nq + 127) / 128, 128, 0, s>>>(d_qs, nq);
  return cudaGetLastError();
}
cudaError_t gba_launch_mlp_forward(const float* W, const float* X, int n, float* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_mlp_forward<<<std::min((n + kFwdRows - 1) / kFwdRows, 1184), H, 0, s>>>(W, X, n, out);
  return cudaGetLastError();
}

int64_t gba_est_nparam() { return NPARAM; }

// Sizes an EstQuery for a query of n rows: sampled tiles, table capacity.
void gba_est_plan(EstQuery* e, int64_t n, int64_t tile_rows) {
  e->n = n;
  e->tile_rows = tile_rows > 0 ? tile_rows : 65536;
  const int64_t ntiles = (n + e->tile_rows - 1) / e->tile_rows;
  e->tile_step = std::max<int64_t>(1, (ntiles + GBA_EST_MAX_TILES - 1) / GBA_EST_MAX_TILES);
  e->sampled_tiles = int((ntiles + e->tile_step - 1) / e->tile_step);
  const uint64_t s_max = uint64_t(e->sampled_tiles) * 1024;
  // load <= 2/3 (slots are addressed by a multiply-shift, so any capacity
  // works; a power of two would cost up to 2x the table clear and footprint)
  e->cap = std::max<uint64_t>(64, s_max + s_max / 2);
}

// ---- host API ---------------------------------------------------------------------
static gba_status est_ensure(gba_context* ctx) {
  if (ctx->d_est) return GBA_OK;
  // params, Adam m, Adam v, grads, loss, scratch
  GBA_CUDA_TRY(ctx, cudaMalloc(&ctx->d_est, sizeof(float) * (4 * size_t(NPARAM) + 64)));
  GBA_CUDA_TRY(ctx, cudaMemset(ctx->d_est, 0, sizeof(float) * (4 * size_t(NPARAM) + 64)));
  return GBA_OK;
}

extern "C" int64_t gba_estimator_param_count(void) { return NPARAM; }

extern "C" gba_status gba_estimator_load(gba_context* ctx, const float* params) {
  if (!ctx || !params) return GBA_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  gba_status st = est_ensure(ctx);
  if (st != GBA_OK) return st;
  GBA_CUDA_TRY(ctx, cudaMemcpy(ctx->d_est, params, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
  GBA_CUDA_TRY(ctx, cudaMemset(ctx->d_est + NPARAM, 0, sizeof(float) * 2 * NPARAM));
  ctx->est_loaded = true;
  return GBA_OK;
}

extern "C" gba_status gba_estimator_get(gba_context* ctx, float* params) {
  if (!ctx || !params || !ctx->d_est) return GBA_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  GBA_CUDA_TRY(ctx, cudaMemcpy(params, ctx->d_est, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
  return GBA_OK;
}

extern "C" gba_status gba_estimator_predict(gba_context* ctx, int32_t n, const float* feats, float* out) {
  if (!ctx || n < 0 || (n > 0 && (!feats || !out))) return GBA_ERR_INVALID_ARG;
  if (!ctx->est_loaded) {
    ctx->err = "no estimator weights loaded";
    return GBA_ERR_INVALID_ARG;
  }
  cudaSetDevice(ctx->device);
  const size_t bytes = sizeof(float) * (size_t(n) * F + n);
  gba_status st = gba_stage_reserve(ctx, bytes, 0);
  if (st != GBA_OK) return st;
  float* X = static_cast<float*>(ctx->stage);
  float* Y = X + size_t(n) * F;
  GBA_CUDA_TRY(ctx, cudaMemcpy(X, feats, sizeof(float) * size_t(n) * F, cudaMemcpyHostToDevice));
  GBA_CUDA_TRY(ctx, gba_launch_mlp_forward(ctx->d_est, X, n, Y, 0));
  GBA_CUDA_TRY(ctx, cudaMemcpy(out, Y, sizeof(float) * n, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; ++i) out[i] *= 32.f;  // t -> log2(groups)
  return GBA_OK;
}

// upload a training set into the staging buffer: X, T (t = log2/32), idx
static gba_status stage_training(gba_context* ctx, int32_t n, const float* feats, const float* target, float** X,
                                 float** T, int** idx) {
  const size_t bytes = sizeof(float) * (size_t(n) * F + n) + sizeof(int) * n + 256;
  gba_status st = gba_stage_reserve(ctx, bytes, 0);
  if (st != GBA_OK) return st;
  *X = static_cast<float*>(ctx->stage);
  *T = *X + size_t(n) * F;
  *idx = reinterpret_cast<int*>(*T + n);
  std::vector<float> t(target, target + n);
  for (auto& v : t) v /= 32.f;
  GBA_CUDA_TRY(ctx, cudaMemcpy(*X, feats, sizeof(float) * size_t(n) * F, cudaMemcpyHostToDevice));
  GBA_CUDA_TRY(ctx, cudaMemcpy(*T, t.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  return GBA_OK;
}

extern "C" gba_status gba_estimator_grad(gba_context* ctx, int32_t n, const float* feats, const float* target,
                                         float* grads, float* loss) {
  if (!ctx || n <= 0 || n > kTrainB || !feats || !target || !grads) return GBA_ERR_INVALID_ARG;
  if (!ctx->est_loaded) {
    ctx->err = "no estimator weights loaded";
    return GBA_ERR_INVALID_ARG;
  }
  cudaSetDevice(ctx->device);
  float *X, *T;
  int* idx;
  gba_status st = stage_training(ctx, n, feats, target, &X, &T, &idx);
  if (st != GBA_OK) return st;
  float* G = ctx->d_est + 3 * size_t(NPARAM);
  float* L = G + NPARAM;
  GBA_CUDA_TRY(ctx, cudaFuncSetAttribute(k_mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, int(train_smem())));
  k_mlp_fwd_bwd<<<1, 1024, train_smem()>>>(ctx->d_est, X, T, nullptr, n, G, L);
  GBA_CUDA_TRY(ctx, cudaGetLastError());
  GBA_CUDA_TRY(ctx, cudaMemcpy(grads, G, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
  if (loss) GBA_CUDA_TRY(ctx, cudaMemcpy(loss, L, sizeof(float), cudaMemcpyDeviceToHost));
  return GBA_OK;
}

extern "C" gba_status gba_estimator_train(gba_context* ctx, int32_t n, const float* feats, const float* target,
                                          int32_t epochs, int32_t batch, float lr, uint64_t seed, float* final_loss) {
  if (!ctx || n <= 0 || !feats || !target || epochs < 0) return GBA_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  gba_status st = est_ensure(ctx);
  if (st != GBA_OK) return st;
  if (!ctx->est_loaded) {
    ctx->err = "initialise the weights with gba_estimator_load first";
    return GBA_ERR_INVALID_ARG;
  }
  const int B = std::max(1, std::min<int>(batch > 0 ? batch : kTrainB, kTrainB));
  float *X, *T;
  int* idx;
  st = stage_training(ctx, n, feats, target, &X, &T, &idx);
  if (st != GBA_OK) return st;
  float* W = ctx->d_est;
  float* M = W + NPARAM;
  float* V = M + NPARAM;
  float* G = V + NPARAM;
  float* L = G + NPARAM;
  GBA_CUDA_TRY(ctx, cudaMemset(M, 0, sizeof(float) * 2 * NPARAM));
  GBA_CUDA_TRY(ctx, cudaFuncSetAttribute(k_mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, int(train_smem())));
  std::vector<int> perm(n);
  uint64_t state = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto rnd = [&]() {
    state = state * 6364136223846793005ull + 1442695040888963407ull;
    return uint32_t(state >> 33);
  };
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  int64_t step = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = n - 1; i > 0; --i) std::swap(perm[i], perm[rnd() % uint32_t(i + 1)]);
    GBA_CUDA_TRY(ctx, cudaMemcpy(idx, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    const float lr_ep = lr * (ep < epochs * 3 / 4 ? 1.0f : 0.1f);
    for (int b0 = 0; b0 + B <= n; b0 += B) {
      ++step;
      k_mlp_fwd_bwd<<<1, 1024, train_smem()>>>(W, X, T, idx + b0, B, G, nullptr);
      const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
      k_adam<<<(NPARAM + 255) / 256, 256>>>(W, G, M, V, NPARAM, lr_ep, b1, b2, eps, c1, c2);
    }
  }
  GBA_CUDA_TRY(ctx, cudaGetLastError());
  if (final_loss) {
    // mean squared error over the whole set, in (log2 groups)^2
    GBA_CUDA_TRY(ctx, cudaDeviceSynchronize());
    std::vector<float> yh(n), tt(n);
    float* Yd = nullptr;
    GBA_CUDA_TRY(ctx, cudaMalloc(&Yd, sizeof(float) * n));
    GBA_CUDA_TRY(ctx, gba_launch_mlp_forward(W, X, n, Yd, 0));
    GBA_CUDA_TRY(ctx, cudaMemcpy(yh.data(), Yd, sizeof(float) * n, cudaMemcpyDeviceToHost));
    GBA_CUDA_TRY(ctx, cudaMemcpy(tt.data(), T, sizeof(float) * n, cudaMemcpyDeviceToHost));
    cudaFree(Yd);
    double se = 0;
    for (int i = 0; i < n; ++i) {
      const double e = 32.0 * (double(yh[i]) - double(tt[i]));
      se += e * e;
    }
    *final_loss = float(se / n);
  }
  return GBA_OK;
}

// Features of a batch of device queries (internal; used by learned sizing and
// the batch path).  feats_out: device [nq][32]; stats_out: device [nq][4].
gba_status gba_est_features_device(gba_context* ctx, const QDesc* qs, int nq, int64_t tile_rows, cudaStream_t s,
                                   float** feats_out, unsigned long long** stats_out) {
  std::vector<EstQuery> eq(nq);
  size_t off = 0;
  auto take = [&](size_t b) {
    const size_t o = off;
    off = gba_round_up(off + b, 256);
    return o;
  };
  const size_t o_q = take(sizeof(EstQuery) * nq);
  const size_t o_f = take(sizeof(float) * F * nq);
  const size_t o_s = take(8 * 4 * size_t(nq));
  const size_t o_h = take(4 * 64 * size_t(nq));
  const size_t o_fr = take(8 * 8 * size_t(nq));
  std::vector<size_t> o_t(nq);
  int64_t chunks = 0;
  for (int i = 0; i < nq; ++i) {
    gba_est_plan(&eq[i], qs[i].n, tile_rows);
    o_t[i] = take(16 * eq[i].cap);
    eq[i].chunk_base = chunks;
    eq[i].nchunks = (eq[i].sampled_tiles + GBA_EST_CHUNK_TILES - 1) / GBA_EST_CHUNK_TILES;
    chunks += eq[i].nchunks;
  }
  gba_status st = gba_est_reserve(ctx, off, s);
  if (st != GBA_OK) return st;
  unsigned char* base = static_cast<unsigned char*>(ctx->est_ws);
  for (int i = 0; i < nq; ++i) {
    eq[i].keys = qs[i].keys;
    eq[i].key64 = qs[i].key64;
    eq[i].table = reinterpret_cast<unsigned long long*>(base + o_t[i]);
    eq[i].hll = reinterpret_cast<unsigned*>(base + o_h) + 64 * i;
    eq[i].feat = reinterpret_cast<float*>(base + o_f) + F * i;
    eq[i].stats = reinterpret_cast<unsigned long long*>(base + o_s) + 4 * i;
    eq[i].freq = reinterpret_cast<unsigned long long*>(base + o_fr) + 8 * i;
  }
  GBA_CUDA_TRY(ctx, cudaMemsetAsync(base + o_h, 0, 4 * 64 * size_t(nq), s));
  GBA_CUDA_TRY(ctx, cudaMemsetAsync(base + o_s, 0, 8 * 4 * size_t(nq), s));
  GBA_CUDA_TRY(ctx, cudaMemsetAsync(base + o_fr, 0, 8 * 8 * size_t(nq), s));
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(base + o_q, eq.data(), sizeof(EstQuery) * nq, cudaMemcpyHostToDevice, s));
  const EstQuery* dq = reinterpret_cast<const EstQuery*>(base + o_q);
  GBA_CUDA_TRY(ctx, gba_launch_est_init(dq, nq, s));
  GBA_CUDA_TRY(ctx, gba_launch_est_sample(dq, nq, chunks, s));
  GBA_CUDA_TRY(ctx, gba_launch_est_reduce(dq, nq, s));
  *feats_out = reinterpret_cast<float*>(base + o_f);
  *stats_out = reinterpret_cast<unsigned long long*>(base + o_s);
  ctx->stats.kernel_launches += 3;
  return GBA_OK;
}

extern "C" gba_status gba_estimator_features(gba_context* ctx, const gba_query* q, int64_t tile_rows, void* stream,
                                             float* out) {
  if (!ctx || !q || !out) return GBA_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  QDesc qd;
  gba_status st = gba_build_qdesc(ctx, q, &qd);
  if (st != GBA_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float* f;
  unsigned long long* stats;
  st = gba_est_features_device(ctx, &qd, 1, tile_rows, s, &f, &stats);
  if (st != GBA_OK) return st;
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(out, f, sizeof(float) * F, cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return GBA_OK;
}

// Learned sizing for one query: features, forward pass, clamp to [d, n].
gba_status gba_predict_groups(gba_context* ctx, const QDesc& q, cudaStream_t s, double* groups) {
  if (!ctx->est_loaded) {
    ctx->err = "no estimator weights loaded";
    return GBA_ERR_INVALID_ARG;
  }
  float* f;
  unsigned long long* stats;
  gba_status st = gba_est_features_device(ctx, &q, 1, 0, s, &f, &stats);
  if (st != GBA_OK) return st;
  // forward into the small host-visible scratch
  float* y = reinterpret_cast<float*>(ctx->d_small + 1024);
  GBA_CUDA_TRY(ctx, gba_launch_mlp_forward(ctx->d_est, f, 1, y, s));
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_small + 1024, y, 4, cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_small + 1032, stats, 32, cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_small + 1088, f, F * sizeof(float), cudaMemcpyDeviceToHost, s));
  GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  ctx->stats.kernel_launches += 1;
  const float t = *reinterpret_cast<float*>(ctx->h_small + 1024);
  const unsigned long long d = *reinterpret_cast<unsigned long long*>(ctx->h_small + 1032);
  const float* feat = reinterpret_cast<const float*>(ctx->h_small + 1088);
  double g = exp2(double(t) * 32.0);
  g = std::max(g, double(d));
  // Beyond the row counts the network was trained on it extrapolates; there
  // it is not trusted below the Chao1 estimate of the same sample (which is
  // close when the sample is mostly singletons, the case a small sample of a
  // very large high-cardinality column gives).  An over-estimate only costs
  // a larger table; an under-estimate costs a re-run.
  if (q.n > GBA_EST_TRAINED_MAX_ROWS) g = std::max(g, exp2(double(feat[9]) * 32.0) - 1.0);
  g = std::min(g, double(std::max<int64_t>(q.n, 1)));
  *groups = g;
  // share of the sample taken by its most frequent key (skew signal)
  ctx->est_skew = double(*reinterpret_cast<unsigned long long*>(ctx->h_small + 1040)) /
                  double(std::max<unsigned long long>(1, *reinterpret_cast<unsigned long long*>(ctx->h_small + 1048)));
  return GBA_OK;
}
