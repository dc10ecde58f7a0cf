// Host driver of the radix-partition strategy and the strategy choice.
//
// Fan-out: the reference uses a fixed P=300 (test/test.cu:96) and then merges
// small partitions greedily so each merged partition fills a global table of
// `Capacity` slots (groupby_agg_intra_partition.cu:13-48).  Here the fan-out is
// chosen so that every final partition's groups fill a quarter of one CTA's
// shared-memory table: bits = ceil(log2(groups / (S / 4))), split over one or
// two MSD passes (two from 10 bits on) so each scatter pass keeps its write
// runs long.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "gba_context.h"
#include "gba_plan.h"
#include "part_kernels.h"

namespace {

constexpr size_t kAlign = 256;
int tbytes(int t) { return gba_type_bytes(t); }

struct Carver {
  size_t off = 0;
  size_t take(size_t bytes) {
    const size_t o = off;
    off = gba_round_up(off + bytes, kAlign);
    return o;
  }
};

size_t row_bytes(const QDesc& q) {
  size_t b = q.key64 ? 8 : 4;
  for (int c = 0; c < q.ncols; ++c) b += tbytes(q.col_type[c]);
  return b;
}

}  // namespace

// shared-memory slots one partition table can use
static int part_table_slots(const gba_context* ctx, const QDesc& q) {
  const size_t slot = (q.key64 ? 8 : 4) + 4 * size_t(q.nwords);
  // 2 KB stay free for the kernel's static shared memory, the side slot and
  // alignment
  const size_t room = size_t(ctx->max_smem_optin) - 2048;
  return int(std::min<size_t>(16384, room / slot));
}

int gba_choose_strategy(const gba_context* ctx, const QDesc& q, const gba_knobs& k, double predicted_groups,
                        const GbaPlan& p) {
  (void)k;
  // The HBM-table strategy is fast while its table stays resident in L2
  // (126 MB; measured: random 64-bit atomics run at ~190 G/s below ~96 MB of
  // table and fall to 20-60 G/s above it).  Beyond that the partition
  // strategy's shared-memory tables win.
  const double slot = 8.0 * gba_gt_stride(q.naccs);
  const double groups = predicted_groups > 0 ? predicted_groups : double(q.n);
  (void)p;
  if (groups <= 0.55 * part_table_slots(ctx, q)) return GBA_STRATEGY_TABLE;  // shared table holds all groups
  const double table_bytes = groups / 0.7 * slot;
  return table_bytes <= 80.0 * (1 << 20) ? GBA_STRATEGY_TABLE : GBA_STRATEGY_PARTITION;
}

gba_status gba_run_partition(gba_context* ctx, const QDesc& q, const gba_output* out, const gba_knobs& k,
                             const GbaPlan& p, double predicted_groups, cudaStream_t s, int64_t* n_groups) {
  ctx->stats.strategy = GBA_STRATEGY_PARTITION;
  const int64_t n = q.n;
  int S = part_table_slots(ctx, q);
  if (k.smem_slots > 0) S = std::max(32, std::min(S, k.smem_slots));
  // groups aimed at per partition: a quarter of the shared table (measured on
  // B200, best or within 8% of the best fan-out on the 2^28-row high-cardinality
  // query (16 bits), the 2^27-row serving query (14) and the 2^26-row skewed
  // query (11 vs 12); fuller tables make k_part_agg probe longer)
  const double per_table = 0.25 * S;
  double groups = double(std::max<int64_t>(n, 1));
  if (k.sizing == GBA_SIZING_LEARNED && predicted_groups > 0) groups = std::min(groups, predicted_groups * 1.25 + 64);
  int B = k.partition_bits > 0 ? k.partition_bits : int(std::ceil(std::log2(std::max(1.0, groups / per_table))));
  B = std::max(1, std::min(B, 20));
  const int T = 2048;  // scatter tile rows (<= 4 per thread of k_part_scatter's 512)
  const int64_t L = std::max<int64_t>(T, ((n + int64_t(ctx->sms) * 8 - 1) / (int64_t(ctx->sms) * 8) + T - 1) / T * T);
  const size_t rb = row_bytes(q);

  for (int attempt = 0;; ++attempt) {
    std::vector<int> passes;
    // one pass up to 512 digits; beyond that two passes (measured on the
    // 2^26-row skewed query: 10 bits in one pass scatter 1.5x slower than
    // 11 bits in two, a 2048-row tile leaving about 2 rows per digit)
    if (B <= 9) passes = {B};
    else passes = {(B + 1) / 2, B / 2};
    ctx->stats.partition_bits = B;

    // upper bounds for the per-pass arrays
    const int64_t max_chunks = n / L + 2 + (int64_t(1) << passes[0]);
    const int maxb = *std::max_element(passes.begin(), passes.end());
    int64_t max_nseg_in = passes.size() > 1 ? (int64_t(1) << passes[0]) : 1;
    const int64_t max_entries = (int64_t(1) << maxb) * (max_chunks + max_nseg_in);
    const int64_t nseg_final = int64_t(1) << B;
    const uint64_t fb_cap = std::max<uint64_t>(1 << 16, uint64_t(std::min<double>(groups * 0.02, 1 << 24)));

    Carver cv;
    size_t bufA[1 + GBA_MAX_COLS], bufB[1 + GBA_MAX_COLS];
    bufA[0] = cv.take(size_t(n) * (q.key64 ? 8 : 4));
    for (int c = 0; c < q.ncols; ++c) bufA[1 + c] = cv.take(size_t(n) * tbytes(q.col_type[c]));
    if (passes.size() > 1) {
      bufB[0] = cv.take(size_t(n) * (q.key64 ? 8 : 4));
      for (int c = 0; c < q.ncols; ++c) bufB[1 + c] = cv.take(size_t(n) * tbytes(q.col_type[c]));
    }
    const size_t o_chunks = cv.take(sizeof(PartChunk) * size_t(max_chunks + max_nseg_in));
    const size_t o_counts = cv.take(sizeof(unsigned) * size_t(max_entries));
    const size_t o_offsets = cv.take(8 * size_t(max_entries));
    const size_t o_status = cv.take(8 * size_t(max_entries / 2048 + 2));
    const size_t o_cbase = cv.take(8 * size_t(max_nseg_in));
    const size_t o_snch = cv.take(4 * size_t(max_nseg_in));
    const size_t o_segs = cv.take(8 * size_t(nseg_final + 1) * 2);
    // final work items: whole partitions packed up to Lp rows, partitions of
    // more than 2 Lp rows (hot keys) split into pieces of Lp rows
    const int64_t Lp = std::max<int64_t>(32768, n / (int64_t(ctx->sms) * 4));
    const int64_t max_split = n / (2 * Lp) + 1;
    const size_t o_work = cv.take(sizeof(PartWork) * size_t(nseg_final + n / Lp + 2));
    // the fallback table goes last: its final size is known after partitioning
    const size_t fb_slot_bytes = size_t(gba_gt_stride(q.naccs)) * 8;
    const size_t o_fb = cv.take((fb_cap + 1 + uint64_t(max_split) * uint64_t(S) * 2) * fb_slot_bytes);
    gba_status st = gba_ws_reserve(ctx, cv.off, s);
    if (st != GBA_OK) return st;
    unsigned char* W = static_cast<unsigned char*>(ctx->ws);
    unsigned* d_flags = reinterpret_cast<unsigned*>(ctx->d_small);
    unsigned long long* d_count = reinterpret_cast<unsigned long long*>(ctx->d_small + 8);
    unsigned* d_tile_ctr = reinterpret_cast<unsigned*>(ctx->d_small + 16);
    unsigned* d_seg_ctr = reinterpret_cast<unsigned*>(ctx->d_small + 20);
    GBA_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_small, 0, 64, s));
    GbaTimer tm{ctx, s, k.timing != 0};
    int launches = 0;

    auto buf_desc = [&](const size_t* b) {
      QDesc d = q;
      d.keys = W + b[0];
      for (int c = 0; c < q.ncols; ++c) d.cols[c] = W + b[1 + c];
      return d;
    };
    QDesc in = q;
    std::vector<long long> seg_in = {0, (long long)n};  // boundaries of the input segments
    long long* d_seg = reinterpret_cast<long long*>(W + o_segs);
    int shift = 0;
    for (size_t pi = 0; pi < passes.size(); ++pi) {
      const int bits = passes[pi];
      const QDesc outq = buf_desc(pi % 2 == 0 ? bufA : bufB);
      const int nseg_in = int(seg_in.size()) - 1;
      std::vector<PartChunk> chunks;
      std::vector<long long> cbase(nseg_in);
      std::vector<int> snch(nseg_in);
      int64_t entries = 0;
      for (int sg = 0; sg < nseg_in; ++sg) {
        const long long b = seg_in[sg], e = seg_in[sg + 1];
        const int nch = int(std::max<int64_t>(1, (e - b + L - 1) / L));
        cbase[sg] = entries;
        snch[sg] = nch;
        for (int c = 0; c < nch; ++c) {
          PartChunk ch;
          ch.row_begin = b + int64_t(c) * L;
          ch.row_end = std::min<int64_t>(e, ch.row_begin + L);
          ch.count_base = entries;
          ch.seg_nchunks = nch;
          ch.chunk_in_seg = c;
          chunks.push_back(ch);
        }
        entries += (int64_t(1) << bits) * nch;
      }
      GBA_CUDA_TRY(ctx, cudaMemcpyAsync(W + o_chunks, chunks.data(), sizeof(PartChunk) * chunks.size(),
                                        cudaMemcpyHostToDevice, s));
      GBA_CUDA_TRY(ctx, cudaMemcpyAsync(W + o_cbase, cbase.data(), 8 * cbase.size(), cudaMemcpyHostToDevice, s));
      GBA_CUDA_TRY(ctx, cudaMemcpyAsync(W + o_snch, snch.data(), 4 * snch.size(), cudaMemcpyHostToDevice, s));
      PartPass pp;
      pp.in = in;
      // the passes only move bytes: an fp64 column travels as I64, which keeps
      // the scatter's column-width test the single compare it is tuned for
      for (int c = 0; c < pp.in.ncols; ++c)
        if (pp.in.col_type[c] == GBA_F64) pp.in.col_type[c] = GBA_I64;
      pp.out = outq;
      pp.chunks = reinterpret_cast<const PartChunk*>(W + o_chunks);
      pp.nchunks = int(chunks.size());
      pp.shift_hi = shift;
      pp.bits = bits;
      pp.counts = reinterpret_cast<unsigned*>(W + o_counts);
      pp.offsets = reinterpret_cast<const unsigned long long*>(W + o_offsets);
      const int g = std::min<int>(pp.nchunks, ctx->sms * 4);
      tm.begin(3);
      GBA_CUDA_TRY(ctx, gba_launch_part_hist(pp, g, s));
      tm.end();
      tm.begin(3);
      GBA_CUDA_TRY(ctx, gba_launch_scan_excl(pp.counts, reinterpret_cast<unsigned long long*>(W + o_offsets), entries,
                                             reinterpret_cast<unsigned long long*>(W + o_status), d_tile_ctr, d_flags,
                                             s));
      tm.end();
      tm.begin(3);
      GBA_CUDA_TRY(ctx, gba_launch_part_scatter(pp, std::min<int>(pp.nchunks, ctx->sms * 2), T, s));
      tm.end();
      GBA_CUDA_TRY(ctx, gba_launch_seg_begins(pp.offsets, reinterpret_cast<const long long*>(W + o_cbase),
                                              reinterpret_cast<const int*>(W + o_snch), nseg_in, bits, n, d_seg, s));
      launches += 4;
      shift += bits;
      in = outq;
      if (pi + 1 < passes.size()) {
        // the next pass is planned on the host from this pass's segment bounds
        std::vector<long long> nb(size_t(nseg_in) * (size_t(1) << bits) + 1);
        GBA_CUDA_TRY(ctx, cudaMemcpyAsync(nb.data(), d_seg, 8 * nb.size(), cudaMemcpyDeviceToHost, s));
        GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
        seg_in.swap(nb);
      }
    }

    // plan the final work items from the partition bounds
    std::vector<long long> sb(size_t(nseg_final) + 1);
    GBA_CUDA_TRY(ctx, cudaMemcpyAsync(sb.data(), d_seg, 8 * sb.size(), cudaMemcpyDeviceToHost, s));
    GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    std::vector<PartWork> work;
    int64_t nsplit = 0;
    for (int64_t sg = 0; sg < nseg_final;) {
      const int64_t rows = sb[sg + 1] - sb[sg];
      if (rows > 2 * Lp) {
        ++nsplit;
        for (int64_t r = sb[sg]; r < sb[sg + 1]; r += Lp)
          work.push_back(PartWork{int(sg), int(sg) + 1, 1, 0, r, std::min<int64_t>(sb[sg + 1], r + Lp)});
        ++sg;
        continue;
      }
      int64_t e = sg + 1;
      while (e < nseg_final && sb[e + 1] - sb[sg] <= Lp && sb[e + 1] - sb[e] <= 2 * Lp) ++e;
      work.push_back(PartWork{int(sg), int(e), 0, 0, sb[sg], sb[e]});
      sg = e;
    }
    std::stable_sort(work.begin(), work.end(), [](const PartWork& x, const PartWork& y) {
      return x.row_end - x.row_begin > y.row_end - y.row_begin;
    });
    GBA_CUDA_TRY(ctx, cudaMemcpyAsync(W + o_work, work.data(), sizeof(PartWork) * work.size(),
                                      cudaMemcpyHostToDevice, s));

    // final aggregation over the 2^B partitions, then the fallback table
    GTable fb;
    fb.base = reinterpret_cast<unsigned long long*>(W + o_fb);
    fb.cap = fb_cap + uint64_t(nsplit) * uint64_t(S) * 2;
    fb.probe_cap = 256;
    GBA_CUDA_TRY(ctx, gba_launch_table_init(fb, q, ctx->sms * 4, s));
    PartAgg pa;
    pa.rows = in;
    pa.seg_begin = d_seg;
    pa.nsegs = int(nseg_final);
    pa.work = reinterpret_cast<const PartWork*>(W + o_work);
    pa.nwork = int(work.size());
    pa.seg_ctr = d_seg_ctr;
    pa.S = S;
    pa.sprobe = p.smem_probe_cap > 0 ? std::max(p.smem_probe_cap, 64) : 64;
    pa.coalesce = p.coalesce;
    pa.fallback = fb;
    pa.flags = d_flags;
    pa.out.keys = out->keys;
    for (int a = 0; a < GBA_MAX_AGGS; ++a) pa.out.accs[a] = static_cast<unsigned long long*>(out->aggs[a]);
    pa.out.capacity = out->capacity;
    pa.out.count = d_count;
    tm.begin(1);
    GBA_CUDA_TRY(ctx, gba_launch_part_agg(pa, std::min<int>(pa.nwork, ctx->sms), s));
    tm.end();
    ctx->stats.main_rows += n;
    ctx->stats.main_bytes += n * int64_t(rb);
    tm.begin(2);
    GBA_CUDA_TRY(ctx, gba_launch_compact(
                          fb, q, pa.out, int(std::max<uint64_t>(1, std::min<uint64_t>(ctx->sms * 8, fb.cap / 256))), s));
    tm.end();
    launches += 3;
    GBA_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_small, ctx->d_small, 16, cudaMemcpyDeviceToHost, s));
    GBA_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    tm.collect();
    ctx->stats.kernel_launches += launches;
    const unsigned flags = *reinterpret_cast<unsigned*>(ctx->h_small);
    const unsigned long long count = *reinterpret_cast<unsigned long long*>(ctx->h_small + 8);
    if (flags & GBA_FLAG_WAIT_TIMEOUT) {
      ctx->err = "a bounded scan wait timed out";
      return GBA_ERR_TIMEOUT;
    }
    if (flags & GBA_FLAG_TABLE_OVERFLOW) {
      if (attempt >= k.max_regrow || B >= 20) {
        ctx->err = "partition fallback table overflow after " + std::to_string(attempt) + " retries";
        return GBA_ERR_TABLE_OVERFLOW;
      }
      ctx->stats.regrows++;
      B = std::min(20, B + 2);
      groups *= 4;
      continue;
    }
    ctx->stats.preagg = 0;
    ctx->stats.table_slots = int64_t(S);
    *n_groups = int64_t(count);
    ctx->stats.n_groups = int64_t(count);
    if (int64_t(count) > out->capacity) {
      ctx->err = "output capacity " + std::to_string(out->capacity) + " < " + std::to_string(count) + " groups";
      return GBA_ERR_OUTPUT_CAPACITY;
    }
    return GBA_OK;
  }
}
