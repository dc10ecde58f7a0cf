// Autotuner: picks knobs by timing the caller's own queries on the device.
//
// No counterpart in the reference, whose tile length, stream count and
// partition count are command-line constants (test/test.cu:94-98).
//
// Coordinate descent from the caller's knobs: each knob in turn is set to each
// of its candidate values with the others held at the best setting so far;
// a setting is timed with CUDA events on `stream` (one untimed run, then the
// mean of `reps` runs) and kept when it is faster.  Knobs searched:
//   one query (gba_groupby):   tile_rows (TMA tile length), blocks_per_sm,
//                              partition_bits (around the automatic choice),
//                              learned_load / load_factor (HBM table load)
//   a batch (gba_groupby_batch): use_tma (which streaming kernel),
//                              blocks_per_sm, block_threads (the bulk-copy
//                              kernel's CTA size), nstages, coalesce, table_slots
//                              (GROW sizing), learned_load / load_factor,
//                              item_rows, smem_probe_cap (buckets probed)
// The outputs are written by every trial; the last trial leaves a complete,
// correct result for the best knobs only if the caller reruns with them.
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "gba_context.h"

namespace {

struct Axis {
  const char* name;
  std::vector<double> values;  // NaN = the knob's automatic setting
  std::function<void(gba_knobs&, double)> set;
};

}  // namespace

extern "C" gba_status gba_autotune(gba_context* ctx, int32_t nq, const gba_query* qs, const gba_output* outs,
                                   const gba_knobs* base, void* stream, int32_t reps, gba_knobs* best_out,
                                   double* best_ms) {
  if (!ctx || nq < 1 || !qs || !outs || !best_out) return GBA_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  gba_knobs best;
  if (base) best = *base;
  else gba_default_knobs(&best);
  best.timing = 0;
  reps = reps > 0 ? reps : 2;
  std::vector<int64_t> ng(nq);
  cudaEvent_t e0, e1;
  GBA_CUDA_TRY(ctx, cudaEventCreate(&e0));
  GBA_CUDA_TRY(ctx, cudaEventCreate(&e1));
  auto run = [&](const gba_knobs& k) -> gba_status {
    return nq == 1 ? gba_groupby(ctx, &qs[0], &outs[0], &k, stream, ng.data())
                   : gba_groupby_batch(ctx, nq, qs, outs, &k, stream, ng.data());
  };
  auto time_it = [&](const gba_knobs& k, double* ms) -> gba_status {
    gba_status st = run(k);  // untimed: workspace growth, graph capture
    if (st != GBA_OK) return st;
    GBA_CUDA_TRY(ctx, cudaEventRecord(e0, s));
    for (int r = 0; r < reps && st == GBA_OK; ++r) st = run(k);
    if (st != GBA_OK) return st;
    GBA_CUDA_TRY(ctx, cudaEventRecord(e1, s));
    GBA_CUDA_TRY(ctx, cudaEventSynchronize(e1));
    float t = 0.f;
    GBA_CUDA_TRY(ctx, cudaEventElapsedTime(&t, e0, e1));
    *ms = double(t) / reps;
    return GBA_OK;
  };

  const bool learned = best.sizing == GBA_SIZING_LEARNED;
  std::vector<Axis> axes;
  auto set_load = [learned](gba_knobs& k, double v) {
    if (learned) k.learned_load = std::isnan(v) ? 0.0 : v;
    else k.load_factor = std::isnan(v) ? 0.5 : v;
  };
  const double nan = std::nan("");
  if (nq == 1) {
    // the automatic fan-out of this query, to search around it
    double auto_ms = 0;
    gba_status st = time_it(best, &auto_ms);
    if (st != GBA_OK) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return st;
    }
    const int pb = ctx->stats.partition_bits;
    axes.push_back({"tile_rows", {nan, 2048, 4096, 8192}, [](gba_knobs& k, double v) {
                      k.tile_rows = std::isnan(v) ? 0 : int32_t(v);
                    }});
    axes.push_back({"blocks_per_sm", {nan, 2}, [](gba_knobs& k, double v) {
                      k.blocks_per_sm = std::isnan(v) ? 0 : int32_t(v);
                    }});
    if (pb > 0)
      axes.push_back({"partition_bits", {nan, double(pb - 1), double(pb + 1)}, [](gba_knobs& k, double v) {
                        k.partition_bits = std::isnan(v) ? 0 : int32_t(v);
                      }});
    axes.push_back({"load", {nan, 0.25, 0.5, 0.7}, set_load});
  } else {
    // the streaming kernel first (bulk-copy staging or register loads), then
    // the knobs of each: CTAs per SM for the register-loading kernel, ring
    // depth and warp combining of equal keys for the bulk-copy one
    axes.push_back({"use_tma", {nan, 0, 1}, [](gba_knobs& k, double v) {
                      k.use_tma = std::isnan(v) ? -1 : int32_t(v);
                    }});
    axes.push_back({"blocks_per_sm", {nan, 1, 2, 4}, [](gba_knobs& k, double v) {
                      k.blocks_per_sm = std::isnan(v) ? 0 : int32_t(v);
                    }});
    axes.push_back({"block_threads", {nan, 512}, [](gba_knobs& k, double v) {
                      k.block_threads = std::isnan(v) ? 0 : int32_t(v);
                    }});
    axes.push_back({"nstages", {nan, 2, 4}, [](gba_knobs& k, double v) {
                      k.nstages = std::isnan(v) ? 0 : int32_t(v);
                    }});
    axes.push_back({"coalesce", {nan, 1}, [](gba_knobs& k, double v) {
                      k.coalesce = std::isnan(v) ? -1 : int32_t(v);
                    }});
    if (best.sizing == GBA_SIZING_GROW)
      axes.push_back({"table_slots", {nan, double(1 << 14), double(1 << 18)}, [](gba_knobs& k, double v) {
                        k.table_slots = std::isnan(v) ? 0 : int64_t(v);
                      }});
    axes.push_back({"load", {nan, 0.25, 0.5}, set_load});
    axes.push_back({"item_rows", {nan, double(1 << 17), double(1 << 19)}, [](gba_knobs& k, double v) {
                      k.item_rows = std::isnan(v) ? 0 : int32_t(v);
                    }});
    axes.push_back({"smem_probe_cap", {nan, 1, 4}, [](gba_knobs& k, double v) {
                      k.smem_probe_cap = std::isnan(v) ? 0 : int32_t(v);
                    }});
  }

  double best_t = 0;
  gba_status st = time_it(best, &best_t);
  for (const Axis& ax : axes) {
    if (st != GBA_OK) break;
    gba_knobs keep = best;
    for (double v : ax.values) {
      gba_knobs k = keep;
      ax.set(k, v);
      if (std::memcmp(&k, &keep, sizeof(k)) == 0) continue;  // the setting already timed
      double t = 0;
      st = time_it(k, &t);
      if (st != GBA_OK) break;
      if (t < best_t) {
        best_t = t;
        best = k;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != GBA_OK) return st;
  *best_out = best;
  if (best_ms) *best_ms = best_t;
  return GBA_OK;
}
