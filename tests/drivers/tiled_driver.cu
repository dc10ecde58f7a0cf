// A caller of the drop-in C++ API, written the way the reference's own driver
// calls the reference (test/test.cu:134-161): groupby_agg_partition<u32,u32>
// over pinned host columns, then groupby_agg_intra_partition with
// min_load_num / max_load_num = 3/5 and 4/5 of Capacity (test/test.cu:104-106).
// It only includes include/tiled_groupby_agg_partition.hpp and links libgba.so.
//
// Test infrastructure: reads  in.bin = [n (i64)][n u32 keys][n u32 values]  and
// writes what the API returned in the same format as the reference's fixture
// driver, so tests/test_gpu_dropin.py compares both against the golden files:
//   <out>.json  phase-1 partition sizes and pair digests, merged layout,
//               whether every phase-1 segment lies at the front of its own tile
//               in the caller's buffers, timings
//   <out>.bin   per merged partition i: par_result_kv_num[i] (u64), then that
//               many u32 keys and u32 sums
// An optional 7th argument R runs both phases R times on the same input (the
// pinned buffers are refilled from a copy before each run, outside the timed
// region, since phase 1 overwrites them) and records every run's times; the
// outputs are those of the last run.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <utility>
#include <vector>

#include "tiled_groupby_agg_partition.hpp"

static uint64_t mix64(uint64_t z) {
  z ^= z >> 31;
  z *= 0x7fb5d329728ea185ull;
  z ^= z >> 27;
  z *= 0x81dadef4bc2dd44dull;
  z ^= z >> 33;
  return z;
}

int main(int argc, char** argv) {
  if (argc < 7) {
    std::fprintf(stderr, "usage: %s in.bin out_prefix tile_len P nstreams capacity\n", argv[0]);
    return 2;
  }
  const std::string in = argv[1], outp = argv[2];
  const size_t tile_len = std::strtoull(argv[3], nullptr, 10);
  const size_t P = std::strtoull(argv[4], nullptr, 10);
  const size_t nstreams = std::strtoull(argv[5], nullptr, 10);
  const size_t Capacity = std::strtoull(argv[6], nullptr, 10);
  const int repeat = argc > 7 ? std::max(1, std::atoi(argv[7])) : 1;
  FILE* f = std::fopen(in.c_str(), "rb");
  if (!f) return 3;
  int64_t n = 0;
  if (std::fread(&n, 8, 1, f) != 1) return 3;
  cudaSetDevice(0);
  key_type* keys = nullptr;
  val_type* vals = nullptr;
  cudaMallocHost(&keys, sizeof(key_type) * (n > 0 ? n : 1));
  cudaMallocHost(&vals, sizeof(val_type) * (n > 0 ? n : 1));
  std::vector<key_type> keys0(n);
  std::vector<val_type> vals0(n);
  if (std::fread(keys0.data(), 4, n, f) != size_t(n) || std::fread(vals0.data(), 4, n, f) != size_t(n)) return 3;
  std::fclose(f);
  cudaFree(nullptr);

  auto sec = [](auto a, auto z) { return std::chrono::duration<double>(z - a).count(); };
  std::vector<double> p1_all, p2_all;
  std::vector<par_result> par_result_vec;
  key_type* out_keys = nullptr;
  val_type* out_vals = nullptr;
  std::vector<size_t> par_kv_begin, par_result_kv_num;
  std::vector<uint32_t> p1_size(P);
  std::vector<uint64_t> p1_digest(P);
  bool in_place = true;
  const size_t tiles = tile_len ? (size_t(n) + tile_len - 1) / tile_len : 0;
  std::vector<uint64_t> tile_fill(tiles, 0);
  for (int rep = 0; rep < repeat; ++rep) {
  std::copy(keys0.begin(), keys0.end(), keys);
  std::copy(vals0.begin(), vals0.end(), vals);
  if (out_keys) cudaFreeHost(out_keys);
  if (out_vals) cudaFreeHost(out_vals);
  out_keys = nullptr;
  out_vals = nullptr;
  par_kv_begin.clear();
  par_result_kv_num.clear();
  par_result_vec.assign(P, par_result());
  in_place = true;
  std::fill(tile_fill.begin(), tile_fill.end(), 0);
  auto t0 = std::chrono::steady_clock::now();
  try {
    groupby_agg_partition<key_type, val_type>(keys, vals, size_t(n), tile_len, P, par_result_vec, nstreams);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "groupby_agg_partition: %s\n", e.what());
    return 5;
  }
  auto t1 = std::chrono::steady_clock::now();

  for (size_t p = 0; p < P; ++p) {
    const par_result& pr = par_result_vec[p];
    uint64_t h = 0;
    for (size_t s = 0; s < pr.key.size(); ++s) {
      // segment s of every partition comes from tile s, at the front of its range
      const int64_t off = pr.key[s] - keys;
      in_place = in_place && pr.key.size() == tiles && pr.val[s] - vals == off && off >= int64_t(s * tile_len) &&
                 off + int64_t(pr.end_indicator[s]) <= int64_t(std::min<size_t>(size_t(n), (s + 1) * tile_len));
      if (s < tiles) tile_fill[s] += pr.end_indicator[s];
      for (uint32_t j = 0; j < pr.end_indicator[s]; ++j) h += mix64(uint64_t(pr.key[s][j]) << 32 | pr.val[s][j]);
    }
    p1_size[p] = pr.size;
    p1_digest[p] = h;
  }

  auto t2 = std::chrono::steady_clock::now();
  try {
    groupby_agg_intra_partition(par_result_vec, out_keys, out_vals, Capacity, Capacity * 3 / 5, Capacity * 4 / 5,
                                nstreams, par_kv_begin, par_result_kv_num);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "groupby_agg_intra_partition: %s\n", e.what());
    return 6;
  }
  auto t3 = std::chrono::steady_clock::now();
  p1_all.push_back(sec(t0, t1));
  p2_all.push_back(sec(t2, t3));
  }

  FILE* b = std::fopen((outp + ".bin").c_str(), "wb");
  for (size_t i = 0; i < par_kv_begin.size(); ++i) {
    const uint64_t m = par_result_kv_num[i];
    std::fwrite(&m, 8, 1, b);
    std::fwrite(out_keys + par_kv_begin[i], 4, m, b);
    std::fwrite(out_vals + par_kv_begin[i], 4, m, b);
  }
  std::fclose(b);

  FILE* j = std::fopen((outp + ".json").c_str(), "w");
  std::fprintf(j, "{\"n\": %lld, \"tile_len\": %zu, \"P\": %zu, \"nstreams\": %zu, \"capacity\": %zu,\n",
               (long long)n, tile_len, P, nstreams, Capacity);
  std::fprintf(j, " \"phase1_s\": %.6f, \"phase2_s\": %.6f, \"segments_in_place\": %s,\n", p1_all.back(),
               p2_all.back(), in_place ? "true" : "false");
  std::fprintf(j, " \"phase1_s_all\": [");
  for (size_t r = 0; r < p1_all.size(); ++r) std::fprintf(j, "%s%.6f", r ? ", " : "", p1_all[r]);
  std::fprintf(j, "],\n \"phase2_s_all\": [");
  for (size_t r = 0; r < p2_all.size(); ++r) std::fprintf(j, "%s%.6f", r ? ", " : "", p2_all[r]);
  std::fprintf(j, "],\n");
  std::fprintf(j, " \"tile_groups\": [");
  for (size_t t = 0; t < tiles; ++t) std::fprintf(j, "%s%llu", t ? ", " : "", (unsigned long long)tile_fill[t]);
  std::fprintf(j, "],\n \"phase1_sizes\": [");
  for (size_t p = 0; p < P; ++p) std::fprintf(j, "%s%u", p ? ", " : "", p1_size[p]);
  std::fprintf(j, "],\n \"phase1_digests\": [");
  for (size_t p = 0; p < P; ++p) std::fprintf(j, "%s\"%016llx\"", p ? ", " : "", (unsigned long long)p1_digest[p]);
  std::fprintf(j, "],\n \"par_kv_begin\": [");
  for (size_t i = 0; i < par_kv_begin.size(); ++i) std::fprintf(j, "%s%zu", i ? ", " : "", par_kv_begin[i]);
  std::fprintf(j, "],\n \"par_result_kv_num\": [");
  for (size_t i = 0; i < par_result_kv_num.size(); ++i)
    std::fprintf(j, "%s%zu", i ? ", " : "", par_result_kv_num[i]);
  std::fprintf(j, "]}\n");
  std::fclose(j);
  cudaFreeHost(out_keys);
  cudaFreeHost(out_vals);
  cudaFreeHost(keys);
  cudaFreeHost(vals);
  return 0;
}
