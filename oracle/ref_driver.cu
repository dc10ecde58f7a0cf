// Driver for the unmodified reference library (compiled into oracle/_ref).
// TEST INFRASTRUCTURE: it produces the golden outputs that pin the oracle.
//
// It calls the reference exactly as its own driver does (test/test.cu:134-161):
// groupby_agg_partition<u32,u32>(keys, vals, n, tile_len, P, par_result_vec,
// nstreams) then groupby_agg_intra_partition(par_result_vec, keys_out,
// vals_out, Capacity, min_load_num, max_load_num, nstreams, par_kv_begin,
// par_result_kv_num), with min/max_load_num = 3/5, 4/5 of Capacity
// (test/test.cu:104-106).  Unlike test.cu it reads its input from a file and
// writes what the reference returns:
//   <out>.json  phase-1 partition sizes and pair digests, merged layout, timings
//   <out>.bin   for every merged partition i: par_result_kv_num[i] (u64) then
//               that many u32 keys and u32 sums from its result range
// An optional 7th argument R runs both phases R times on the same input (the
// pinned buffers are refilled from a copy before each run, outside the timed
// region; the reference overwrites them in phase 1) and records every run's
// times; the outputs are those of the last run.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include <algorithm>
#include <cuda_runtime.h>

#include "group_then_partition.cuh"
#include "groupby_agg_intra_partition.cuh"

// Order-independent digest of a multiset of (key, value) pairs:
// sum over pairs of mix64(key << 32 | value), mod 2^64.
static uint64_t mix64(uint64_t z) {
  z ^= z >> 31;
  z *= 0x7fb5d329728ea185ull;
  z ^= z >> 27;
  z *= 0x81dadef4bc2dd44dull;
  z ^= z >> 33;
  return z;
}
static uint64_t digest_pairs(const std::vector<std::pair<uint32_t, uint32_t>>& v) {
  uint64_t h = 0;
  for (auto& kv : v) h += mix64(uint64_t(kv.first) << 32 | kv.second);
  return h;
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
  u_int32_t *keys, *vals;
  cudaMallocHost(&keys, sizeof(u_int32_t) * n);
  cudaMallocHost(&vals, sizeof(u_int32_t) * n);
  std::vector<u_int32_t> keys0(n), vals0(n);
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
  auto t0 = std::chrono::steady_clock::now();
  groupby_agg_partition<u_int32_t, u_int32_t>(keys, vals, n, tile_len, P, par_result_vec, nstreams);
  cudaDeviceSynchronize();
  auto t1 = std::chrono::steady_clock::now();

  // phase-1 result: per partition, the multiset of (key, per-tile sum) pairs
  for (size_t p = 0; p < P; ++p) {
    std::vector<std::pair<uint32_t, uint32_t>> pairs;
    auto& pr = par_result_vec[p];
    for (size_t s = 0; s < pr.key.size(); ++s)
      for (uint32_t j = 0; j < pr.end_indicator[s]; ++j) pairs.emplace_back(pr.key[s][j], pr.val[s][j]);
    p1_size[p] = pr.size;
    p1_digest[p] = digest_pairs(pairs);
  }

  auto t2 = std::chrono::steady_clock::now();
  groupby_agg_intra_partition(par_result_vec, out_keys, out_vals, Capacity, Capacity * 3 / 5, Capacity * 4 / 5,
                              nstreams, par_kv_begin, par_result_kv_num);
  cudaDeviceSynchronize();
  auto t3 = std::chrono::steady_clock::now();
  p1_all.push_back(sec(t0, t1));
  p2_all.push_back(sec(t2, t3));
  }

  FILE* b = std::fopen((outp + ".bin").c_str(), "wb");
  for (size_t i = 0; i < par_kv_begin.size(); ++i) {
    uint64_t m = par_result_kv_num[i];
    std::fwrite(&m, 8, 1, b);
    std::fwrite(out_keys + par_kv_begin[i], 4, m, b);
    std::fwrite(out_vals + par_kv_begin[i], 4, m, b);
  }
  std::fclose(b);

  FILE* j = std::fopen((outp + ".json").c_str(), "w");
  std::fprintf(j, "{\"n\": %lld, \"tile_len\": %zu, \"P\": %zu, \"nstreams\": %zu, \"capacity\": %zu,\n",
               (long long)n, tile_len, P, nstreams, Capacity);
  std::fprintf(j, " \"phase1_s\": %.6f, \"phase2_s\": %.6f,\n", p1_all.back(), p2_all.back());
  std::fprintf(j, " \"phase1_s_all\": [");
  for (size_t r = 0; r < p1_all.size(); ++r) std::fprintf(j, "%s%.6f", r ? ", " : "", p1_all[r]);
  std::fprintf(j, "],\n \"phase2_s_all\": [");
  for (size_t r = 0; r < p2_all.size(); ++r) std::fprintf(j, "%s%.6f", r ? ", " : "", p2_all[r]);
  std::fprintf(j, "],\n");
  std::fprintf(j, " \"phase1_sizes\": [");
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
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e));
    return 4;
  }
  return 0;
}
