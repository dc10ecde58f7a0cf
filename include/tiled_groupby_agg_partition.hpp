// Drop-in C++ entry points with the signatures of the reference's
// tiled_groupby_agg_partition library (PneNPproof/cpu_gpu_coprocess_groupby_agg):
//
//   groupby_agg_partition<K, V>   tiled_groupby_agg_partition/include/lib_header.hpp:6-12,
//                                 group_then_partition.cuh:5-11 (instantiated for
//                                 u32 keys and values, group_then_partition.cu:531-538)
//   groupby_agg_intra_partition   groupby_agg_intra_partition.cuh:5-13
//   par_result                    par_result.cuh:11-82
//   key_type, val_type, empty_k   util.cuh:6-8
//
// A caller of the reference (test/test.cu:134-161) compiles unchanged against
// this header and links libgba.so.  Both functions run on the current CUDA
// device and are built on the C ABI of include/gba.h.
//
// Behaviour kept from the reference:
//  * Phase 1 cuts the host input into tiles of tile_len rows, reduces each
//    tile to its distinct keys with the u32 SUM of their values (wrapping mod
//    2^32), orders the tile's groups by partition murmur3_32(key, 0) % P and
//    writes them over the start of the tile's own range of the caller's
//    buffers.  par_result_vec[p] receives, for every tile, one segment
//    (pointer into the caller's buffers, length; empty segments included).
//  * Phase 2 merges small partitions with the reference's greedy min-heap
//    (groupby_agg_intra_partition.cu:13-48) up to min_load_num rows, replaces
//    par_result_vec by the merged list, allocates the two result arrays with
//    cudaMallocHost (the caller frees them with cudaFreeHost) and writes merged
//    partition i's groups at [par_kv_begin[i], par_kv_begin[i] +
//    par_result_kv_num[i]).
//
// Differences, all in the caller's favour:
//  * Errors throw std::runtime_error (std::invalid_argument for bad sizes)
//    instead of being ignored or ending the process with exit(2)
//    (groupby_agg_intra_partition.cu:235).
//  * Calls share no process-global state (the reference keeps global tile
//    counters, group_then_partition.cu:9-11), so separate calls may run
//    concurrently from different threads.
//  * The key 0xffffffff (empty_k) is an ordinary key.
//  * Capacity and max_load_num are accepted but not needed: the tables are
//    sized by the library and grow on overflow.  P may be up to 16384 (the
//    reference's shared histogram stops at 1024).
//  * Segments are pushed in tile order, so par_result_vec is deterministic.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <vector>

typedef uint32_t key_type;
typedef uint32_t val_type;
const key_type empty_k = 0xffffffff;

// One partition's phase-1 output: segments of (key, value) pairs that live in
// the caller's host buffers (pointers are not owned).
class par_result {
 public:
  std::vector<key_type*> key;
  std::vector<val_type*> val;
  std::vector<uint32_t> end_indicator;  // segment lengths
  uint32_t size = 0;                    // total pairs over all segments
  std::mutex par_lock;

  par_result() = default;
  par_result(const par_result& o) : key(o.key), val(o.val), end_indicator(o.end_indicator), size(o.size) {}
  par_result& operator=(const par_result& o) {
    if (this != &o) {
      key = o.key;
      val = o.val;
      end_indicator = o.end_indicator;
      size = o.size;
    }
    return *this;
  }

  // appends one segment (thread safe)
  void push(key_type* keys, val_type* vals, uint32_t n) {
    std::lock_guard<std::mutex> g(par_lock);
    key.push_back(keys);
    val.push_back(vals);
    end_indicator.push_back(n);
    size += n;
  }

  // appends every segment of o
  void merge(const par_result& o) {
    key.insert(key.end(), o.key.begin(), o.key.end());
    val.insert(val.end(), o.val.begin(), o.val.end());
    end_indicator.insert(end_indicator.end(), o.end_indicator.begin(), o.end_indicator.end());
    size += o.size;
  }

  // Moves the last n pairs (taken from the back segments first) into the
  // device arrays on `stream`, removing them from this list; a segment that
  // is only partly taken keeps its front part.
  void pop2device(key_type* device_keys, val_type* device_vals, uint32_t n, cudaStream_t stream) {
    while (n > 0 && !end_indicator.empty()) {
      const uint32_t len = end_indicator.back();
      const uint32_t take = len < n ? len : n;
      const uint32_t from = len - take;
      cudaMemcpyAsync(device_keys, key.back() + from, size_t(take) * sizeof(key_type), cudaMemcpyHostToDevice,
                      stream);
      cudaMemcpyAsync(device_vals, val.back() + from, size_t(take) * sizeof(val_type), cudaMemcpyHostToDevice,
                      stream);
      device_keys += take;
      device_vals += take;
      size -= take;
      n -= take;
      if (take == len) {
        key.pop_back();
        val.pop_back();
        end_indicator.pop_back();
      } else {
        end_indicator.back() = from;
      }
    }
  }
};

// Phase 1: see the file comment.  nstreams host workers, each with its own CUDA
// stream and library context, take tiles in turn.  Only <uint32_t, uint32_t> is
// provided, as in the reference.
template <typename K, typename V>
void groupby_agg_partition(K* host_keys_buffer, V* host_vals_buffer, size_t kv_buffer_len, size_t tile_len,
                           size_t P, std::vector<par_result>& par_result_vec, size_t nstreams);
template <>
void groupby_agg_partition<uint32_t, uint32_t>(uint32_t* host_keys_buffer, uint32_t* host_vals_buffer,
                                               size_t kv_buffer_len, size_t tile_len, size_t P,
                                               std::vector<par_result>& par_result_vec, size_t nstreams);

// Phase 2: see the file comment.
void groupby_agg_intra_partition(std::vector<par_result>& par_result_vec, key_type*& host_groupby_keys_result,
                                 val_type*& host_agg_vals_result, size_t Capacity, size_t min_load_num,
                                 size_t max_load_num, size_t nstreams, std::vector<size_t>& par_kv_begin,
                                 std::vector<size_t>& par_result_kv_num);
