// Stand-in for cuCollections' <cuco/detail/hash_functions/murmurhash3.cuh>,
// which the reference includes (tiled_groupby_agg_partition/src/kernel.cu:3) but
// does not vendor.  TEST INFRASTRUCTURE: used only to compile the unmodified
// reference into oracle/_ref.  MurmurHash3_x86_32 of the key's bytes, written
// from the published public-domain algorithm; oracle/oracle.cpp has the same
// function and tests/test_oracle.py pins both to independent known answers.
#pragma once
#include <cstdint>

namespace cuco {
namespace detail {

template <typename Key>
struct MurmurHash3_32 {
  __host__ __device__ constexpr MurmurHash3_32(uint32_t seed = 0) : seed_(seed) {}

  __host__ __device__ uint32_t operator()(Key const& key) const {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&key);
    constexpr int len = int(sizeof(Key));
    uint32_t h = seed_;
    for (int i = 0; i + 4 <= len; i += 4) {
      uint32_t k = uint32_t(p[i]) | uint32_t(p[i + 1]) << 8 | uint32_t(p[i + 2]) << 16 | uint32_t(p[i + 3]) << 24;
      k *= 0xcc9e2d51u;
      k = (k << 15) | (k >> 17);
      k *= 0x1b873593u;
      h ^= k;
      h = (h << 13) | (h >> 19);
      h = h * 5u + 0xe6546b64u;
    }
    uint32_t k = 0;
    const int tail = len & ~3;
    switch (len & 3) {
      case 3: k ^= uint32_t(p[tail + 2]) << 16; [[fallthrough]];
      case 2: k ^= uint32_t(p[tail + 1]) << 8; [[fallthrough]];
      case 1:
        k ^= p[tail];
        k *= 0xcc9e2d51u;
        k = (k << 15) | (k >> 17);
        k *= 0x1b873593u;
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

 private:
  uint32_t seed_;
};

}  // namespace detail
}  // namespace cuco
