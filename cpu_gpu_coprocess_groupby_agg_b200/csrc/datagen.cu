// Host and device front-ends of the seeded column generator (datagen.h).
#include <algorithm>
#include <thread>
#include <vector>

#include "datagen.h"
#include "gba_kernels.h"

namespace {

__host__ __device__ inline void store_row(const gba_gen_spec& sp, int64_t i, uint64_t key, const int64_t* iv,
                                          const float* fv, void* keys, void* const* cols) {
  if (sp.key_bits == 64) static_cast<uint64_t*>(keys)[i] = key;
  else static_cast<uint32_t*>(keys)[i] = uint32_t(key);
  for (int c = 0; c < sp.ncols && c < GBA_GEN_MAX_COLS; ++c) {
    switch (sp.col_kind[c]) {
      case GBA_GEN_UNIFORM_I64: static_cast<int64_t*>(cols[c])[i] = iv[c]; break;
      case GBA_GEN_NORMAL_F32: static_cast<float*>(cols[c])[i] = fv[c]; break;
      default: static_cast<int32_t*>(cols[c])[i] = int32_t(iv[c]);
    }
  }
}

struct DevCols {
  void* c[GBA_GEN_MAX_COLS];
};

__global__ void k_gen(gba_gen_spec sp, gba_zipf z, int64_t row0, int64_t n, void* keys, DevCols cols) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    uint64_t key;
    int64_t iv[GBA_GEN_MAX_COLS];
    float fv[GBA_GEN_MAX_COLS];
    gba_gen_row(&sp, &z, uint64_t(row0 + i), &key, iv, fv);
    store_row(sp, i, key, iv, fv, keys, cols.c);
  }
}

bool spec_ok(const gba_gen_spec* sp) {
  if (!sp || (sp->key_bits != 32 && sp->key_bits != 64) || sp->ndv < 1 || sp->ncols < 0 ||
      sp->ncols > GBA_GEN_MAX_COLS || sp->zipf_s < 0)
    return false;
  for (int c = 0; c < sp->ncols; ++c)
    if (sp->col_kind[c] != GBA_GEN_NORMAL_F32 && sp->col_kind[c] != GBA_GEN_ONES_I32 &&
        sp->col_hi[c] <= sp->col_lo[c])
      return false;
  return true;
}

}  // namespace

extern "C" gba_status gba_gen_host(const gba_gen_spec* sp, int64_t row0, int64_t n, void* keys, void* const* cols,
                                   int32_t nthreads) {
  if (!spec_ok(sp) || n < 0 || (n > 0 && !keys)) return GBA_ERR_INVALID_ARG;
  const gba_zipf z = gba_zipf_make(sp->ndv, sp->zipf_s > 0 ? sp->zipf_s : 1.0);
  const int T = std::max(1, std::min<int>(nthreads, 256));
  auto work = [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; ++i) {
      uint64_t key;
      int64_t iv[GBA_GEN_MAX_COLS];
      float fv[GBA_GEN_MAX_COLS];
      gba_gen_row(sp, &z, uint64_t(row0 + i), &key, iv, fv);
      store_row(*sp, i, key, iv, fv, keys, cols);
    }
  };
  if (T == 1 || n < 65536) {
    work(0, n);
  } else {
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) th.emplace_back(work, n * t / T, n * (t + 1) / T);
    for (auto& x : th) x.join();
  }
  return GBA_OK;
}

extern "C" gba_status gba_gen_device(const gba_gen_spec* sp, int64_t row0, int64_t n, void* keys, void* const* cols,
                                     void* stream) {
  if (!spec_ok(sp) || n < 0 || (n > 0 && !keys)) return GBA_ERR_INVALID_ARG;
  if (n == 0) return GBA_OK;
  const gba_zipf z = gba_zipf_make(sp->ndv, sp->zipf_s > 0 ? sp->zipf_s : 1.0);
  DevCols dc{};
  for (int c = 0; c < sp->ncols; ++c) dc.c[c] = cols[c];
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = int(std::min<int64_t>((n + 255) / 256, int64_t(sms) * 8));
  k_gen<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(*sp, z, row0, n, keys, dc);
  return cudaGetLastError() == cudaSuccess ? GBA_OK : GBA_ERR_CUDA;
}

extern "C" int64_t gba_abi_struct_size(int32_t which) {
  switch (which) {
    case 0: return int64_t(sizeof(gba_query));
    case 1: return int64_t(sizeof(gba_output));
    case 2: return int64_t(sizeof(gba_knobs));
    case 3: return int64_t(sizeof(gba_stats));
    case 4: return int64_t(sizeof(gba_gen_spec));
    case 5: return int64_t(sizeof(gba_server_config));
    case 6: return int64_t(sizeof(gba_request_info));
  }
  return -1;
}
