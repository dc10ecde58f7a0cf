// Host-visible interface of the reference-layout partition kernels (k_refpart.cu).
#pragma once
#include "gba_kernels.h"

// Largest partition fan-out of the drop-in API (the shared histogram of
// k_rp_hist holds P 4-byte counters; the reference itself stops at 1024).
#define GBA_REFPART_MAX_P 16384

// Writes the n groups (keys, int64 sums) ordered by partition
// murmur3_32(key, 0) % P into out_keys / out_vals (sums narrowed to u32);
// offsets[P + 1] receives each partition's start and the total.  hist[P] and
// cursor[P] are scratch.  out_* must not alias keys / sums.
cudaError_t gba_launch_refpart(const unsigned* keys, const unsigned long long* sums, int64_t n, int P,
                               unsigned* out_keys, unsigned* out_vals, unsigned* hist, unsigned long long* offsets,
                               unsigned long long* cursor, int sms, cudaStream_t s);
