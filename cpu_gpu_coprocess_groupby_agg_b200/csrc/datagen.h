// Seeded synthetic column generator shared by the host library, the device
// generator kernel and the bench.  It replaces the reference's test-data
// generator (test/include/data_generator.hpp:7-105), which draws keys with
// std::rand and samples Zipf through a sampler that only accepts 0 < s < 1
// (test/include/zipfian_int_distribution.h:85,92); the workloads here need
// s = 1.0 and s up to 1.5, so the Zipf draw is Hoermann & Derflinger's
// rejection-inversion method (ACM TOMACS 6(3), 1996) written from the paper.
//
// Every row r draws from its own PCG32 stream (state seeded from the spec seed,
// increment 2r+1), so any slice of rows can be produced independently and in
// parallel, on the host or on the device, with the same integer results.
#pragma once
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define GBA_HD __host__ __device__ __forceinline__
#else
#define GBA_HD static inline
#endif

// Value-column kinds.
enum { GBA_GEN_UNIFORM_I32 = 0, GBA_GEN_UNIFORM_I64 = 1, GBA_GEN_NORMAL_F32 = 2, GBA_GEN_ONES_I32 = 3 };

#define GBA_GEN_MAX_COLS 4

typedef struct gba_gen_spec {
  uint64_t seed;
  int key_bits;          // 32 or 64
  uint64_t ndv;          // size of the key domain (distinct ids drawn from)
  double zipf_s;         // 0 = uniform over the domain
  int permute_ids;       // 1: key = bijective mix of the id; 0: key = id
  int avoid_all_ones;    // 1: never emit 0xffffffff (the reference's empty key)
  int ncols;
  int col_kind[GBA_GEN_MAX_COLS];
  int64_t col_lo[GBA_GEN_MAX_COLS];  // uniform: [lo, hi)
  int64_t col_hi[GBA_GEN_MAX_COLS];
} gba_gen_spec;

typedef struct gba_pcg32 {
  uint64_t state, inc;
} gba_pcg32;

GBA_HD uint32_t gba_pcg32_next(gba_pcg32* g) {
  uint64_t old = g->state;
  g->state = old * 6364136223846793005ULL + g->inc;
  uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
  uint32_t rot = (uint32_t)(old >> 59u);
  return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
}

GBA_HD gba_pcg32 gba_pcg32_seed(uint64_t seed, uint64_t stream) {
  gba_pcg32 g;
  g.state = 0;
  g.inc = (stream << 1u) | 1u;
  gba_pcg32_next(&g);
  g.state += seed;
  gba_pcg32_next(&g);
  return g;
}

GBA_HD uint64_t gba_pcg64_draw(gba_pcg32* g) {
  uint64_t hi = gba_pcg32_next(g);
  return (hi << 32) | gba_pcg32_next(g);
}

// uniform double in (0, 1): 53 random bits, never 0
GBA_HD double gba_unit_open(gba_pcg32* g) {
  uint64_t b = gba_pcg64_draw(g) >> 11;
  return ((double)b + 0.5) * (1.0 / 9007199254740992.0);
}

// uniform integer in [0, range) by 64x64->128 multiply (range < 2^63)
GBA_HD uint64_t gba_below(gba_pcg32* g, uint64_t range) {
  uint64_t x = gba_pcg64_draw(g);
#if defined(__CUDA_ARCH__)
  return __umul64hi(x, range);
#else
  return (uint64_t)(((unsigned __int128)x * range) >> 64);
#endif
}

// Bijective 64-bit and 32-bit finalisers used to turn dense ids into keys that
// look random ("randomly permuted ids").  Both are invertible (xor-shift and
// multiplication by an odd constant), so distinct ids stay distinct.
GBA_HD uint64_t gba_mix64(uint64_t z) {
  z ^= z >> 31;
  z *= 0x7fb5d329728ea185ULL;
  z ^= z >> 27;
  z *= 0x81dadef4bc2dd44dULL;
  z ^= z >> 33;
  return z;
}
GBA_HD uint32_t gba_mix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x7feb352dU;
  h ^= h >> 15;
  h *= 0x846ca68bU;
  h ^= h >> 16;
  return h;
}

// ---- Zipf over {1..N}, P(k) ~ k^-s, rejection-inversion ----------------------
// H(x) = integral of x^-s = ((x^(1-s)) - 1) / (1-s), written with
// expm1/log1p helpers so that s = 1 (H = log x) is handled without a branch.
GBA_HD double gba_zipf_helper_expm1_over(double x) {  // (e^x - 1)/x
  return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + x * 0.5 * (1.0 + x / 3.0 * (1.0 + 0.25 * x));
}
GBA_HD double gba_zipf_helper_log1p_over(double x) {  // log(1+x)/x
  return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * (0.5 - x * (1.0 / 3.0 - 0.25 * x));
}
GBA_HD double gba_zipf_H(double x, double s) {
  double lx = log(x);
  return gba_zipf_helper_expm1_over((1.0 - s) * lx) * lx;
}
GBA_HD double gba_zipf_Hinv(double u, double s) {
  double t = u * (1.0 - s);
  if (t < -1.0) t = -1.0;  // guards rounding at the domain edge
  return exp(gba_zipf_helper_log1p_over(t) * u);
}
GBA_HD double gba_zipf_h(double x, double s) { return exp(-s * log(x)); }

typedef struct gba_zipf {
  double s, n, hx1, hn, sq;
} gba_zipf;

GBA_HD gba_zipf gba_zipf_make(uint64_t n, double s) {
  gba_zipf z;
  z.s = s;
  z.n = (double)n;
  z.hx1 = gba_zipf_H(1.5, s) - 1.0;
  z.hn = gba_zipf_H(z.n + 0.5, s);
  z.sq = 2.0 - gba_zipf_Hinv(gba_zipf_H(2.5, s) - gba_zipf_h(2.0, s), s);
  return z;
}

// returns a rank in [1, n]
GBA_HD uint64_t gba_zipf_draw(const gba_zipf* z, gba_pcg32* g) {
  for (int it = 0; it < 64; ++it) {
    double u = z->hn + gba_unit_open(g) * (z->hx1 - z->hn);
    double x = gba_zipf_Hinv(u, z->s);
    double kd = floor(x + 0.5);
    if (kd < 1.0) kd = 1.0;
    if (kd > z->n) kd = z->n;
    if (kd - x <= z->sq || u >= gba_zipf_H(kd + 0.5, z->s) - gba_zipf_h(kd, z->s)) return (uint64_t)kd;
  }
  return 1;  // acceptance probability per round is > 0.5; 64 straight rejections do not occur
}

// ---- one row --------------------------------------------------------------------
// Key id -> key bits (as uint64; the low 32 bits are the key for 32-bit keys).
GBA_HD uint64_t gba_gen_key_of_id(const gba_gen_spec* sp, uint64_t id) {
  if (sp->key_bits == 64) return sp->permute_ids ? gba_mix64(id ^ (sp->seed * 0x9e3779b97f4a7c15ULL)) : id;
  uint32_t salt = (uint32_t)(sp->seed * 0x9e3779b9u);
  uint32_t k = sp->permute_ids ? gba_mix32((uint32_t)id ^ salt) : (uint32_t)id;
  if (sp->avoid_all_ones && k == 0xffffffffu)
    // the image of an id outside [0, ndv) is unused by every drawn id
    k = sp->permute_ids ? gba_mix32((uint32_t)sp->ndv ^ salt) : (uint32_t)sp->ndv;
  return k;
}

// Fills row r.  Stream layout per row: key draw(s) first, then one draw group
// per value column, in column order.
GBA_HD void gba_gen_row(const gba_gen_spec* sp, const gba_zipf* z, uint64_t r, uint64_t* key,
                        int64_t* ival, float* fval) {
  gba_pcg32 g = gba_pcg32_seed(sp->seed, r);
  uint64_t id = (sp->zipf_s > 0.0) ? gba_zipf_draw(z, &g) - 1 : gba_below(&g, sp->ndv);
  *key = gba_gen_key_of_id(sp, id);
  for (int c = 0; c < sp->ncols && c < GBA_GEN_MAX_COLS; ++c) {
    switch (sp->col_kind[c]) {
      case GBA_GEN_NORMAL_F32: {
        double u1 = gba_unit_open(&g), u2 = gba_unit_open(&g);
        fval[c] = (float)(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
        ival[c] = 0;
        break;
      }
      case GBA_GEN_ONES_I32:
        ival[c] = 1;
        fval[c] = 0.f;
        break;
      default: {
        uint64_t range = (uint64_t)(sp->col_hi[c] - sp->col_lo[c]);
        ival[c] = sp->col_lo[c] + (int64_t)gba_below(&g, range);
        fval[c] = 0.f;
      }
    }
  }
}
