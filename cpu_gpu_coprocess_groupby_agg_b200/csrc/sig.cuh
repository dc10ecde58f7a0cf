// Aggregate signatures: how each accumulator of a query is computed, known
// either at run time (from the QDesc) or at compile time.
//
// The aggregation kernels are instruction-bound (measured with ncu: ~220
// instructions per row in the first generic kernel, mostly per-accumulator
// op/type dispatch and column loops), so the query shapes that matter are
// compiled with their ops, source columns and column types as constants and
// every other query runs the generic instantiation.
#pragma once
#include <type_traits>

#include "gba_kernels.h"

// spec code of one accumulator: op | source column << 4 | column type << 8
constexpr int sig_code(int op, int col, int ctype) { return op | (col << 4) | (ctype << 8); }

// 4-byte words of one accumulator in a shared-memory slot (gba_acc_smem_words)
constexpr int sig_words(int op) { return op == ACC_CNT ? 1 : op == ACC_ADD_F ? 6 : 2; }

// run-time signature with NA accumulators
template <int NA_>
struct SigRT {
  static constexpr int NA = NA_;
  __device__ __forceinline__ static int op(const QDesc& q, int a) { return q.acc_op[a]; }
  __device__ __forceinline__ static int col(const QDesc& q, int a) { return q.acc_col[a]; }
  __device__ __forceinline__ static int ctype(const QDesc& q, int a) { return q.acc_ctype[a]; }
  __device__ __forceinline__ static int woff(const QDesc& q, int a) { return q.acc_woff[a]; }
  __device__ __forceinline__ static int nwords(const QDesc& q) { return q.nwords; }
  __device__ __forceinline__ static int ncols(const QDesc& q) { return q.ncols; }
  __device__ __forceinline__ static int coltype(const QDesc& q, int c) { return q.col_type[c]; }
};

// compile-time signature
template <int... S>
struct SigCT {
  static constexpr int NA = sizeof...(S);
  __host__ __device__ __forceinline__ static constexpr int code(int a) {
    constexpr int v[] = {S...};
    return v[a];
  }
  __host__ __device__ __forceinline__ static constexpr int op(const QDesc&, int a) { return code(a) & 15; }
  __host__ __device__ __forceinline__ static constexpr int col(const QDesc&, int a) { return (code(a) >> 4) & 15; }
  __host__ __device__ __forceinline__ static constexpr int ctype(const QDesc&, int a) { return code(a) >> 8; }
  __host__ __device__ __forceinline__ static constexpr int woff(const QDesc& q, int a) {
    int w = 0;
    for (int i = 0; i < a; ++i) w += sig_words(code(i) & 15);
    return w;
  }
  __host__ __device__ __forceinline__ static constexpr int nwords(const QDesc& q) { return woff(q, NA); }
  __host__ __device__ __forceinline__ static constexpr int ncols(const QDesc&) {
    int n = 0;
    for (int i = 0; i < NA; ++i)
      if ((code(i) & 15) != ACC_CNT && ((code(i) >> 4) & 15) + 1 > n) n = ((code(i) >> 4) & 15) + 1;
    return n;
  }
  __host__ __device__ __forceinline__ static constexpr int coltype(const QDesc&, int c) {
    for (int i = 0; i < NA; ++i)
      if ((code(i) & 15) != ACC_CNT && ((code(i) >> 4) & 15) == c) return code(i) >> 8;
    return GBA_I32;
  }
  // does a (compacted) query have exactly this signature?
  static bool matches(const QDesc& q) {
    if (q.naccs != NA || q.ncols != ncols(q)) return false;
    for (int a = 0; a < NA; ++a) {
      if (q.acc_op[a] != op(q, a)) return false;
      if (q.acc_op[a] != ACC_CNT && (q.acc_col[a] != col(q, a) || q.acc_ctype[a] != ctype(q, a))) return false;
    }
    for (int c = 0; c < q.ncols; ++c)
      if (q.col_type[c] != coltype(q, c)) return false;
    return true;
  }
};

// The compiled query shapes.
using SigCount = SigCT<sig_code(ACC_CNT, 0, GBA_I64)>;
using SigSumI32Count = SigCT<sig_code(ACC_ADD_I, 0, GBA_I32), sig_code(ACC_CNT, 0, GBA_I64)>;
using SigSumU32Count = SigCT<sig_code(ACC_ADD_I, 0, GBA_U32), sig_code(ACC_CNT, 0, GBA_I64)>;
using SigSumU32 = SigCT<sig_code(ACC_ADD_I, 0, GBA_U32)>;
using SigSumI64Count = SigCT<sig_code(ACC_ADD_I, 0, GBA_I64), sig_code(ACC_CNT, 0, GBA_I64)>;
using SigSumSumCount =
    SigCT<sig_code(ACC_ADD_I, 0, GBA_I64), sig_code(ACC_ADD_I, 1, GBA_I64), sig_code(ACC_CNT, 0, GBA_I64)>;
using SigSkewed = SigCT<sig_code(ACC_ADD_I, 0, GBA_I64), sig_code(ACC_CNT, 0, GBA_I64),
                        sig_code(ACC_MIN_I, 0, GBA_I64), sig_code(ACC_MAX_I, 0, GBA_I64),
                        sig_code(ACC_ADD_F, 1, GBA_F32)>;

// A distinct number for each signature type (queries of one number can share
// one batched launch; run-time signatures read their ops per query).
template <int NA>
constexpr int gba_sig_index(SigRT<NA>) {
  return 100 + NA;
}
template <typename S>
constexpr int gba_sig_index(S) {
  return std::is_same<S, SigSkewed>::value        ? 1
         : std::is_same<S, SigSumSumCount>::value ? 2
         : std::is_same<S, SigSumI64Count>::value ? 3
         : std::is_same<S, SigSumI32Count>::value ? 4
         : std::is_same<S, SigSumU32Count>::value ? 5
         : std::is_same<S, SigSumU32>::value      ? 6
         : std::is_same<S, SigCount>::value       ? 7
                                                  : 0;
}

// Calls f(std::bool_constant<K64>, Sig) for the query's signature.
template <typename F>
inline cudaError_t gba_dispatch_sig(const QDesc& q, F&& f) {
  const bool k64 = q.key64 != 0;
  auto run = [&](auto sig) -> cudaError_t {
    return k64 ? f(std::true_type{}, sig) : f(std::false_type{}, sig);
  };
  if (SigSkewed::matches(q)) return run(SigSkewed{});
  if (SigSumSumCount::matches(q)) return run(SigSumSumCount{});
  if (SigSumI64Count::matches(q)) return run(SigSumI64Count{});
  if (SigSumI32Count::matches(q)) return run(SigSumI32Count{});
  if (SigSumU32Count::matches(q)) return run(SigSumU32Count{});
  if (SigSumU32::matches(q)) return run(SigSumU32{});
  if (SigCount::matches(q)) return run(SigCount{});
  switch (q.naccs) {
    case 1: return run(SigRT<1>{});
    case 2: return run(SigRT<2>{});
    case 3: return run(SigRT<3>{});
    case 4: return run(SigRT<4>{});
    case 5: return run(SigRT<5>{});
    case 6: return run(SigRT<6>{});
    case 7: return run(SigRT<7>{});
    case 8: return run(SigRT<8>{});
  }
  return cudaErrorInvalidValue;
}
