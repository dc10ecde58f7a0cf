/* B200-native hash GROUP BY aggregation: the C ABI.
 *
 * Plain C types only (pointers, sizes, enums); `stream` arguments are
 * cudaStream_t passed as void*.  Every entry point returns a gba_status and
 * never exits the process.  A context is not shared between threads without
 * external locking; separate contexts run concurrently.
 *
 * Reference interfaces replaced (PneNPproof/cpu_gpu_coprocess_groupby_agg):
 *   - groupby_agg_partition<K,V>(host_keys, host_vals, kv_buffer_len, tile_len,
 *     P, par_result_vec, nstreams)          tiled_groupby_agg_partition/include/
 *                                           lib_header.hpp:6-12,
 *                                           group_then_partition.cuh:5-11
 *   - groupby_agg_intra_partition(par_result_vec, keys_out, vals_out, Capacity,
 *     min_load_num, max_load_num, nstreams, par_kv_begin, par_result_kv_num)
 *                                           groupby_agg_intra_partition.cuh:5-13
 * Together they compute an exact GROUP BY SUM of u32 values by u32 key.  The
 * C++ drop-ins with those exact signatures are declared in
 * tiled_groupby_agg_partition.hpp and are built on gba_groupby_partition_u32.
 */
#ifndef GBA_H
#define GBA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GBA_MAX_COLS 4
#define GBA_MAX_AGGS 8

typedef enum gba_status {
  GBA_OK = 0,
  GBA_ERR_INVALID_ARG = 1,
  GBA_ERR_CUDA = 2,
  GBA_ERR_OOM = 3,
  GBA_ERR_OUTPUT_CAPACITY = 4, /* more groups than gba_output.capacity; *n_groups holds the count */
  GBA_ERR_TABLE_OVERFLOW = 5,  /* table still overflowing after the regrow limit */
  GBA_ERR_TIMEOUT = 6,         /* a bounded device wait gave up */
  GBA_ERR_UNSUPPORTED = 7,
  GBA_ERR_BUDGET = 8           /* serving: request larger than the device-memory budget */
} gba_status;

/* Column and key types.  GBA_U32 is the reference's key_type/val_type
 * (u_int32_t, tiled_groupby_agg_partition/include/util.cuh:6-7).  Keys are
 * I32, U32 or I64; F32 and F64 are value columns only. */
typedef enum gba_type { GBA_I32 = 0, GBA_I64 = 1, GBA_F32 = 2, GBA_U32 = 3, GBA_F64 = 4 } gba_type;

/* Aggregates.  SUM/COUNT/MIN/MAX of integer columns accumulate in int64 and are
 * exact (SUM wraps mod 2^64); SUM of an F32 or F64 column accumulates in fp64
 * (F32 and F64 columns take SUM and AVG only).  AVG
 * (gba_groupby and gba_groupby_batch; the other entry points return
 * GBA_ERR_UNSUPPORTED) is the double SUM / COUNT of the group: the int64 sum
 * (fp64 for an F32 column) rounded to double, divided by the row count.  The reference computes SUM
 * only, in u32 (kernel.cu:48,152,334). */
/* GBA_COUNT counts rows (COUNT(*)); GBA_COUNT_VALID counts the rows whose
 * column value is present (COUNT(col); gba_groupby and gba_groupby_batch). */
typedef enum gba_op { GBA_SUM = 0, GBA_COUNT = 1, GBA_MIN = 2, GBA_MAX = 3, GBA_AVG = 4, GBA_COUNT_VALID = 5 } gba_op;

typedef struct gba_column {
  int32_t type;     /* gba_type */
  const void* data; /* n_rows elements, device (or host for *_host calls) */
  /* Nullable value columns (gba_groupby and gba_groupby_batch; elsewhere, and
   * on keys, GBA_ERR_UNSUPPORTED): a validity bitmap in device memory, bit
   * (i & 7) of byte i >> 3 set when row i's value is present (the Arrow
   * layout); null = every value present.  SUM, MIN, MAX and AVG skip absent
   * values; a group with none gets SUM 0, MIN the type's largest value, MAX
   * its smallest, AVG NaN, and validity 0 in gba_output.agg_valid. */
  const uint8_t* valid;
} gba_column;

typedef struct gba_agg {
  int32_t op;  /* gba_op */
  int32_t col; /* index into gba_query.cols; ignored for COUNT */
} gba_agg;

typedef struct gba_query {
  int64_t n_rows;
  gba_column key; /* GBA_I32, GBA_U32 or GBA_I64 */
  int32_t n_cols;
  gba_column cols[GBA_MAX_COLS];
  int32_t n_aggs;
  gba_agg aggs[GBA_MAX_AGGS];
  /* Composite key (gba_groupby and gba_groupby_batch; the other entry points
   * return GBA_ERR_UNSUPPORTED): when key2.data is set the query groups by the
   * pair (key, key2), both GBA_I32 or GBA_U32, and gba_output.keys2 receives
   * the second key of every group.  No reference counterpart: the reference
   * groups by one u32 key (tiled_groupby_agg_partition/include/util.cuh:6). */
  gba_column key2;
} gba_query;

/* Output columns: one row per distinct key, in no particular order.  aggs[a]
 * holds capacity 8-byte values: int64, or double for SUM of an F32 column and
 * for AVG. */
typedef struct gba_output {
  void* keys;
  void* aggs[GBA_MAX_AGGS];
  int64_t capacity;
  void* keys2; /* composite keys only: capacity second keys */
  /* optional (gba_groupby and gba_groupby_batch): one byte per group for
   * aggregate a, 1 when it saw a present value (always 1 for COUNT and for
   * columns without a validity bitmap) */
  uint8_t* agg_valid[GBA_MAX_AGGS];
} gba_output;

typedef enum gba_sizing {
  GBA_SIZING_PLAIN = 0,   /* fixed load factor on the row count, overflow -> regrow */
  GBA_SIZING_LEARNED = 1, /* MLP cardinality estimate, overflow -> regrow */
  GBA_SIZING_FIXED = 2,   /* table_slots as given, overflow -> regrow */
  GBA_SIZING_GROW = 3     /* estimator-free: the plain capacity, but at most table_slots (default 2^16)
                             to start with; a query whose table overflows reruns with 4x the slots */
} gba_sizing;

typedef enum gba_strategy {
  GBA_STRATEGY_AUTO = 0,
  GBA_STRATEGY_TABLE = 1,    /* shared-memory pre-aggregation + one HBM table */
  GBA_STRATEGY_PARTITION = 2 /* radix hash partition + per-partition shared-memory tables */
} gba_strategy;

/* Tuning knobs; 0 / -1 fields mean "choose automatically". */
typedef struct gba_knobs {
  int32_t sizing;         /* gba_sizing */
  int32_t strategy;       /* gba_strategy */
  double load_factor;     /* HBM table target load (default 0.5) */
  int64_t table_slots;    /* FIXED sizing */
  int32_t preagg;         /* -1 auto, 0 off, 1 on */
  int32_t smem_slots;     /* shared-memory table slots per CTA */
  int32_t partition_bits; /* radix fan-out 2^bits */
  int32_t blocks_per_sm;  /* single query: CTAs per SM of the pre-aggregation grid; batch: 1, 2, 3 or 4 (0 = 3)
                             for the register-loading kernel, and 1 or 2 CTAs of 512 threads for the
                             bulk-copy one (0: see block_threads) */
  int32_t block_threads;  /* single query: threads per CTA of its kernels.  Batch: the bulk-copy kernel's
                             CTAs, one of 1024 threads per SM (automatic: one shared table of twice the
                             slots for as many warps) or, with 512 or blocks_per_sm 1 or 2, CTAs of 512
                             threads */
  int32_t tile_rows;
  int32_t nstages;        /* TMA pipeline depth */
  int32_t use_tma;        /* -1 auto, 0 off, 1 on.  Single query: the TMA tile loader of the table
                             strategy.  Batch: which streaming kernel (1: the bulk-copy one, whose warps
                             stage rows with cp.async.bulk; 0: the register-loading one; auto: bulk copy
                             for queries whose predicted groups outgrow the other's shared table) */
  int32_t coalesce;       /* -1 auto, 0 off, 1 on: __match_any_sync pre-combining (batch: opt-in) */
  int32_t probe_cap;      /* HBM table probe cap (0 = auto) */
  int32_t smem_probe_cap; /* shared table probe cap (0 = auto) */
  int32_t max_regrow;     /* regrow attempts before GBA_ERR_TABLE_OVERFLOW */
  int32_t timing;         /* 1: time each kernel with CUDA events (gba_stats.kernel_ms) */
  int32_t use_graph;      /* batch: -1 auto (on), 0 off, 1 on: replay the launch sequence as a CUDA graph */
  int32_t item_rows;      /* batch: rows per work-queue item (0 = auto) */
  double learned_load;    /* learned sizing: HBM table load at the predicted group count (0 = auto: 0.35 for
                             one query, 0.25 in a batch) */
  int64_t learned_min_rows; /* single query, learned sizing: smaller queries are sized plainly
                               (0 = auto: while the plain table is <= 256 MB; -1 = always estimate) */
  int32_t sort_output;    /* gba_groupby, gba_groupby_batch, gba_groupby_host: 1 = groups in ascending key
                             order (signed for I32/I64 keys, unsigned for U32), sorted on the device;
                             0 (default) = hash-table order.  No reference counterpart: its partitions
                             hold their groups in table order (groupby_agg_intra_partition.cu:245-276). */
  int32_t cluster_ctas;   /* batch, learned sizing, bulk-copy kernel: the most CTAs of a thread-block
                             cluster whose shared tables together hold one query's table (distributed
                             shared memory), for queries whose predicted groups outgrow one CTA's table
                             (0 or 1 = off, the default; 2, 4, 8 or 16) */
  int32_t exchange;       /* batch: owner-exchange aggregation (-1 auto, 0 off, 1 every table query):
                             every SM owns a range of keys and holds their groups in its shared table;
                             rows reach their owner through exchange buffers that stay in L2.  Auto:
                             learned sizing, queries of at least 2^19 rows whose predicted groups
                             outgrow one CTA's table but fit the SMs' tables together, without a key
                             taking 1/32 of the sample */
} gba_knobs;

/* What the last call on a context did. */
typedef struct gba_stats {
  int32_t strategy;         /* gba_strategy actually run */
  int32_t preagg;           /* 1 if shared-memory pre-aggregation ran */
  int64_t table_slots;      /* HBM table capacity of the final attempt */
  int32_t partition_bits;
  int32_t regrows;          /* overflow re-runs */
  double predicted_groups;  /* estimator output (learned sizing), else -1 */
  int64_t n_groups;
  int32_t kernel_launches;  /* kernels launched by the call */
  /* with gba_knobs.timing: device time of the call's kernels, by role:
   * [0] table/partition setup, [1] the main aggregation kernel,
   * [2] final reduce / compaction, [3] everything else */
  double kernel_ms[4];
  /* input rows and their bytes (key + value columns) read by the main
   * aggregation kernels of the call, summed over launches: the algorithmic
   * bytes behind kernel_ms[1] */
  int64_t main_rows;
  int64_t main_bytes;
} gba_stats;

typedef struct gba_context gba_context;

/* sizeof() of the ABI structs, for binding generators: which = 0 gba_query,
 * 1 gba_output, 2 gba_knobs, 3 gba_stats, 4 gba_gen_spec, 5 gba_server_config,
 * 6 gba_request_info. */
int64_t gba_abi_struct_size(int32_t which);

void gba_default_knobs(gba_knobs* k);
const char* gba_status_string(gba_status s);

/* Creates a context bound to CUDA device `device`.  The context owns a device
 * workspace that grows on demand and is reused across calls. */
gba_status gba_create(gba_context** out, int32_t device);
gba_status gba_destroy(gba_context* ctx);
const char* gba_last_error(const gba_context* ctx);
gba_status gba_last_stats(const gba_context* ctx, gba_stats* out);

/* Exact GROUP BY over device-resident columns, enqueued on `stream`; returns
 * after the result is complete with *n_groups set (host pointer).  Replaces the
 * two reference phases (lib_header.hpp:6-12 + groupby_agg_intra_partition.cuh:5-13)
 * for data already in HBM. */
gba_status gba_groupby(gba_context* ctx, const gba_query* q, const gba_output* out, const gba_knobs* knobs,
                       void* stream, int64_t* n_groups);

/* The same over HOST columns and HOST output buffers: rows are streamed to the
 * device in chunks overlapped with aggregation (the reference's host-resident
 * "coprocess" tiling, group_then_partition.cu:353-418), the result is copied
 * back.  Pinned host memory gives full link speed. */
gba_status gba_groupby_host(gba_context* ctx, const gba_query* q, const gba_output* out,
                            const gba_knobs* knobs, void* stream, int64_t* n_groups);

/* Many independent queries (device columns) in one persistent launch over a
 * device work queue of (query, tile) items, replayed from a CUDA graph when the
 * same shapes repeat.  n_groups: host array of n_queries counts.  No
 * counterpart in the reference (its tile loop runs one query, one tile per
 * host thread at a time: group_then_partition.cu:332-424). */
gba_status gba_groupby_batch(gba_context* ctx, int32_t n_queries, const gba_query* qs, const gba_output* outs,
                             const gba_knobs* knobs, void* stream, int64_t* n_groups);

/* gba_groupby_batch over HOST columns (and validity bitmaps) and HOST output
 * buffers.  The queries are cut, in order, into parts of about a quarter of
 * the input bytes; all input copies are queued at once on a copy stream, part
 * p runs as one gba_groupby_batch call while part p + 1 crosses the link, and
 * part p's groups are copied back on a third stream while later parts run.
 * Pinned host memory gives full link speed.  Returns after every group is in
 * the host buffers; gba_last_stats describes the last part.  No reference
 * counterpart (its host-resident tiling runs one query:
 * group_then_partition.cu:353-418). */
gba_status gba_groupby_batch_host(gba_context* ctx, int32_t n_queries, const gba_query* qs, const gba_output* outs,
                                  const gba_knobs* knobs, void* stream, int64_t* n_groups);

/* gba_groupby without any device allocation: the table strategy (plain
 * sizing, 2 n + 64 slots) over a fixed 16 MiB scratch that is a static device
 * array of the library, not the context's workspace.  No counterpart in the
 * reference.
 *
 * For callers that must not allocate device memory per call: a process whose
 * device memory a pool allocator already reserved (a fresh cudaMalloc can fail
 * there), or a latency-sensitive thread whose device also runs other streams
 * (cudaFree synchronises the whole device).
 *
 * Limit: (2 n_rows + 65) * (1 + n_aggs) * 8 + 256 bytes must fit in 16 MiB
 * (about 349,000 rows with 2 aggregates); larger queries return
 * GBA_ERR_INVALID_ARG with the limit in gba_last_error and launch nothing.
 * The call synchronises `stream` to read its group count back, so no call can
 * be captured into a CUDA graph: on a capturing stream it returns
 * GBA_ERR_INVALID_ARG and launches nothing.  The first call on a device looks
 * up the scratch's address, which may load the library's device code (while
 * another thread captures a stream, that load may break its capture).  The
 * address is kept until the process exits, so do not call this entry point
 * after resetting the device (cudaDeviceReset).  Nullable columns, validity
 * outputs and composite keys return GBA_ERR_UNSUPPORTED.  Every
 * call clears the scratch's status and counter words and initialises its table
 * itself.  All calls on one device share the scratch: calls that overlap in
 * time on one device race; serialise them.  Synchronises `stream`. */
gba_status gba_groupby_noalloc(gba_context* ctx, const gba_query* q, const gba_output* out, void* stream,
                               int64_t* n_groups);

/* One tile of the reference's phase 1 on DEVICE columns: the exact GROUP BY
 * SUM of u32 values by u32 key (the sum wraps mod 2^32 like the reference's
 * u32 atomicAdd, kernel.cu:48,152), with the groups written to
 * out_keys / out_vals ordered by partition murmur3_32(key, seed 0) % P.
 * part_offsets (HOST, P + 1 entries) receives each partition's first group and
 * the group count.  1 <= P <= 16384.  out_keys / out_vals hold n_rows entries
 * and may be keys / vals themselves (the reference writes a tile's partitioned
 * groups over its input, group_then_partition.cu:413-417).  Replaces
 * compute_groupby_agg_result + compute_partition_result
 * (group_then_partition.cu:24-306).  Synchronises `stream`.  The C++ drop-ins
 * of include/tiled_groupby_agg_partition.hpp are built on it. */
gba_status gba_groupby_partition_u32(gba_context* ctx, const uint32_t* keys, const uint32_t* vals, int64_t n_rows,
                                     int32_t P, uint32_t* out_keys, uint32_t* out_vals, uint64_t* part_offsets,
                                     void* stream);

/* Sharded GROUP BY across ranks (one process per GPU; the exchange is
 * torch.distributed's all-to-all in the Python package): gba_avg_divide turns
 * each of n_cols device columns of n group SUMs (int64, or double where
 * sum_is_fp[i]) into the double SUM / counts[i] in place, for AVGs merged from
 * partial SUMs and COUNTs.  Synchronises `stream`.  No reference counterpart:
 * the reference runs on one device (test/test.cu:35). */
gba_status gba_avg_divide(gba_context* ctx, int32_t n_cols, void* const* sums, const int32_t* sum_is_fp,
                          const int64_t* counts, int64_t n, void* stream);

/* Autotuner: times the caller's own queries (device columns, as gba_groupby /
 * gba_groupby_batch take them) under candidate knobs by coordinate descent
 * from `base` and writes the fastest setting to *best (and its mean time per
 * call in ms to *best_ms).  One query: tile_rows, blocks_per_sm,
 * partition_bits and the HBM table load; a batch (n_queries > 1):
 * blocks_per_sm, the table load, item_rows and smem_probe_cap.  The load tuned is learned_load under
 * learned sizing, load_factor otherwise.  Every trial writes the outputs; rerun
 * with *best for the result.  No counterpart in the reference (its tile
 * length and partition count are constants, test/test.cu:94-98). */
gba_status gba_autotune(gba_context* ctx, int32_t n_queries, const gba_query* qs, const gba_output* outs,
                        const gba_knobs* base, void* stream, int32_t reps, gba_knobs* best, double* best_ms);

/* ---- serving: continuous batching under a device-memory budget ----------
 * No counterpart in the reference (one query per call).  A server runs `lanes`
 * host workers, each with its own CUDA stream and context, so their work
 * overlaps on the device and each keeps its tables and workspace resident
 * between requests (lanes run without CUDA graphs: knobs.use_graph is
 * ignored; knobs.blocks_per_sm defaults to 2 so that two lanes' batch kernels
 * fit on the GPU together).  Submitted requests (device columns in, device output
 * columns out, as gba_groupby) queue in arrival order; a free lane takes the
 * head of the queue and, when it is small (n_rows <= batch_rows), every
 * following small request (up to max_batch) that still fits the budget, and
 * runs them as one gba_groupby_batch call; a larger request runs alone.
 * Admission: the estimated device bytes of the running requests never exceed
 * memory_budget; a request that alone exceeds it is refused at submit with
 * GBA_ERR_BUDGET.  The caller keeps a request's columns and output buffers
 * alive until it is collected (gba_server_wait / gba_server_next_done). */
typedef struct gba_server gba_server;

typedef struct gba_server_config {
  int32_t device;
  int32_t lanes;         /* concurrent lanes (default 4, at most 64) */
  int64_t memory_budget; /* bytes (default 120 GiB) */
  int32_t max_batch;     /* requests per batch call (default 64) */
  int64_t batch_rows;    /* larger requests run alone (default 2^24) */
  gba_knobs knobs;       /* knobs of every call (sizing, strategy, ...) */
} gba_server_config;

typedef struct gba_request_info {
  int32_t status; /* gba_status of the request */
  int32_t lane;
  int32_t batch_size; /* requests in the call it ran in */
  int64_t n_groups;
  double queue_ms;   /* submit -> taken by a lane */
  double service_ms; /* taken -> result complete */
  double latency_ms; /* submit -> result complete */
} gba_request_info;

void gba_server_default_config(gba_server_config* c);
gba_status gba_server_create(gba_server** out, const gba_server_config* cfg);
/* Loads estimator weights into every lane (learned sizing); only while idle. */
gba_status gba_server_estimator_load(gba_server* sv, const float* params);
gba_status gba_server_submit(gba_server* sv, const gba_query* q, const gba_output* out, int64_t* ticket);
/* Waits up to timeout_s for one request; GBA_ERR_TIMEOUT if it is not done. */
gba_status gba_server_wait(gba_server* sv, int64_t ticket, double timeout_s, gba_request_info* info);
/* Waits up to timeout_s for any finished request and collects it. */
gba_status gba_server_next_done(gba_server* sv, double timeout_s, int64_t* ticket, gba_request_info* info);
gba_status gba_server_pending(gba_server* sv, int64_t* queued, int64_t* running, int64_t* inflight_bytes);
/* Where the server's time went so far (any pointer may be null): lane calls
 * made, batch calls that failed and were rerun request by request, workspace
 * releases (a lane frees its workspace when the lanes together hold more than
 * the budget; cudaFree synchronises the device), queries rerun with a larger
 * table after an overflow, the longest lane call and the longest release in
 * milliseconds. */
gba_status gba_server_counters(gba_server* sv, int64_t* lane_calls, int64_t* batch_failures, int64_t* ws_releases,
                               int64_t* regrows, double* lane_ms_max, double* release_ms_max);
/* The latest failed request's lane and message, else the latest refused submit's. */
const char* gba_server_last_error(const gba_server* sv);
/* Finishes every submitted request, then stops the lanes and frees them. */
gba_status gba_server_destroy(gba_server* sv);

/* ---- learned cardinality estimator -------------------------------------- */
#define GBA_EST_FEATURES 32
#define GBA_EST_HIDDEN 64
#define GBA_EST_SAMPLE 1024

/* Features of a device key column: per tile of `tile_rows` rows, a strided
 * 1024-row sample; out[GBA_EST_FEATURES] (host) gets the pooled features. */
gba_status gba_estimator_features(gba_context* ctx, const gba_query* q, int64_t tile_rows, void* stream,
                                  float* out);
/* Loads MLP weights (host fp32 array laid out as gba_estimator_param_count()
 * values) into the context; learned sizing uses them. */
int64_t gba_estimator_param_count(void);
gba_status gba_estimator_load(gba_context* ctx, const float* params);
gba_status gba_estimator_get(gba_context* ctx, float* params);
/* Predicts log2(groups) for n feature rows (host arrays). */
gba_status gba_estimator_predict(gba_context* ctx, int32_t n, const float* feats, float* out_log2_groups);
/* Trains on the GPU with the library's own forward/backward/Adam kernels:
 * feats[n][GBA_EST_FEATURES], target log2(groups)[n]; returns the final mean
 * squared error. */
gba_status gba_estimator_train(gba_context* ctx, int32_t n, const float* feats, const float* target,
                               int32_t epochs, int32_t batch, float lr, uint64_t seed, float* final_loss);
/* One forward+backward pass on the GPU for a batch (gradient check):
 * grads receives gba_estimator_param_count() values, *loss the MSE. */
gba_status gba_estimator_grad(gba_context* ctx, int32_t n, const float* feats, const float* target,
                              float* grads, float* loss);

/* ---- seeded synthetic data ---------------------------------------------- */
/* Host generator (any thread count); see csrc/datagen.h for the spec. */
struct gba_gen_spec;
gba_status gba_gen_host(const struct gba_gen_spec* spec, int64_t row0, int64_t n, void* keys, void* const* cols,
                        int32_t nthreads);
/* Device generator (same rows as the host generator up to libm rounding in the
 * Zipf / normal draws). */
gba_status gba_gen_device(const struct gba_gen_spec* spec, int64_t row0, int64_t n, void* keys, void* const* cols,
                          void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GBA_H */
