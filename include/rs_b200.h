/*
 * rs_b200 — B200-native Reed-Solomon encode/reconstruct behind a C ABI.
 *
 * Drop-in boundary for the tape-reed-solomon (spool-labs/reed-solomon 0.2.2) coder
 * API. Each entry point below names the reference item it replaces (paths relative
 * to the reference crate root). All arithmetic runs in hand-written sm_100a CUDA
 * kernels; there is no CPU fallback: without a usable CUDA device every computing
 * call returns RS_ERR_NO_DEVICE.
 *
 * Conventions
 *  - Status 0 is success. 1..14 follow the reference `Error` enum in declaration
 *    order (src/errors.rs:7-20). Values >= 100 are device/runtime errors.
 *  - Host-pointer calls (no suffix) take host buffers like the reference's slices,
 *    copy them to the device, run the kernels and copy results back before they
 *    return. `_dev` calls take device pointers and a cudaStream_t (as void*), and
 *    return once the work is enqueued.
 *  - The caller owns every shard buffer; the library owns codec and decoder handles
 *    and the device tables they hold. Handles are safe to share between threads.
 *  - Shards of the GF((2^8)^2) coder use the split-plane wire: a shard of 2N bytes
 *    holds the N low bytes then the N high bytes (src/reedsolomon16.rs:4-7).
 */
#ifndef RS_B200_H
#define RS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- status codes: src/errors.rs:7-20 ---- */
enum rs_status {
  RS_OK = 0,
  RS_TOO_FEW_SHARDS = 1,
  RS_TOO_MANY_SHARDS = 2,
  RS_TOO_FEW_DATA_SHARDS = 3,
  RS_TOO_MANY_DATA_SHARDS = 4,
  RS_TOO_FEW_PARITY_SHARDS = 5,
  RS_TOO_MANY_PARITY_SHARDS = 6,
  RS_TOO_FEW_BUFFER_SHARDS = 7,
  RS_TOO_MANY_BUFFER_SHARDS = 8,
  RS_INCORRECT_SHARD_SIZE = 9,
  RS_TOO_FEW_SHARDS_PRESENT = 10,
  RS_EMPTY_SHARD = 11,
  RS_INVALID_SHARD_FLAGS = 12,
  RS_INVALID_INDEX = 13,
  RS_SINGULAR_MATRIX = 14,
  RS_ERR_CUDA = 100,          /* a CUDA runtime call failed */
  RS_ERR_ALLOC = 101,         /* host or device allocation failed */
  RS_ERR_INVALID_ARGUMENT = 102, /* null handle/pointer or unsupported option */
  RS_ERR_NO_DEVICE = 103,     /* no usable CUDA device */
  RS_ERR_TIMEOUT = 104,       /* a bounded device wait gave up */
  RS_ERR_LENGTH_MISMATCH = 105, /* gf8_mul_slice lengths differ (the reference panics) */
  RS_ERR_TOO_LARGE = 106       /* the request needs more than a fixed working area holds */
};

/* Message text for a status (src/errors.rs:24-41 for 1..14). Never NULL. */
const char *rs_strerror(int status);
/* ABI version, (major << 16) | minor. */
uint32_t rs_abi_version(void);

typedef struct rs8_codec rs8_t;
typedef struct rs8_decoder rs8_dec_t;
typedef struct rs16_codec rs16_t;
typedef struct rs16_decoder rs16_dec_t;

/* =========================== ReedSolomon (GF(2^8)) =========================== */

/* ReedSolomon::new, src/reedsolomon.rs:166-196. k = 0 -> TooFewDataShards,
 * m = 0 -> TooFewParityShards, k + m > 256 -> TooManyShards. Builds the systematic
 * generator on the current CUDA device and keeps its tables resident there. */
int rs8_new(size_t data_shards, size_t parity_shards, rs8_t **out);
/* impl Clone for ReedSolomon, src/reedsolomon.rs:725-739 (copies the plan cache). */
int rs8_clone(const rs8_t *codec, rs8_t **out);
void rs8_free(rs8_t *codec);
/* data_shard_count / parity_shard_count / total_shard_count, src/reedsolomon.rs:255-265 */
size_t rs8_data_shard_count(const rs8_t *codec);
size_t rs8_parity_shard_count(const rs8_t *codec);
size_t rs8_total_shard_count(const rs8_t *codec);
/* impl PartialEq for ReedSolomon, src/reedsolomon.rs:741-746: compares (k, m). */
int rs8_equal(const rs8_t *a, const rs8_t *b);
/* Generator rows k..n-1 (m x k bytes) as built on the device; row-major. */
int rs8_parity_matrix(const rs8_t *codec, uint8_t *out, size_t out_len);

/* ReedSolomon::encode, src/reedsolomon.rs:271-278. shards[0..k) data, [k..n) parity,
 * all `len` bytes. n != k+m -> TooFew/TooManyShards; len 0 -> EmptyShard. */
int rs8_encode(rs8_t *codec, uint8_t *const *shards, size_t n_shards, size_t len);
/* ReedSolomon::encode_sep, src/reedsolomon.rs:284-309. Like the reference it does
 * not reject len 0 (then it is a no-op). */
int rs8_encode_sep(rs8_t *codec, const uint8_t *const *data, size_t n_data,
                   uint8_t *const *parity, size_t n_parity, size_t len);
/* ReedSolomon::encode_rows_into, src/reedsolomon.rs:667-697: data is k rows of
 * row_len bytes back to back, parity m rows. Wrong sizes -> IncorrectShardSize;
 * row_len 0 is a no-op. (encode_rows, :652, is the facade asserting the same.) */
int rs8_encode_rows(rs8_t *codec, const uint8_t *data, size_t data_len, size_t row_len,
                    uint8_t *parity, size_t parity_len);
/* Many stripes of one shape from host memory (the batched form of encode_rows_into):
 * stripe s reads k rows of row_len bytes at data + s*data_stride and writes m rows at
 * parity + s*parity_stride. Copies to and from the device are pipelined with the
 * kernels over chunks of stripes on three streams; pinned host buffers copy at full
 * PCIe rate in both directions at once. Returns when the parity is in host memory. */
int rs8_encode_batch(rs8_t *codec, const uint8_t *data, size_t data_stride, uint8_t *parity,
                     size_t parity_stride, size_t n_stripes, size_t row_len);
/* ReedSolomon::verify, src/reedsolomon.rs:430-463: *ok = 1 iff every parity shard
 * matches the recomputed parity. */
int rs8_verify(rs8_t *codec, const uint8_t *const *shards, size_t n_shards, size_t len,
               int *ok);
/* ReedSolomon::reconstruct / reconstruct_data, src/reedsolomon.rs:470-477,615-641.
 * present[i] != 0 marks a valid shard; lens[i] is the length of buffer i (a present
 * shard's length; an absent buffer must already have the shard length, as for the
 * reference's `(T, bool)` shards). data_only leaves missing parity untouched. */
int rs8_reconstruct(rs8_t *codec, uint8_t *const *shards, const size_t *lens,
                    const uint8_t *present, size_t n_shards, int data_only);
/* ReedSolomon::reconstruct_rows, src/reedsolomon.rs:514-535. */
int rs8_reconstruct_rows(rs8_t *codec, uint8_t *rows, size_t rows_len, size_t row_len,
                         const uint8_t *present, size_t n_present);
/* ReedSolomon::prepare_decode, src/reedsolomon.rs:484-505 -> PreparedDecoder. */
int rs8_prepare_decode(rs8_t *codec, const uint8_t *present, size_t n_present,
                       rs8_dec_t **out);
/* PreparedDecoder::{reconstruct, reconstruct_data}, src/reedsolomon.rs:760-797:
 * a different presence pattern -> InvalidShardFlags. */
int rs8_dec_reconstruct(rs8_dec_t *dec, uint8_t *const *shards, const size_t *lens,
                        const uint8_t *present, size_t n_shards, int data_only);
int rs8_dec_clone(const rs8_dec_t *dec, rs8_dec_t **out);
void rs8_dec_free(rs8_dec_t *dec);
/* ReedSolomon::encode_route, src/reedsolomon.rs:239-253 (bench/test introspection):
 * "fft-bitsliced" ((K,K), K a power of two), "generator-bitsliced" ((7,13), (10,10),
 * (14,14), (18,6): the reference's other generated shapes; (20,12); the storage codes
 * (4,2), (6,3), (8,4), (10,4), (12,4), (16,4), (17,3): the generator compiled in) or
 * "matrix" for this shard length. Never NULL. */
const char *rs8_encode_route(const rs8_t *codec, size_t len);
/* Test/bench hook like the reference's encode_scalar/encode_forced
 * (src/reedsolomon.rs:365-424): route 0 = automatic, 1 = matrix, 2 = the shape's
 * compiled bitsliced kernel, FFT or generator (falls back to matrix where the shape has
 * none). */
int rs8_set_route(rs8_t *codec, int route);

/* ---- device-resident variants (device pointers, enqueued on `stream`) ---- */
int rs8_encode_dev(rs8_t *codec, uint8_t *const *d_shards, size_t n_shards, size_t len,
                   void *stream);
int rs8_encode_sep_dev(rs8_t *codec, const uint8_t *const *d_data, size_t n_data,
                       uint8_t *const *d_parity, size_t n_parity, size_t len, void *stream);
int rs8_encode_rows_dev(rs8_t *codec, const uint8_t *d_data, size_t row_len,
                        uint8_t *d_parity, void *stream);
/* Many stripes of one shape in one launch: stripe s reads k rows of row_len bytes at
 * d_data + s*data_stride and writes m rows at d_parity + s*parity_stride. */
int rs8_encode_batch_dev(rs8_t *codec, const uint8_t *d_data, size_t data_stride,
                         uint8_t *d_parity, size_t parity_stride, size_t n_stripes,
                         size_t row_len, void *stream);
/* Recomputes parity and compares on the device; waits for the result. */
int rs8_verify_dev(rs8_t *codec, const uint8_t *const *d_shards, size_t n_shards, size_t len,
                   int *ok, void *stream);
/* Reconstruct over device shard buffers (same checks as rs8_reconstruct). */
int rs8_reconstruct_dev(rs8_t *codec, uint8_t *const *d_shards, const size_t *lens,
                        const uint8_t *present, size_t n_shards, int data_only, void *stream);
/* Many stripes of one shape, each with its own erasure pattern, in one launch.
 * Stripe s is n contiguous rows of row_len bytes at d_rows + s*stripe_stride;
 * present is n_stripes x n flags (host memory). Decode matrices for all patterns
 * are built on the device. statuses (host, optional) gets a per-stripe status. */
int rs8_reconstruct_batch_dev(rs8_t *codec, uint8_t *d_rows, size_t stripe_stride,
                              size_t n_stripes, size_t row_len, const uint8_t *present,
                              int data_only, int *statuses, void *stream);

/* Batched reconstruct that allocates nothing. No counterpart in the reference.
 * For callers that cannot allocate device memory while they run: a latency-critical
 * path that must not stall on the allocator, a process whose memory budget was fixed
 * at start-up, or a host whose device allocator belongs to another framework. Same
 * arguments, checks and results as rs8_reconstruct_batch_dev, but all working memory
 * (survivor and target lists, decode rows, plan statuses) lives in one 8 MiB device
 * array inside this library, which every GPU that loads the library holds until the
 * process exits, and the host side stages through one fixed buffer: no cudaMalloc,
 * cudaFree or other allocating call is made. A call needing more than 8 MiB of working
 * memory (see rs8_reconstruct_batch_noalloc_limit) returns RS_ERR_TOO_LARGE; split the
 * batch. The first call on each device looks up the array's device address, which
 * (with CUDA's default lazy module loading) loads this entry point's device code and
 * reserves the 8 MiB array on that device then: make that first call at start-up,
 * while memory is still free, and before capturing any stream on that device; it
 * returns RS_ERR_CUDA if the device has no 8 MiB left. Later calls take no device
 * memory. The index lists travel through a host buffer that the next call
 * overwrites, so a call on a stream that is capturing returns RS_ERR_INVALID_ARGUMENT.
 * Missing parity rows are rebuilt on the matrix route (one pass over the k
 * survivors), never on the shape's compiled FFT or generator kernel: the bytes are the
 * same as rs8_reconstruct_batch_dev's, the speed lower on shapes with such a kernel.
 * Nothing in the array has to start at zero: each call writes every entry it reads
 * before reading it. Every call shares the one array and it keeps the last call's
 * contents: calls whose GPU work overlaps (other streams, or other host threads) race
 * on it, so run them one after another. */
int rs8_reconstruct_batch_noalloc(rs8_t *codec, uint8_t *d_rows, size_t stripe_stride,
                                  size_t n_stripes, size_t row_len, const uint8_t *present,
                                  int data_only, int *statuses, void *stream);
/* Bytes of that fixed working area a call of this shape and stripe count needs
 * (SIZE_MAX when the stripe count is beyond any working area). */
size_t rs8_reconstruct_batch_noalloc_limit(size_t data_shards, size_t parity_shards,
                                           size_t n_stripes);

/* ---- mixed batches: stripes of any GF(2^8) shapes, lengths and erasure patterns ----
 * No counterpart in the reference (it codes one stripe per call on one core). A batch
 * is validated and planned once: decode matrices for every reconstruct item are built
 * on the device in one launch per shape, the work is grouped by route (one compiled
 * bitsliced launch per FFT or generator shape, one ragged matrix launch for the rest;
 * missing parity of reconstructs on compiled shapes is regenerated by a compiled launch
 * that stores only the missing rows, after the data rows) and captured into a CUDA
 * graph; rs_batch_launch replays it. Each item's status is the reference error its
 * single-stripe call would return (0 = Ok); failed items are left out of the graph. */
enum rs_batch_op {
  RS_BATCH_ENCODE = 0,           /* rows [0,k) -> rows [k,n) */
  RS_BATCH_RECONSTRUCT = 1,      /* rebuild every absent row */
  RS_BATCH_RECONSTRUCT_DATA = 2  /* rebuild absent data rows only */
};
enum rs_batch_flags {
  RS_BATCH_MATRIX_ONLY = 1, /* the plain route for every item (comparison baseline) */
  RS_BATCH_NO_GRAPH = 2     /* launch kernels directly instead of through a graph */
};
typedef struct {
  rs8_t *codec;           /* the stripe's shape (k, m) */
  uint8_t *d_rows;        /* n = k+m rows of row_len bytes, row_stride apart (device) */
  size_t row_stride;
  size_t row_len;
  int op;                 /* enum rs_batch_op */
  const uint8_t *present; /* n flags (host memory), reconstruct ops only */
} rs_batch_item;
typedef struct rs_batch rs_batch_t;
int rs_batch_create(const rs_batch_item *items, size_t n_items, int flags, int *statuses,
                    rs_batch_t **out);
/* rs_batch_create with a launch configuration per encode item (configs[i], an index
 * into the tuner's configurations, rs_tuning_config; -1 = the library's automatic
 * choice): matrix configurations put the item on the ragged matrix launch, FFT and
 * generator configurations on the shape's compiled kernel with that launch shape (one
 * launch per shape and configuration); a configuration the item's shape has no kernel
 * for gives the item RS_ERR_INVALID_ARGUMENT. Reconstruct items ignore it. Results are
 * the same bytes whatever the configurations. */
int rs_batch_create_configured(const rs_batch_item *items, size_t n_items, int flags,
                               const int *configs, int *statuses, rs_batch_t **out);
typedef struct rs_mlp rs_mlp_t;
/* The cost model's choice for a batch: encode items of shapes with a compiled kernel
 * are grouped by shape and row alignment (each group is one launch); the model (an
 * rs_mlp_t with rs_tuning_features inputs and rs_tuning_config_count outputs, e.g. one
 * loaded with rs_mlp_load) predicts every item's log time per configuration from
 * (k, m, row bytes, erasures 0, stripes in its group, alignment), and each group gets
 * the applicable configuration with the least predicted total where that is predicted
 * at least 10% faster than the library's automatic choice (else -1, the automatic
 * choice). configs[i] = -1 for every other item. Pass the result to
 * rs_batch_create_configured. */
int rs_batch_choose(const rs_batch_item *items, size_t n_items, rs_mlp_t *model, int *configs);
/* Launch configurations the autotuner times and the cost model scores: index 0..count-1
 * -> route (0 matrix, 1 FFT, 2 generator kernel), p0 (matrix tile variant, or FFT
 * lane-group width 0 narrow / 1 wide), p1 (FFT launch shape, rs_set_fft_variant). */
int rs_tuning_config_count(void);
int rs_tuning_config(int index, int *route, int *p0, int *p1);
/* Inputs of the cost model: log2(k)/8, log2(m)/8, log2(row bytes)/20, erasures/m,
 * log2(stripes per launch)/8 (a launch group is scored as at most 512 stripes and at
 * most 64 MiB, the autotuner's range), 1 when rows are not 16-byte aligned. */
int rs_tuning_features(void);
/* Enqueues one replay of the batch on `stream`. */
int rs_batch_launch(rs_batch_t *batch, void *stream);
/* Kernel launches per replay, stripes on each route (a stripe with any matrix work
 * counts as a matrix item, one with compiled-kernel work only as an FFT item),
 * algorithmic bytes per replay ((k+m)*len per encode, (k+e)*len per reconstruct
 * rebuilding e rows). */
int rs_batch_stats(const rs_batch_t *batch, size_t *launches, size_t *fft_items,
                   size_t *matrix_items, uint64_t *bytes);
void rs_batch_free(rs_batch_t *batch);

/* ---- persistent work queue: one long-running launch fed while it runs ----
 * No counterpart in the reference. A session starts one persistent kernel (a captured
 * graph, replayed per session) and the host then pushes stripes (rs_batch_item: any
 * GF(2^8) shape, shard length and erasure pattern, validated as rs_batch_create does;
 * each item's status as its single-stripe call would return it) while it runs; every
 * stripe is cut into units of at most 16 matrix-kernel blocks, and the kernel's CTAs
 * take units in order as they are published. Every device wait is bounded: a CTA that
 * waits longer than timeout_ns (global timer; 0 = 1 s) for a unit that is not published
 * and not closed gives up, and the session ends with RS_ERR_TIMEOUT (the device stays
 * usable; units published before were run). Reconstruct units use decode rows built on
 * the host and copied to the queue's device arena (arena_bytes; 0 = 64 MiB) before they
 * are published. All work runs on the matrix route. While a session runs the caller
 * frees no device or pinned memory (rs8_free included): CUDA's frees synchronize the
 * device and would wait for the session's kernel, which ends only at close or at the
 * timeout. The kernel keeps two CTAs per SM, leaving room for the kernels of other
 * calls made meanwhile. */
typedef struct rs_queue rs_queue_t;
int rs_queue_create(size_t max_units, size_t arena_bytes, uint64_t timeout_ns, rs_queue_t **out);
/* Begins a session (RS_ERR_INVALID_ARGUMENT while one runs). */
int rs_queue_start(rs_queue_t *queue);
/* Appends and publishes stripes; RS_ERR_TOO_LARGE when the session's units or arena
 * would overflow (nothing is published then). The rows must stay valid until the
 * session ends. */
int rs_queue_push(rs_queue_t *queue, const rs_batch_item *items, size_t n_items, int *statuses);
/* Units finished by the device so far and units published in this session. */
int rs_queue_progress(rs_queue_t *queue, uint64_t *done_units, uint64_t *published_units);
/* Closes the session (nothing more will be pushed), waits for the kernel and returns
 * its status: 0, or RS_ERR_TIMEOUT when a wait gave up before the close. */
int rs_queue_finish(rs_queue_t *queue);
/* Waits for the kernel without closing (it ends when a wait gives up: RS_ERR_TIMEOUT). */
int rs_queue_wait(rs_queue_t *queue);
void rs_queue_free(rs_queue_t *queue);

/* ---- request server: continuous batching on one GPU ----
 * No counterpart in the reference (a caller there runs one encode or reconstruct per
 * call on its own thread). A server owns a device arena, a set of streams and a
 * scheduler thread. Submitted requests wait in a FIFO queue and are admitted while a
 * slot is free and their working set fits in the arena: the staged payload
 * (host-memory requests), descriptors and decode rows, plus the generator table of
 * their shape unless it is already resident. Tables stay resident across requests and
 * idle ones are evicted, least recently used first, when space is needed. Every
 * completion frees its memory and slot, so new work is admitted while older work is
 * still running. GF(2^8) requests admitted together share one launch group (one FFT
 * launch per (K,K) shape, one ragged matrix launch for the rest); GF(2^16) requests
 * with k + m <= 256 are validated as such and then run as GF(2^8) requests (their
 * coefficients lie in the subfield); other GF(2^16) requests run one per group;
 * groups overlap on the server's streams. Results are the bytes the single-stripe
 * entry points produce. */
typedef struct {
  int field;                /* 8: ReedSolomon (k+m <= 256), 16: ReedSolomon16 (<= 65536) */
  int op;                   /* enum rs_batch_op */
  size_t data_shards;       /* k */
  size_t parity_shards;     /* m */
  size_t row_len;           /* shard bytes (even for field 16: low plane, then high) */
  uint8_t *rows;            /* k+m rows of row_len bytes back to back, data first */
  int rows_on_host;         /* 1: host memory, staged through the arena (pin it for
                               overlap); 0: device memory the caller keeps alive */
  const uint8_t *present;   /* k+m flags, reconstruct ops; copied at submit */
  uint64_t tag;             /* returned in the completion */
} rs_request;
typedef struct {
  uint64_t tag;
  int status;               /* 0 or a reference error / device error */
  uint32_t group_size;      /* requests in its launch group (0: nothing to do) */
  uint64_t submit_ns, admit_ns, done_ns; /* host steady clock */
  uint64_t bytes;           /* algorithmic bytes: (k+m)*len encode, (k+e)*len rebuild */
} rs_completion;
typedef struct {
  size_t arena_bytes;       /* device working memory (0: 1 GiB) */
  size_t pinned_bytes;      /* pinned host staging for descriptors (0: 64 MiB) */
  int slots;                /* requests in flight at most (0: 64) */
  int streams;              /* device streams (0: 4) */
  int max_batch;            /* GF(2^8) requests per launch group (0: 64) */
  int lookahead;            /* queued requests that may pass a head that does not fit */
  struct rs_mlp *model;     /* cost model choosing each FFT launch group's launch shape
                               (rs_batch_choose's inputs and outputs; null: the library's
                               automatic choice); must outlive the server */
} rs_server_config;
typedef struct {
  uint64_t submitted, completed, rejected;
  uint64_t groups, launches, merged; /* merged: requests that shared a group */
  uint64_t bytes;                    /* algorithmic bytes of completed requests */
  uint64_t table_builds, table_hits, evictions;
  size_t arena_bytes, arena_used, arena_peak;
  size_t queued, in_flight, resident_tables;
} rs_server_stats;
typedef struct rs_server rs_server_t;
/* RS_ERR_TOO_LARGE when the arena cannot be allocated with 256 MiB to spare. */
int rs_server_create(const rs_server_config *config, rs_server_t **out);
/* Validates and queues n requests; statuses[i] (optional) is the request's reference
 * error (as its single-stripe call would return it) or RS_ERR_TOO_LARGE when it can
 * never fit the arena. Rejected requests produce no completion; a reconstruct with
 * nothing to rebuild completes at once. Never blocks on the device. */
int rs_server_submit(rs_server_t *server, const rs_request *reqs, size_t n, int *statuses);
/* Moves up to cap completions into out; waits up to timeout_ms (-1: until one
 * arrives, 0: no wait) when none is ready. */
int rs_server_poll(rs_server_t *server, rs_completion *out, size_t cap, size_t *n_out,
                   int timeout_ms);
/* Route of (K,K) GF(2^8) encodes of 2^log2_bytes..2^(log2_bytes+1)-1 byte shards:
 * 0 automatic (FFT from 64 bytes), 1 matrix, 2 FFT. Set from the cost model. */
int rs_server_set_fft_route(rs_server_t *server, size_t k, int log2_bytes, int route);
int rs_server_stats_get(rs_server_t *server, rs_server_stats *out);
/* Waits for admitted work, drops requests still queued, frees everything. */
void rs_server_free(rs_server_t *server);

/* ========================= ReedSolomon16 (GF((2^8)^2)) ========================= */

/* ReedSolomon16::new, src/reedsolomon16.rs:281-319 (k + m <= 65536). */
int rs16_new(size_t data_shards, size_t parity_shards, rs16_t **out);
int rs16_clone(const rs16_t *codec, rs16_t **out);
void rs16_free(rs16_t *codec);
size_t rs16_data_shard_count(const rs16_t *codec);
size_t rs16_parity_shard_count(const rs16_t *codec);
size_t rs16_total_shard_count(const rs16_t *codec);
int rs16_equal(const rs16_t *a, const rs16_t *b);
/* Generator rows k..n-1 (m x k tower symbols) as built; row-major. */
int rs16_parity_matrix(const rs16_t *codec, uint16_t *out, size_t out_len);
/* ReedSolomon16::encode, src/reedsolomon16.rs:412-419: even nonzero equal lengths. */
int rs16_encode(rs16_t *codec, uint8_t *const *shards, size_t n_shards, size_t len);
/* ReedSolomon16::encode_sep, src/reedsolomon16.rs:422-446. */
int rs16_encode_sep(rs16_t *codec, const uint8_t *const *data, size_t n_data,
                    uint8_t *const *parity, size_t n_parity, size_t len);
/* ReedSolomon16::verify, src/reedsolomon16.rs:450-505. */
int rs16_verify(rs16_t *codec, const uint8_t *const *shards, size_t n_shards, size_t len,
                int *ok);
/* ReedSolomon16::{reconstruct, reconstruct_data}, src/reedsolomon16.rs:508-515. */
int rs16_reconstruct(rs16_t *codec, uint8_t *const *shards, const size_t *lens,
                     const uint8_t *present, size_t n_shards, int data_only);
/* ReedSolomon16::reconstruct_rows, src/reedsolomon16.rs:544-565 (even row_len). */
int rs16_reconstruct_rows(rs16_t *codec, uint8_t *rows, size_t rows_len, size_t row_len,
                          const uint8_t *present, size_t n_present);
/* ReedSolomon16::prepare_decode -> PreparedDecoder16, src/reedsolomon16.rs:518-541,710-753 */
int rs16_prepare_decode(rs16_t *codec, const uint8_t *present, size_t n_present,
                        rs16_dec_t **out);
int rs16_dec_reconstruct(rs16_dec_t *dec, uint8_t *const *shards, const size_t *lens,
                         const uint8_t *present, size_t n_shards, int data_only);
int rs16_dec_clone(const rs16_dec_t *dec, rs16_dec_t **out);
void rs16_dec_free(rs16_dec_t *dec);
/* ReedSolomon16::encode_route, src/reedsolomon16.rs:335-346: "fft" (bitsliced tower
 * LCH transform, src/fft16.rs; any k >= 2 and m, picked when its estimated work is
 * below the matrix kernel's) or "matrix". This is the shape's route; on the automatic
 * route an encode of few short stripes, where the transform's pass launches dominate,
 * takes the matrix kernel when that is estimated to finish first. "subfield": with
 * k + m <= 256 every evaluation point, hence every coefficient, lies in GF(2^8), which
 * scales the low and the high byte plane alike, so on the automatic route encode,
 * verify and reconstruct run the GF(2^8) codec of the same shape over the shard bytes
 * (after the tower's own argument checks; prepared decoders keep the tower kernels),
 * except an encode that would run the GF(2^8) matrix kernel where the tower FFT is
 * estimated faster (rs16_encode_route_for then reports "fft"). */
const char *rs16_encode_route(const rs16_t *codec);
/* The route an encode of n_stripes stripes of len-byte shards takes (introspection;
 * no counterpart in the reference). */
const char *rs16_encode_route_for(const rs16_t *codec, size_t len, size_t n_stripes);
/* Forced-route test hook like rs8_set_route: 0 automatic, 1 matrix, 2 FFT (encode for
 * k >= 2; reconstruct plans built afterwards use the FFT erasure decoder). Both routes
 * give identical bytes. */
int rs16_set_route(rs16_t *codec, int route);
/* Tuning hook, no counterpart in the reference: the tower FFT pass kernels, 2 (default)
 * runtime constants dispatched to compiled XOR networks, in passes of four levels
 * (radix 16, through shared memory), of five for one pass when the level count is odd,
 * then of two; 1 the same networks in passes of two levels; 0 constants applied through
 * shared-memory mask tables. All give the same bytes. Returns the previous value, or
 * -1 for another value. */
int rs_set_fft16_pass(int variant);
int rs16_encode_dev(rs16_t *codec, uint8_t *const *d_shards, size_t n_shards, size_t len,
                    void *stream);
/* Many stripes of one shape: stripe s reads k rows at d_data + s*data_stride and
 * writes m rows at d_parity + s*parity_stride, rows of row_len (even) bytes. */
int rs16_encode_batch_dev(rs16_t *codec, const uint8_t *d_data, size_t data_stride,
                          uint8_t *d_parity, size_t parity_stride, size_t n_stripes,
                          size_t row_len, void *stream);
int rs16_reconstruct_dev(rs16_t *codec, uint8_t *const *d_shards, const size_t *lens,
                         const uint8_t *present, size_t n_shards, int data_only,
                         void *stream);

/* ============================ payload framing ============================
 * The steps the reference's callers take on either side of the coder, with no
 * counterpart in the crate itself: shred-style FEC sets (the reference's Agave test
 * shape, RS(32,32) x 987-byte shards, src/reedsolomon.rs:973) and the tape outer
 * coder's segment chunking (benches/gf16-bench/src/bin/live.rs:1-16).
 * A payload of payload_len bytes fills stripes of k data shards of shard_len bytes in
 * order: byte p goes to stripe p / (k*shard_len), data shard (p / shard_len) % k,
 * offset p % shard_len, and the rest of the last stripe's data shards is zero. Stripes
 * are stored [stripe][k + m rows][shard_len] in device memory (d_stripes, n_stripes =
 * rs_frame_stripe_count(...), else RS_INCORRECT_SHARD_SIZE; shard_len 0 ->
 * RS_EMPTY_SHARD). */
size_t rs_frame_stripe_count(size_t payload_len, size_t data_shards, size_t shard_len);
/* Split d_payload into the stripes' data rows and encode every stripe's parity. */
int rs8_frame_encode_dev(rs8_t *codec, const uint8_t *d_payload, size_t payload_len,
                         size_t shard_len, uint8_t *d_stripes, size_t n_stripes, void *stream);
/* Rebuild the missing data shards of every stripe (present: n_stripes x n host flags,
 * the reference's data-only reconstruct) and reassemble the payload into d_payload.
 * statuses (host, optional) gets each stripe's status; the return value is the first
 * stripe's error (e.g. RS_TOO_FEW_SHARDS_PRESENT), whose payload bytes are then not
 * rebuilt, or 0. */
int rs8_frame_decode_dev(rs8_t *codec, uint8_t *d_stripes, size_t n_stripes, size_t shard_len,
                         const uint8_t *present, uint8_t *d_payload, size_t payload_len,
                         int *statuses, void *stream);
/* The same over ReedSolomon16 (shard_len even; split-plane shards hold the payload's
 * bytes in order). */
int rs16_frame_encode_dev(rs16_t *codec, const uint8_t *d_payload, size_t payload_len,
                          size_t shard_len, uint8_t *d_stripes, size_t n_stripes, void *stream);
int rs16_frame_decode_dev(rs16_t *codec, uint8_t *d_stripes, size_t n_stripes, size_t shard_len,
                          const uint8_t *present, uint8_t *d_payload, size_t payload_len,
                          int *statuses, void *stream);
/* Tape outer coder shape for a snapshot of `groups` groups: k = ceil(groups / 3) data
 * shards, m = groups - k parity shards (errors as rs16_new's). */
int rs_outer_shape(size_t groups, size_t *data_shards, size_t *parity_shards);
/* Its shard size for a segment: ceil(segment_len / k) rounded up to a multiple of 64
 * (at least 64); above 4 MiB -> RS_ERR_TOO_LARGE (the coder's "too much data"). */
int rs_outer_shard_bytes(size_t segment_len, size_t data_shards, size_t *shard_bytes);

/* ============================== gf slice kernels ============================== */

/* gf::mul_slice / mul_slice_xor, src/gf/mod.rs:69-85: out[i] (^)= c * in[i] over
 * GF(2^8). Differing lengths -> RS_ERR_LENGTH_MISMATCH (the reference panics). */
int gf8_mul_slice(uint8_t *out, size_t out_len, const uint8_t *in, size_t in_len, uint8_t c,
                  int xor_into);
int gf8_mul_slice_dev(uint8_t *d_out, const uint8_t *d_in, size_t n, uint8_t c, int xor_into,
                      void *stream);

/* ========================== learned cost model (MLP) ==========================
 * No counterpart in the reference. An FP32 MLP (n_in -> hidden x3 ReLU -> n_out)
 * trained and evaluated on the GPU by this library's kernels; the tuner maps a
 * workload's features to one predicted log-time per candidate launch configuration.
 * Device arrays are row-major float: x [batch x n_in], y and mask [batch x n_out]. */
int rs_mlp_create(int n_in, int hidden, int n_out, uint64_t seed, rs_mlp_t **out);
/* Input, hidden and output widths. */
int rs_mlp_dims(const rs_mlp_t *mlp, int *n_in, int *hidden, int *n_out);
/* The network to a file and back (magic, widths, float32 parameters). A file that is
 * not such a network -> RS_ERR_INVALID_ARGUMENT. */
int rs_mlp_save(const rs_mlp_t *mlp, const char *path);
int rs_mlp_load(const char *path, rs_mlp_t **out);
void rs_mlp_free(rs_mlp_t *mlp);
size_t rs_mlp_param_count(const rs_mlp_t *mlp);
int rs_mlp_get_params(const rs_mlp_t *mlp, float *out, size_t n);
int rs_mlp_set_params(rs_mlp_t *mlp, const float *in, size_t n);
int rs_mlp_predict(rs_mlp_t *mlp, const float *d_x, int batch, float *d_out);
/* Gradients of the masked mean squared error (sum over mask / mask_count) for every
 * parameter, in parameter order, into host memory; no update. */
int rs_mlp_gradients(rs_mlp_t *mlp, const float *d_x, const float *d_y, const float *d_mask, int batch,
                     float mask_count, float *grads_out, size_t n, float *loss);
/* One Adam step on the batch; *loss (optional) receives the loss before the step. */
int rs_mlp_train_step(rs_mlp_t *mlp, const float *d_x, const float *d_y, const float *d_mask, int batch,
                      float mask_count, float lr, float *loss);

/* ============================ device / diagnostics ============================ */

/* 0 when a CUDA device is usable, RS_ERR_NO_DEVICE otherwise. */
int rs_device_check(void);
/* Host-side construction (no device needed), for tests and offline tools.
 * field 8 or 16. Parity rows k..k+m-1 of the systematic generator the reference
 * builds as vandermonde(n,k) * inverse(top) (src/reedsolomon.rs:155-159), m x k
 * row-major, as u16. */
int rs_generator_rows(int field, size_t k, size_t m, uint16_t *out, size_t out_len);
/* Decode rows of a presence pattern: one row per missing shard (data ascending,
 * then parity ascending), mapping the first k present shards to it; the composed
 * form of src/reedsolomon.rs:539-585 and :877-889. *n_rows receives the count. */
int rs_decode_rows(int field, size_t k, size_t m, const uint8_t *present, uint16_t *out,
                   size_t out_len, size_t *n_rows);
/* Number of this library's kernel launches so far in this process. */
uint64_t rs_kernel_launch_count(void);
/* Tuning hook (autotuner): launch shape of the (k,k) bitsliced FFT kernel for batched
 * calls, 0..rs_fft_variant_count()-1 (CTAs per SM), or -1 for the automatic choice (the
 * default: this shape's tuned value on 16-byte aligned rows, a wide-lane shape on
 * unaligned ones). Setting a value fixes the shape for every call. Returns the previous
 * value, or -1 when out of range or (k,k) has no FFT kernel. */
int rs_set_fft_variant(size_t k, int variant);
int rs_fft_variant_count(void);
/* Tuning hook: lane-group width of the (k,k) FFT kernel, 0 = narrow, 1 = wide (more
 * lanes per 32-column group, fewer registers per lane), -1 = automatic (as above).
 * Returns the previous value, or -1 when (k,k) has no FFT kernel. */
int rs_set_fft_lanes(size_t k, int wide);
/* Tuning hook, no counterpart in the reference: host threads (1..64, default 8) that
 * gather a host-pointer stripe into pinned memory and scatter its parity back, for
 * stripes with at least 8 MiB to move. Returns the previous value; other values leave
 * it unchanged. */
int rs_set_host_copy_threads(int n);
/* Tuning hook, no counterpart in the reference: host-pointer encodes and reconstructs
 * gather their rows into pinned memory and cross the link in one copy each way (1, the
 * default, up to 256 MiB per call) or copy each shard on its own (0). Same bytes.
 * Returns the previous value. */
int rs_set_host_staging(int on);
/* Tuning hook: tile shape of the matrix kernel for batched and single calls
 * (parity rows per thread x output rows per CTA), 0..rs_matrix_variant_count()-1. */
int rs_set_matrix_variant(int variant);
int rs_matrix_variant_count(void);
/* Tuning hook, no counterpart in the reference: the kernel of strided matrix-route
 * calls (batched encode on the matrix route, batched and single-stripe reconstruct
 * rows) and of the ragged launches of batches and the request server: 3 (default) the
 * lookup kernel (per input row, the XORs of every subset of each nibble's bit planes in
 * shared memory; a coefficient is 16 lookups), 8- or 16-row output tiles by call size;
 * 4 the same with 8-row tiles only; 2 the bitsliced kernel whose warp-uniform
 * coefficients select compiled XOR networks, two output rows per network call; 1 the
 * same, one call per coefficient; 0 the SWAR kernel. Same bytes either way. Returns the
 * previous value, or -1 for another value. */
int rs_set_matrix_bits(int on);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif
