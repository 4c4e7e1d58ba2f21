/*
 * fgss.h -- C ABI of libfgss, the B200 (sm_100a) Jaccard set-similarity
 * self-join.  Plain C types only; every call returns a status and never exits.
 *
 * The reference project (RafaelQuirino/new_fgssjoin) has no library API: its
 * boundary is the `fgssjoin <ppjoin.bin> <threshold>` process
 * (src/fgssjoin_cli.cu:13-112) over four internal host calls.  Each entry
 * point below names the reference interface it replaces.
 *
 * Record order.  Record arrays are in the reference's MEMORY order: the .bin
 * file order reversed (src/fgssjoin/data.cu:97-113), i.e. descending size for
 * a well-formed file.  Pairs are oriented as the reference prints them:
 * (record with the lower memory index, record with the higher one) -- the
 * larger set first.
 *
 * Ownership.  The caller owns its inputs.  The library owns what it returns
 * (fgss_sets, fgss_pairs) until the matching *_free call.  The host columns
 * of a result are one page-locked block where one can be had (the copies
 * from the device run at the link's rate); fgss_pairs_free gives that block
 * back to a process-wide pool, which keeps at most 1 GiB of free blocks for
 * later results and releases the rest.
 *
 * Threading.  A context is bound to one device and one stream and is not
 * thread-safe; separate contexts are independent.
 */
#ifndef FGSS_H_
#define FGSS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FGSS_VERSION_MAJOR 0
#define FGSS_VERSION_MINOR 1

typedef enum fgss_status {
    FGSS_OK = 0,
    FGSS_ERR_INVALID = 1,      /* bad argument */
    FGSS_ERR_CUDA = 2,         /* CUDA runtime error (message in fgss_last_error) */
    FGSS_ERR_NOMEM = 3,        /* host or device allocation failed */
    FGSS_ERR_FORMAT = 4,       /* malformed input (truncated .bin, unsorted tokens ...) */
    FGSS_ERR_IO = 5,           /* file could not be opened / read / written */
    FGSS_ERR_UNSUPPORTED = 6,  /* outside the supported limits (set length > 65535 ...) */
    FGSS_ERR_TIMEOUT = 7,      /* a bounded device wait gave up */
    FGSS_ERR_CAPACITY = 8      /* a caller-sized buffer is too small */
} fgss_status;

typedef struct fgss_ctx fgss_ctx;

/* ---------------------------------------------------------------- context */

typedef struct fgss_options {
    int device;                  /* CUDA device ordinal (reference: device 0, fgssjoin_cli.cu:81) */
    void* stream;                /* cudaStream_t to run on; NULL = the library creates its own */
    int verbose;                 /* per-stage timings on stderr */
    const char* tune_cache_path; /* autotuner cache (JSON); NULL = in-memory only */
} fgss_options;

void fgss_options_default(fgss_options* opt);
fgss_status fgss_create(fgss_ctx** ctx, const fgss_options* opt);
void fgss_destroy(fgss_ctx* ctx);
const char* fgss_strerror(fgss_status st);
/* Detailed message of the last failing call on this context ("" if none). */
const char* fgss_last_error(const fgss_ctx* ctx);
int fgss_version(void);

/* ------------------------------------------------------------------- sets */

/* Library-owned record arrays (host memory), MEMORY order.
 * Reference: sets_t, include/fgssjoin/data.cuh:12-50. */
typedef struct fgss_sets {
    uint32_t* id;       /* record id (1-based input line number for tokenized text) */
    uint32_t* pos;      /* offset of each record in tokens */
    uint32_t* len;      /* size of each record */
    uint32_t* tokens;   /* all records concatenated, ascending term ids per record */
    uint32_t* loc;      /* per token: its q-gram position in the line (NULL when unknown) */
    uint64_t n_sets;
    uint64_t n_tokens;
    uint32_t n_terms;   /* max token + 1 (data.cu:77-78) */
    uint32_t max_len;
} fgss_sets;

/* A borrowed view of record arrays, host or device memory, MEMORY order. */
typedef struct fgss_sets_view {
    const uint32_t* id;
    const uint32_t* pos;
    const uint32_t* len;
    const uint32_t* tokens;
    uint64_t n_sets;
    uint64_t n_tokens;
    uint32_t n_terms;
    int on_device;      /* 1 = the four pointers are device pointers on the context's device */
} fgss_sets_view;

/* Reads a ppjoin .bin ([int32 id][int32 size][int32 token x size]...) into
 * MEMORY order.  Replaces sets_t* ppjoin_format(const char*, char)
 * (include/fgssjoin/data.cuh:57-60, src/fgssjoin/data.cu:31-126). */
fgss_status fgss_load_bin(const char* path, fgss_sets* out);

/* Writes sets (MEMORY order) as a .bin in FILE order (ascending size), and the
 * .loc side file when loc_path is not NULL and sets->loc is set.  The reference
 * has no writer (src/preprocess_cli.cpp:346-347 "TODO"); the layout is the one
 * its loader reads. */
fgss_status fgss_write_bin(const char* path, const char* loc_path, const fgss_sets* sets);

void fgss_sets_free(fgss_sets* sets);
fgss_sets_view fgss_sets_view_of(const fgss_sets* sets);

/* ------------------------------------------------------------- tokenizer */

enum { FGSS_TOK_QGRAM = 0, FGSS_TOK_KMER = 1 };

typedef struct fgss_tok_opts {
    int q;          /* q-gram size, or k for k-mers (<= 32) */
    int mode;       /* FGSS_TOK_QGRAM / FGSS_TOK_KMER */
    int pad;        /* q-grams: pad each line with q-1 pad_char on both sides */
    int pad_char;   /* padding byte (default 0x01) */
    int suffix;     /* q-grams: 1 = each repeat is its own token (gram + occurrence,
                       src/preprocess/string/qgram.cpp:27-44); 0 = distinct grams */
    int lower;      /* ASCII lower-case first (src/preprocess/string/data.cpp:36-40) */
} fgss_tok_opts;

void fgss_tok_opts_default(fgss_tok_opts* o);

/* Text (lines separated by '\n'; empty lines skipped, src/io.cpp:8-26) ->
 * token sets on the GPU: q-grams or canonical k-mers, term ids by ascending
 * document frequency with ties broken by first occurrence
 * (src/preprocess_cli.cpp:266-340 and the fixture
 * test/data/string/small.txt.3gram.bin), ids ascending within a record,
 * records ordered as a .bin lists them and returned in MEMORY order.
 * Lines that yield no token are dropped.  Replaces the reference's
 * preprocess pipeline (src/preprocess_cli.cpp:222-358). */
fgss_status fgss_tokenize(fgss_ctx* ctx, const char* text, uint64_t n_bytes,
                          const fgss_tok_opts* opts, fgss_sets* out);

/* Two texts tokenized over one vocabulary (the text of R, then the text of S,
 * as one input to fgss_tokenize): term ids by document frequency over both.
 * out_r and out_s get the records of each text in MEMORY order, ids counting
 * the non-empty lines of their own text, n_terms of the shared vocabulary.
 * The reference's preprocess CLI has a "dualjoin" mode with this purpose
 * (src/preprocess_cli.cpp:22-32,93-119) that reads only its first file. */
fgss_status fgss_tokenize_dual(fgss_ctx* ctx, const char* text_r, uint64_t n_r, const char* text_s,
                               uint64_t n_s, const fgss_tok_opts* opts, fgss_sets* out_r, fgss_sets* out_s);

/* ------------------------------------------------------------------ join */

enum { FGSS_BOUNDS_REFERENCE = 0, /* float32 bounds exactly as similarity.cuh:9-82 */
       FGSS_BOUNDS_EXACT = 1 };   /* exact rational bounds of the decimal threshold */
enum { FGSS_METHOD_PLAIN = 0,     /* per-stage launches, exact two-pass counts */
       FGSS_METHOD_BATCHED = 1 }; /* persistent fused kernel, learned presizing, CUDA graph */
/* Filter strategies of the batched method (its candidate generation +
 * verification); every one gives the same pairs and counters.  The
 * reference's live filter is a thread per query (src/fgssjoin/filtering.cu:76-141);
 * its dead variants a CTA per query (filtering.cu:300-407). */
enum { FGSS_FILTER_AUTO = 0,      /* the autotuner's choice for the join's workload class */
       FGSS_FILTER_WARP = 1,      /* fused kernel, one warp per query (32-thread CTAs, small slot table) */
       FGSS_FILTER_CTA = 2,       /* fused kernel, one 128-thread CTA per query (large slot table) */
       FGSS_FILTER_GLOBAL = 3 };  /* every query on the dense global-memory accumulator kernel */

typedef struct fgss_join_opts {
    float threshold;        /* Jaccard threshold in (0, 1) (fgssjoin_cli.cu:31-35) */
    int bounds;             /* FGSS_BOUNDS_* */
    int method;             /* FGSS_METHOD_* */
    int out_on_device;      /* 1 = pairs stay in device memory (library-owned) */
    int want_candidates;    /* 1 = also return the candidate list (debug / tests) */
    int use_model;          /* batched method: presize and bin with the learned model */
    uint64_t result_capacity; /* batched method: presized result slots; 0 = learned / automatic.
                                 Too small a value only costs an exact re-run. */
    uint64_t query_begin;   /* only queries (first records of pairs) in [query_begin, query_end) */
    uint64_t query_end;     /* are processed; 0, 0 = all.  Used to shard one join over GPUs. */
    int no_graph;           /* batched method on device inputs: 1 = never capture / replay a CUDA graph */
    int filter;             /* batched method: FGSS_FILTER_* */
} fgss_join_opts;

void fgss_join_opts_default(fgss_join_opts* o);

typedef struct fgss_stats {
    uint64_t candidates;      /* "# Candidates"  (block.cu:180,209) */
    uint64_t intersections;   /* "# Intersections" (block.cu:181,210) */
    uint64_t results;         /* "# Results" (block.cu:194,211) */
    uint64_t index_entries;   /* "# Inverted Index Entries" (fgssjoin_cli.cu:92) */
    uint64_t probe_tokens;    /* sum of probe-prefix lengths */
    uint64_t window_entries;  /* list entries inside the id+size windows that the filter read */
    uint64_t verified;        /* candidates that needed a merge */
    uint64_t heavy_queries;   /* queries that took the global-memory accumulator */
    uint32_t overflow_retries;/* presized buffers that overflowed and were re-run exactly */
    float ms_total;           /* device time of the whole call (CUDA events) */
    float ms_index;           /* prefix lengths + inverted index */
    float ms_filter;          /* candidate generation (+ verification when fused) */
    float ms_verify;          /* verification (plain method) */
    float ms_output;          /* compaction, sort, copy-out */
    float ms_probe;           /* batched method: the fused filter+verify kernel alone */
    uint64_t merged_tokens;   /* source tokens the fused kernel's merges read */
    uint64_t launches;        /* kernels launched by the call */
    uint64_t predicted_candidates; /* batched method with use_model: the learned model's estimates */
    uint64_t predicted_results;    /* of candidates and results (0 otherwise; compare with the exact counts) */
    uint64_t query_tokens;    /* batched method: tokens of the query records the fused kernel staged */
    float ms_heavy;           /* batched method: the global-memory accumulator's launch alone */
    float ms_reserved;
} fgss_stats;

typedef struct fgss_pairs {
    uint32_t* q;        /* memory index of the first record */
    uint32_t* s;        /* memory index of the second record */
    uint32_t* id_q;     /* id[q] */
    uint32_t* id_s;     /* id[s] */
    uint32_t* overlap;  /* |x n y| */
    float* sim;         /* float(overlap) / float(|x| + |y| - overlap) (similarity.cuh:78-82) */
    uint64_t n;
    int on_device;
    /* candidates (want_candidates): (q, s, partial score) triples, host memory */
    uint32_t* cand;
    uint64_t n_cand;
    void* priv;  /* the library's: the page-locked block holding the host columns, or NULL */
} fgss_pairs;

/* Self-join at one threshold; pairs sorted by (q, s).  Replaces
 * prepare_data + inverted_index + process_blocks
 * (data.cuh:72-74, index.cuh:99-100, block.cuh:13-14; src/fgssjoin_cli.cu:86-100). */
fgss_status fgss_selfjoin(fgss_ctx* ctx, const fgss_sets_view* sets, const fgss_join_opts* opts,
                          fgss_pairs* out, fgss_stats* stats);

/* Many independent self-joins (each with its own sets and threshold) in one
 * launch per stage for the whole batch with the batched method (prefix
 * lengths, index, pre-pass, work items, the persistent fused filter+verify
 * kernel, result sort and output; a batch whose tokens or records exceed the
 * 32-bit batch offsets runs as consecutive groups).  outs and stats are arrays
 * of n (stats may be NULL).  No reference counterpart: it runs process_blocks
 * once per join. */
fgss_status fgss_selfjoin_batch(fgss_ctx* ctx, const fgss_sets_view* sets, const fgss_join_opts* opts,
                                int n, fgss_pairs* outs, fgss_stats* stats);

void fgss_pairs_free(fgss_pairs* p);

/* Per-query work estimates of one join, for splitting its queries (the first
 * records of pairs) over GPUs: costs[q] (n_sets values, host memory) = the
 * window entries of q's probe prefix + 4 x the learned model's predicted
 * candidates of q (opts->use_model and a trained model) + |q|, the cost the
 * batched method balances its work items by.  Runs the index build and the
 * batched pre-pass on the device.  No reference counterpart (the reference
 * runs on device 0 only, src/fgssjoin_cli.cu:81). */
fgss_status fgss_query_costs(fgss_ctx* ctx, const fgss_sets_view* sets, const fgss_join_opts* opts,
                             uint64_t* costs);

/* Formats pairs as the reference prints them: "%d %d %f\n" per pair
 * (block.cu:193).  Writes to the FILE* given as a void* (stdout if NULL). */
fgss_status fgss_pairs_print(const fgss_pairs* p, void* file);

enum { FGSS_OUT_TEXT = 0, FGSS_OUT_BINARY = 1 };

/* Streaming self-join for result sets too large to hold: the join runs as
 * n_shards query ranges of about equal work (records are in memory order, the
 * work of a query grows with its size squared), and a host thread formats and
 * writes each shard's pairs to `path` while the GPU joins the next one, so
 * output overlaps compute and at most two shards' pairs are in host memory.
 * FGSS_OUT_TEXT writes the reference's "%d %d %f\n" line per pair (block.cu:193,
 * printed there inside the join); FGSS_OUT_BINARY writes uint32 id_q, uint32 id_s,
 * float sim per pair.  Pairs come out sorted by (q, s) as with fgss_selfjoin.
 * stats: summed over the shards.  opts as for fgss_selfjoin, without a query
 * range, out_on_device or want_candidates. */
fgss_status fgss_selfjoin_to_file(fgss_ctx* ctx, const fgss_sets_view* sets, const fgss_join_opts* opts,
                                  const char* path, int format, int n_shards, fgss_stats* stats);

/* ------------------------------------------------------------- autotuner */

typedef struct fgss_tune_result {
    int threads;       /* CTA size of the fused filter+verify kernel */
    int hash_log2;     /* shared-memory slot table size (log2) */
    int regs_rt;       /* resident threads per SM the register budget is sized for */
    int ctas_per_sm;   /* resident CTAs per SM (0 = as many as fit) */
    float ms;          /* best filter+verify time measured (device) */
    char key[64];      /* workload class the choice is cached under */
    int filter;        /* the winning strategy: FGSS_FILTER_WARP / _CTA / _GLOBAL */
} fgss_tune_result;

/* Times every filter strategy of the batched method on this join -- each launch
 * shape of the fused kernel (one warp or one CTA per query) and the dense
 * global-memory accumulator for every query -- (reps runs each, best kept)
 * and caches the fastest for its workload class
 * (threshold, record-count and average-size buckets), in the context and in
 * the JSON file of fgss_options.tune_cache_path when one was given.  Later
 * batched joins of the same class use it.  No reference counterpart. */
fgss_status fgss_autotune(fgss_ctx* ctx, const fgss_sets_view* sets, const fgss_join_opts* opts, int reps,
                          fgss_tune_result* best);

/* R-S join: every pair (r, s), r a record of R and s a record of S over one
 * vocabulary (fgss_tokenize_dual), with Jaccard >= t.  No reference
 * counterpart (the reference's "dualjoin" stops at tokenizing).  Defined as
 * the self-join of R and S together -- the union in memory order: descending
 * size, R before S at equal size, then the index within its side -- restricted
 * to pairs with one record from each side; so FGSS_BOUNDS_EXACT gives exactly
 * the pairs with J >= t, and the reference bounds the self-join's float32
 * boundary behaviour.  Pairs are (q = index in R, s = index in S), sorted by
 * (q, s); the counters count pairs across only.  opts: threshold, bounds,
 * method (plain or batched), use_model, result_capacity, out_on_device;
 * query ranges and want_candidates are rejected. */
fgss_status fgss_rsjoin(fgss_ctx* ctx, const fgss_sets_view* r, const fgss_sets_view* s,
                        const fgss_join_opts* opts, fgss_pairs* out, fgss_stats* stats);

/* ------------------------------------------------------- learned cost model */

/* Trains the 2-layer FP32 MLP of the batched method on counts logged by the
 * exact count pass over the given joins (GPU forward/backward kernels), and
 * keeps it in the context.  No reference counterpart. */
fgss_status fgss_model_train(fgss_ctx* ctx, const fgss_sets_view* sets, const float* thresholds,
                             int n, int epochs, float lr, uint64_t seed, float* final_loss);
fgss_status fgss_model_save(fgss_ctx* ctx, const char* path);
/* One forward + backward pass of the MLP on host arrays (n x 8 features,
 * n x 2 targets = per-query counts of candidates and results), for gradient
 * checks: params (354 floats) -> grads, loss.  The loss is the mean over rows
 * of sum_j exp(r_j) - y_j r_j with log-rates r_j = 8 * output_j clamped to
 * [-30, 30] (Poisson regression). */
fgss_status fgss_model_grad(fgss_ctx* ctx, const float* feat, const float* target, uint64_t n, const float* params,
                            float* grads, float* loss);
/* Number of MLP parameters (W1, b1, W2, b2). */
int fgss_model_num_params(void);
fgss_status fgss_model_load(fgss_ctx* ctx, const char* path);

/* Host-side bound tables of one threshold (no device needed): for lengths
 * n <= max_len the probe prefix (jac_max_prefix), index prefix
 * (jac_mid_prefix), floor(n t) and floor(n / t) of
 * include/fgssjoin/similarity.cuh:9-58, and for length sums S <= 2 max_len the
 * smallest overlap the final test of src/fgssjoin/block.cu:190-193 accepts.
 * Any output pointer may be NULL. */
fgss_status fgss_bounds_table(float threshold, int bounds, uint32_t max_len, uint16_t* probe, uint16_t* index,
                              uint32_t* min_size, uint32_t* max_size, uint32_t* need);

/* Host-side overlap tables of one threshold (no device needed), per length sum
 * S <= max_sum (<= 131070): cand_min[S], the smallest integer k that the
 * positional test of src/fgssjoin/filtering.cu:130-132 does not reject
 * (!(k < jac_min_overlap)); inter_min[S], checking.cu:110's
 * floor(jac_min_overlap).  With fgss_bounds_table these are every bound the
 * join reads.  Any output pointer may be NULL. */
fgss_status fgss_overlap_table(float threshold, int bounds, uint32_t max_sum, uint32_t* cand_min,
                               uint32_t* inter_min);

/* ------------------------------------------------- device-level primitives */
/* Stage kernels exposed for tests and callers that keep data on the device.
 * All pointers are device pointers; the work runs on the context's stream
 * and the call returns after it completes. */

/* Exclusive prefix sum of n uint32 values (out may alias in).
 * Replaces exclusive_scan<unsigned int> (include/fgssjoin/scan.cuh:39-105). */
fgss_status fgss_dev_exclusive_scan_u32(fgss_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t n);

/* Exclusive prefix sum of n uint32 values that allocates no device memory,
 * for callers that cannot call cudaMalloc: a host that pre-allocates all
 * device memory up front and forbids later allocations, or a latency-critical
 * loop where cudaMalloc / cudaFree (which synchronizes the device) would
 * stall it.  No reference counterpart: the reference's scan
 * (include/fgssjoin/scan.cuh:39-105) allocates through Thrust.
 *   - Needs no context: it runs on `stream` (a cudaStream_t, NULL = the
 *     default stream) of the current device and returns once the work is
 *     queued; the result is ready when the stream reaches that point.
 *   - Scratch is a fixed 256 KiB array in the library (one per device, kept
 *     until the process exits), so n is limited to 268,435,456 elements;
 *     larger n returns FGSS_ERR_CAPACITY (message in fgss_last_error(NULL)).
 *   - Calls look the array's device address up (cudaGetSymbolAddress)
 *     whenever their stream is not capturing, so a device reset never leaves
 *     a stale address behind; make the first call on a device, and the first
 *     after a device reset, before any stream capture.
 *   - Every call shares that one array: calls that overlap on the GPU (other
 *     streams, other host threads) race and must be serialized by the caller.
 * Same result as fgss_dev_exclusive_scan_u32 (out may alias in). */
fgss_status fgss_dev_exclusive_scan_u32_noalloc(const uint32_t* in, uint32_t* out, uint64_t n, void* stream);

/* Stable LSD radix sort of n (key, value) pairs by key bits [begin_bit, end_bit).
 * No reference counterpart (the reference sorts on the host, preprocess_cli.cpp:170-215). */
fgss_status fgss_dev_sort_pairs_u64(fgss_ctx* ctx, uint64_t* keys, uint32_t* values, uint64_t n,
                                    int begin_bit, int end_bit);

#ifdef __cplusplus
}
#endif

#endif /* FGSS_H_ */
