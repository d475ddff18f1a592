/*
 * cupami_b200 -- C ABI of the B200 vertical-bitset frequent-itemset engine.
 *
 * The entry points replace the GPU path behind cuPAMI's cuEclat / cuApriori.
 * Reference locations are given relative to the cuPAMI project root.
 *
 *   cpm_db_from_csr / cpm_db_from_ids
 *       replace cuApriori._getDevicePairs + _bitsets.build_bitsets
 *       (cupami/frequentPattern/cuApriori.py:378-404,
 *        cupami/frequentPattern/_bitsets.py:20-28, 91-100)
 *   cpm_mine(algo = CPM_ECLAT)
 *       replaces cuEclat.mine + cuEclat._searchClass
 *       (cupami/frequentPattern/cuEclat.py:168-245)
 *   cpm_mine(algo = CPM_APRIORI)
 *       replaces cuApriori.mine + _generateCandidates + _countCandidateSupports
 *       (cupami/frequentPattern/cuApriori.py:473-535)
 *   cpm_tdb_from_csr + cpm_mine_periodic
 *       replace TemporalInput._prepare + cuPFEclat.mine / cuPFApriori.mine
 *       (cupami/periodicFrequentPattern/_temporal.py:150-171,
 *        cuPFEclat.py:146-175, cuPFApriori.py:141-157)
 *   cpm_periodic_counts
 *       replaces the periodic_counts kernel (_temporal.py:26-53, :156-165)
 *   cpm_build_bitsets / cpm_count_supports / cpm_intersect_extensions
 *       replace the three kernel wrappers of cupami/frequentPattern/_bitsets.py:91-125
 *       one for one (same 32-bit word layout, device pointers in, device
 *       pointers out) for callers that drive their own search, such as the
 *       cuSpatialEclat hooks (cupami/georeferencedFrequentPattern/cuSpatialEclat.py:197-211).
 *
 * Conventions
 *   - Every function returns CPM_OK (0) or a negative CPM_E* code; no C++
 *     exception crosses the boundary.  cpm_last_error(ctx) describes the last
 *     failure on that context.
 *   - A context owns one CUDA device and one stream.  Calls on one context
 *     must not overlap (no internal locking); use one context per thread.
 *   - Pointers named d_* are device pointers on the context's device; every
 *     other pointer is host memory owned by the caller and only read or
 *     written during the call.
 *   - Item columns are indices into the caller's label table.  The reference
 *     orders labels as sorted strings (cuApriori.py:397); cpm_db_from_ids does
 *     that ordering itself for integer ids and returns the label table.
 *   - Supports pass when support >= min_sup (cuEclat.py:177,191,236).  A
 *     min_sup <= 0 lets every candidate through, zero supports included.
 */
#ifndef CUPAMI_B200_H
#define CUPAMI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CPM_OK          0
#define CPM_EINVAL     -1   /* bad argument */
#define CPM_ENOMEM     -2   /* device or host allocation failed */
#define CPM_ECUDA      -3   /* CUDA runtime error */
#define CPM_EOVERFLOW  -4   /* a device queue or arena stayed too small after retries */
#define CPM_ETIMEOUT   -5   /* a bounded device wait ran out (spin limit) */
#define CPM_ENODEV     -6   /* no usable CUDA device */
#define CPM_EINTERNAL  -7

#define CPM_ECLAT    0
#define CPM_APRIORI  1

/* Pattern order produced by cpm_result_copy. */
#define CPM_ORDER_ECLAT    0  /* insertion order of cuEclat.mine (cuEclat.py:168-245) */
#define CPM_ORDER_APRIORI  1  /* insertion order of cuApriori.mine: by length, then tuple */
#define CPM_ORDER_NONE     2  /* device emission order (fastest) */
#define CPM_ORDER_DEPTH_FIRST 3  /* insertion order of cuPFEclat.mine: singletons, then for each
                                    pattern in depth-first order its extensions
                                    (cupami/periodicFrequentPattern/cuPFEclat.py:150-173) */

/* Deep-level scheduler. */
#define CPM_SCHED_PLAIN    0  /* frames admitted largest first by member count */
#define CPM_SCHED_LEARNED  1  /* frames ordered by the cost model's predicted subtree cost */

typedef struct cpm_ctx cpm_ctx;
typedef struct cpm_db cpm_db;
typedef struct cpm_result cpm_result;

typedef struct {
    int32_t  scheduler;            /* CPM_SCHED_* */
    int32_t  pair_engine;          /* 0 auto, 1 tensor-core Gram, 2 CUDA-core Gram */
    uint64_t pair_batch;           /* mirrors cuEclat._PAIR_BATCH_SIZE; 0 = no limit */
    uint64_t intersection_bytes;   /* mirrors cuEclat._INTERSECTION_BATCH_BYTES; 0 = no limit */
    uint64_t arena_bytes;          /* device arena for child tidsets; 0 = automatic */
    uint64_t spin_limit;           /* bounded device waits; 0 = default */
    int32_t  collect_trace;        /* 1: record per-frame features and costs for the cost model */
    int32_t  deep_block;           /* deep-level kernel threads per CTA: 128, 256, 512 or 1024; 0 = automatic */
    int32_t  deep_ctas_per_sm;     /* resident deep-level CTAs per SM, 1-4 (capped by occupancy); 0 = automatic */
    int32_t  autotune;             /* 1: use the launch shape cpm_autotune found for this tidset length */
    int32_t  tidsets;              /* deep-level tidset forms.  0: bitsets, plus transaction-id lists for
                                      tidsets held by under 1/32 of the transactions when a database's
                                      frequent bitsets exceed half the L2 and one bitset fits in shared
                                      memory; 1: bitsets only; 2: lists wherever a bitset fits in shared
                                      memory */
    int32_t  list_div;             /* a tidset is stored as a list when its list takes at most 1/list_div
                                      of its bitset; 0 = the autotuner's choice, else 1 */
    int32_t  deep_balance;         /* deep-level siblings: 0 = automatic (a warp per sibling), 1 = a warp
                                      per sibling, 2 = split over warps by size */
    int32_t  deep_project;         /* deep levels: a unit whose prefix holds at most L transactions writes
                                      its children as bitsets numbered by rank within the prefix, mined one
                                      unit per warp.  0 = automatic (L = 65,408 when the search has at least
                                      16 root units per SM, else off), 1 = off, 128..65408 = L */
    int32_t  deep_rows;            /* deep levels of one database, with projection: 0 = automatic (a unit
                                      whose prefix rows take less work than its siblings' tidsets counts
                                      and writes its children row by row), 1 = off */
} cpm_opts;

typedef struct {
    uint64_t n_patterns;
    uint64_t n_frequent_items;
    uint64_t n_frequent_pairs;
    uint64_t frames;               /* deep equivalence classes processed */
    uint64_t work_items;           /* (frame, position) units processed */
    uint64_t intersections;        /* sibling AND+popcount operations */
    uint64_t bytes_alg;            /* sum over units of 8*W*(1 + siblings + survivors) */
    uint64_t pair_ops;             /* tensor ops issued by the pair Gram (2*K*rows*cols) */
    uint64_t kernel_launches;
    uint64_t retries;              /* arena/queue overflow retries (failed rounds included) */
    uint64_t deep_rounds;          /* memory-bounded rounds of the deep phase (0: one launch) */
    double   ms_pack;
    double   ms_pairs;
    double   ms_deep;
    double   ms_total;
    double   deep_gbs;             /* bytes_alg / ms_deep */
    double   pair_tops;            /* pair_ops / ms_pairs */
    uint64_t projected_units;      /* of work_items: units below a projected prefix (one warp each) */
    double   ms_local;             /* of ms_deep: the launches that mine those units */
    uint64_t row_units;            /* of work_items: units counted row by row (deep_rows) */
} cpm_stats;

/* ---- context ------------------------------------------------------------ */
int         cpm_init(int device, cpm_ctx **out);
void        cpm_shutdown(cpm_ctx *ctx);
const char *cpm_last_error(const cpm_ctx *ctx);
const char *cpm_version(void);
int         cpm_default_opts(cpm_opts *opts);

/* ---- databases ------------------------------------------------------------ */
/* CSR of item columns.  Empty rows are dropped and the rest renumbered in
 * order (cuApriori.py:391-392, 401-403); repeated columns in a row are
 * harmless.  Every column must be < n_items. */
int cpm_db_from_csr(cpm_ctx *ctx, const uint64_t *offsets, uint64_t n_rows,
                    const uint32_t *cols, uint64_t nnz, uint32_t n_items, cpm_db **out);

/* CSR of raw integer item ids (the BIN layout, docs/transaction-formats.md).
 * The library finds the distinct ids, orders them as their decimal strings
 * sort (cuApriori.py:383-385) and maps every id to its column.  After the
 * call, cpm_db_labels() returns the ids in column order. */
int cpm_db_from_ids(cpm_ctx *ctx, const uint64_t *offsets, uint64_t n_rows,
                    const uint32_t *ids, uint64_t nnz, cpm_db **out);

/* Many integer-id databases at once (cpm_db_from_ids for each, with one
 * upload, one presence pass and one packing pass for all of them); out[d]
 * is the database built from offsets[d] / ids[d]. */
int cpm_db_from_ids_batch(cpm_ctx *ctx, uint32_t n_db, const uint64_t *const *offsets,
                          const uint64_t *n_rows, const uint32_t *const *ids, const uint64_t *nnz,
                          cpm_db **out);

/* Autotuner of the deep level.  Mines db (Eclat) once per launch shape --
 * threads per CTA in {128, 256, 512, 1024} x resident CTAs per SM in 1..4, as far as
 * occupancy allows -- then, at the fastest shape, once per tidset form
 * (bitsets only, or lists at divisors 1, 2, 4, 8), keeping the best of two
 * deep-phase times each, and records the fastest shape and form in the
 * context for tidsets of this length (power-of-two bucket of the row stride);
 * mines whose opts set autotune = 1 (and leave tidsets and list_div at 0) use
 * them.  Neither changes the output.  No reference counterpart: the
 * reference launches one 256-thread block per candidate
 * (cupami/frequentPattern/_bitsets.py:103-125). */
int cpm_autotune(cpm_ctx *ctx, cpm_db *db, int64_t min_sup, const cpm_opts *opts,
                 int32_t *block, int32_t *ctas_per_sm, int32_t *list_div, double *ms_deep);

int  cpm_db_info(const cpm_db *db, uint64_t *n_transactions, uint32_t *n_items,
                 uint64_t *words);
int  cpm_db_labels(const cpm_db *db, uint32_t *ids_out);  /* n_items entries */
void cpm_db_free(cpm_db *db);

/* ---- mining --------------------------------------------------------------- */
int  cpm_mine(cpm_ctx *ctx, cpm_db *db, int64_t min_sup, int algo,
              const cpm_opts *opts, cpm_result **out);
/* Eclat over many independent databases in one pass: one launch per stage
 * and one persistent deep-level launch for the whole batch.  out[d] is the
 * result of dbs[d] at min_sups[d], equal to cpm_mine(dbs[d], min_sups[d],
 * CPM_ECLAT); each result's statistics are those of the whole batch.  The
 * reference mines one database per call (cuEclat.py:168-203). */
int  cpm_mine_batch(cpm_ctx *ctx, cpm_db **dbs, uint32_t n_db, const int64_t *min_sups,
                    const cpm_opts *opts, cpm_result **out);
int  cpm_result_size(const cpm_result *res, uint64_t *n_patterns, uint64_t *n_item_slots);
/* Flattened patterns in the requested order: pattern k is
 * items[offsets[k] .. offsets[k+1]) (columns, increasing), support supports[k]. */
int  cpm_result_copy(const cpm_result *res, int order, uint64_t *offsets,
                     uint32_t *items, uint64_t *supports);
/* Many results at once (e.g. from cpm_mine_batch): sizes[2k], sizes[2k+1] =
 * patterns and item slots of res[k]; with the output arrays non-null, the
 * results are written one after another, result k taking sizes[2k] + 1
 * offsets (restarting at 0), sizes[2k+1] items and sizes[2k] supports. */
int  cpm_results_copy(cpm_result *const *res, uint32_t n, int order, uint64_t *sizes,
                      uint64_t *offsets, uint32_t *items, uint64_t *supports);
/* Pattern tree form: pattern k = pattern parent[k] (or nothing when -1) plus item[k]. */
int  cpm_result_tree(const cpm_result *res, int64_t *parent, uint32_t *item,
                     uint64_t *support);
int  cpm_result_stats(const cpm_result *res, cpm_stats *stats);
/* Builds a result from a pattern tree held in host memory (parent[k] < k or
 * -1).  No device work: lets callers and tests reorder patterns with
 * cpm_result_copy without a GPU. */
int  cpm_result_from_tree(const int64_t *parent, const uint32_t *item, const uint64_t *support,
                          uint64_t n, cpm_result **out);
void cpm_result_free(cpm_result *res);

/* ---- learned scheduler cost model -------------------------------------------
 * No counterpart in the reference, whose class search runs in a fixed order
 * (cuEclat.py:195-245).  A one-hidden-layer FP32 MLP predicts
 * log(1 + subtree intersections) of every root unit (one position of a
 * top-level class) from cheap features; with CPM_SCHED_LEARNED and a loaded
 * model, root units are started in order of predicted cost (tidset length
 * included), largest first.  The order never changes the patterns or their
 * supports.  Traces (features and true costs) come from cpm_mine with
 * opts.collect_trace = 1 via cpm_result_trace.  Training, prediction and
 * gradients run in this library's CUDA kernels. */
int cpm_costmodel_params(uint32_t *n_features, uint32_t *n_params);
int cpm_costmodel_train(cpm_ctx *ctx, const float *X, const float *y, uint64_t n, uint32_t epochs, float lr,
                        uint64_t seed, float *params, float *loss_history);
int cpm_costmodel_predict(cpm_ctx *ctx, const float *params, const float *X, uint64_t n, float *y);
/* Gradient of (1/2n) * sum (f(x_i) - t_i)^2 in the standardised target space,
 * for every parameter (zero for the fixed standardisation entries). */
int cpm_costmodel_gradient(cpm_ctx *ctx, const float *params, const float *X, const float *y, uint64_t n,
                           float *grad, float *loss);
/* Loads the model used by CPM_SCHED_LEARNED on this context (NULL unloads). */
int cpm_costmodel_set(cpm_ctx *ctx, const float *params);
int cpm_result_trace(const cpm_result *res, float *X, float *y, uint64_t *n);

/* ---- reference kernel-module API (cupami/frequentPattern/_bitsets.py) ------- */
/* d_bitsets: uint32[items][ceil(transactions/32)], zero-filled here, then one
 * bit per (row, column) pair (_bitsets.py:20-28, 91-100). */
int cpm_build_bitsets(cpm_ctx *ctx, const uint64_t *d_rows, const uint32_t *d_columns,
                      uint64_t count, uint64_t transactions, uint32_t items,
                      uint32_t *d_bitsets);
/* supports[c] = popcount of the AND of the width rows candidates[c][0..width)
 * over words32 words (_bitsets.py:30-53, 103-113). */
int cpm_count_supports(cpm_ctx *ctx, const uint32_t *d_bitsets, uint64_t words32,
                       const uint32_t *d_candidates, uint64_t n_candidates, uint32_t width,
                       uint64_t *d_supports);
/* out[e] = prefix & extensions[e]; supports[e] = popcount(out[e])
 * (_bitsets.py:55-77, 116-125). */
int cpm_intersect_extensions(cpm_ctx *ctx, const uint32_t *d_prefix,
                             const uint32_t *d_extensions, uint64_t words32,
                             uint64_t n_extensions, uint32_t *d_out, uint64_t *d_supports);
/* Waits for the context's stream. */
int cpm_synchronize(cpm_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), so that callers can order their
 * own work or timing events with the library's launches. */
void *cpm_stream(const cpm_ctx *ctx);

/* ---- periodic-frequent patterns (cupami/periodicFrequentPattern) -----------
 * A temporal database holds one row per transaction in timestamp order, empty
 * baskets included (they keep their timestamp and count in the support
 * denominator, _temporal.py:109-136).  The periodicity of an itemset held by
 * rows r_1 < ... < r_s is max(ts[r_1] - 0, ts[r_2] - ts[r_1], ...,
 * ts[r_s] - ts[r_{s-1}], end - ts[r_s]), or end when s = 0 (_temporal.py:26-53). */

/* CSR of item columns, every row kept; timestamps[r] for row r, nonnegative and
 * nondecreasing; end >= the last timestamp.  Every column must be < n_items. */
int cpm_tdb_from_csr(cpm_ctx *ctx, const uint64_t *offsets, uint64_t n_rows, const uint32_t *cols,
                     uint64_t nnz, uint32_t n_items, const int64_t *timestamps, int64_t end, cpm_db **out);
/* Itemsets with support >= min_sup, support > 0 and periodicity <= max_per
 * (_temporal.py:166-171).  algo CPM_ECLAT (cuPFEclat) or CPM_APRIORI
 * (cuPFApriori): the same itemsets; copy them with cpm_result_copy_periodic in
 * CPM_ORDER_DEPTH_FIRST or CPM_ORDER_APRIORI for the reference's insertion order. */
int cpm_mine_periodic(cpm_ctx *ctx, cpm_db *db, int64_t min_sup, int64_t max_per, int algo,
                      cpm_result **out);
/* cpm_result_from_tree for periodic results: period[k] is pattern k's periodicity. */
int cpm_result_from_tree_periodic(const int64_t *parent, const uint32_t *item, const uint64_t *support,
                                  const int64_t *period, uint64_t n, cpm_result **out);
/* cpm_result_copy plus the periodicity of every pattern (periodic results only). */
int cpm_result_copy_periodic(const cpm_result *res, int order, uint64_t *offsets, uint32_t *items,
                             uint64_t *supports, int64_t *periods);
/* The reference kernel periodic_counts: for every candidate (width columns of
 * the 32-bit bitsets of cpm_build_bitsets), its support and periodicity over
 * rows < n_transactions with d_timestamps[row] (_temporal.py:26-53). */
int cpm_periodic_counts(cpm_ctx *ctx, const uint32_t *d_bitsets, uint64_t words32,
                        const uint32_t *d_candidates, uint64_t n_candidates, uint32_t width,
                        const int64_t *d_timestamps, uint64_t n_transactions, int64_t end,
                        uint64_t *d_supports, int64_t *d_periods);

/* ---- Pattern keys (host only) ------------------------------------------------
 * The dict keys of getPatterns() (cuApriori.py:537-539: "\t".join of the
 * pattern's labels) for a result in CSR form, built in C: pattern k's labels
 * (labels[label_off[c] .. label_off[c+1]) for column c) joined by `sep`, each
 * key followed by `end`, written back to back into `out`.  *len gets the bytes
 * needed; with `out` null or `cap` below it nothing is written. */
int cpm_join_labels(const uint64_t *offsets, const uint32_t *items, uint64_t n_patterns, const char *labels,
                    const uint64_t *label_off, uint32_t n_labels, char sep, char end, char *out, uint64_t cap,
                    uint64_t *len);

/* ---- Delimited text of integer baskets, parsed on the device ----------------
 * Replaces cupami/frequentPattern/_gpu_io.py:34-54 (read_text: cuDF parse of
 * a CSV/TSV file whose stripped, non-empty lines are unquoted integer baskets,
 * exploded to rows and items on the GPU), called from cuApriori._tryGpuFile
 * (cuApriori.py:223-254).  `text` holds the file's bytes; `sep` is the
 * one-byte separator.  Every line is stripped of ASCII whitespace; blank lines
 * become empty rows; any other line must be tokens separated by `sep` (with
 * optional whitespace around it), each token a canonical decimal id (no
 * leading zero unless "0", at most 4294967295).  A line outside that layout,
 * a non-ASCII byte or an empty token returns CPM_EINVAL, and the caller reads
 * the file on the CPU as the reference does for such layouts.  The result is a
 * host CSR (row k = ids[offsets[k], offsets[k+1])) for cpm_db_from_ids; ids
 * name the same labels as the tokens' strings. */
typedef struct cpm_csr cpm_csr;
int cpm_parse_int_text(cpm_ctx *ctx, const char *text, uint64_t n_bytes, int32_t sep, cpm_csr **out);
int cpm_csr_size(const cpm_csr *csr, uint64_t *n_rows, uint64_t *nnz);
int cpm_csr_copy(const cpm_csr *csr, uint64_t *offsets, uint32_t *ids);
void cpm_csr_free(cpm_csr *csr);

/* ---- Eclat without device allocation ---------------------------------------
 * No counterpart in the reference: cuPAMI allocates through CuPy's pool on
 * every call.  This entry point is for callers that cannot allocate device
 * memory while they mine -- their device memory is owned by another runtime's
 * pool, or allocation is forbidden once they have started.  The caller passes
 * the tidsets (d_bits: n_items rows of `stride` 64-bit words, stride even,
 * base 16-byte aligned, bit r of row c set when transaction r holds column c,
 * bits past n_transactions zero) and the outputs (pattern tree in device
 * memory: pattern k = pattern d_parent[k] (0xffffffff: none) plus column
 * d_item[k], support d_support[k], at most `capacity` patterns; the count goes
 * to *n_patterns).  The patterns and supports are those cpm_mine(CPM_ECLAT)
 * finds on the same tidsets; cpm_result_from_tree + cpm_result_copy order
 * them as the reference does.
 *
 * No cudaMalloc, cudaFree or other allocating call is made: every
 * intermediate buffer lives in one static device array of
 * CPM_NOALLOC_SCRATCH_BYTES, held by every GPU that loads the library until
 * the process exits.  Inputs needing more (a pair matrix or child tidsets that
 * do not fit) are rejected with CPM_EINVAL or CPM_EOVERFLOW and a message in
 * cpm_last_error.  The first call on each device looks up the array's device
 * address, so make that first call before any stream capture; the address is
 * kept for the life of the process and does not survive cudaDeviceReset (do
 * not reset a device between calls).  All calls share the array, so calls that
 * overlap on the GPU (two contexts, two threads) race and must be serialised
 * by the caller.  `opts` may be null; only its spin_limit is read (the bounded
 * wait of the deep-level work queue, CPM_ETIMEOUT when it runs out).  With
 * n_items == 0 the call returns CPM_OK and no patterns. */
#define CPM_NOALLOC_SCRATCH_BYTES (64ull << 20)
int cpm_mine_eclat_noalloc(cpm_ctx *ctx, const uint64_t *d_bits, uint64_t stride, uint32_t n_items,
                           uint64_t n_transactions, int64_t min_sup, const cpm_opts *opts,
                           uint32_t *d_parent, uint32_t *d_item, uint32_t *d_support,
                           uint64_t capacity, uint64_t *n_patterns);

#ifdef __cplusplus
}
#endif
#endif /* CUPAMI_B200_H */
