/*
 * cj_b200.h — C ABI of the B200 join-pipeline library (libcj_b200.so).
 *
 * The library executes CalamariJoins-style equi-join plans on one NVIDIA
 * B200: paged columnar inputs (8 KiB pages, INT32 / INT64 / FP64 / VARCHAR,
 * NULL bitmaps, long-string pages) go in, a paged columnar result comes out.
 * Everything between (page decode, radix-partitioned hash build with Bloom
 * tags, probe, nested-loop join for tiny build sides, late-materialised
 * intermediates, page writing) runs as CUDA kernels on the device.
 *
 * Conventions
 *   - Every entry point returns a cj_status (0 = CJ_OK) and never throws or
 *     aborts. cj_last_error() returns a message for the calling thread.
 *   - Only plain C types and pointers cross this boundary.
 *   - Host page pointers may point to read-only memory; the library never
 *     writes input pages.
 *   - A cj_context is used by one host thread at a time (the reference's
 *     execute() is not re-entrant either: src/execute.cpp:311-313 resets a
 *     global arena). Different contexts may be used concurrently.
 *
 * Reference interfaces replaced (paths relative to the CalamariJoins tree):
 *   Contest::build_context()   include/data_model/plan.h:380, src/execute.cpp:327
 *   Contest::destroy_context() include/data_model/plan.h:382, src/execute.cpp:329
 *   Contest::execute()         include/data_model/plan.h:384, src/execute.cpp:311-325
 *   Contest::TimingStats       include/data_model/plan.h:370-378
 *   Plan / PlanNode / ScanNode / JoinNode   include/data_model/plan.h:46-72, 149-185
 *   ColumnarTable / Column / Page           include/data_model/plan.h:75-147
 *   DataType                                include/foundation/attribute.h:7-12
 *   ColumnInserter<T> (page encoder)        include/data_model/plan.h:187-366
 */
#ifndef CJ_B200_H
#define CJ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CJ_PAGE_SIZE 8192u
#define CJ_ABI_VERSION 1u

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
typedef enum cj_status {
    CJ_OK = 0,
    CJ_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad index, bad flag        */
    CJ_ERR_INVALID_PLAN = 2,     /* plan refers to missing nodes/columns,
                                    declared type differs from column type   */
    CJ_ERR_MALFORMED_PAGE = 3,   /* page header/bitmap inconsistent with the
                                    table's declared row count               */
    CJ_ERR_OUT_OF_MEMORY = 4,    /* device or pinned-host allocation failed  */
    CJ_ERR_CUDA = 5,             /* any other CUDA runtime error             */
    CJ_ERR_UNSUPPORTED = 6,      /* e.g. FP64 or VARCHAR join keys           */
    CJ_ERR_LIMIT = 7,            /* a documented size limit is exceeded      */
    CJ_ERR_NO_DEVICE = 8,        /* no CUDA device visible                   */
    CJ_ERR_REJECTED = 9,         /* serving: admission refused (budget)      */
    CJ_ERR_TIMEOUT = 10,         /* serving: wait gave up                    */
    CJ_ERR_CANCELLED = 11,       /* serving: request cancelled               */
    CJ_ERR_INTERNAL = 12         /* library invariant violated               */
} cj_status;

/* Values equal DataType's enumerators (include/foundation/attribute.h:7-12). */
typedef enum cj_data_type {
    CJ_INT32 = 0,
    CJ_INT64 = 1,
    CJ_FP64 = 2,
    CJ_VARCHAR = 3
} cj_data_type;

/* Values equal NodeType's enumerators (include/data_model/plan.h:46-49). */
typedef enum cj_node_type {
    CJ_NODE_HASH_JOIN = 0,
    CJ_NODE_SCAN = 1
} cj_node_type;

/* ------------------------------------------------------------------------ */
/* Plan description (POD mirror of Plan, include/data_model/plan.h:149-185)  */
/* ------------------------------------------------------------------------ */

/* One column of an input table: a type and an array of host pointers to
 * CJ_PAGE_SIZE-byte pages (Column, plan.h:82-142). */
typedef struct cj_column_desc {
    int32_t type;             /* cj_data_type                               */
    uint32_t reserved;
    uint64_t num_pages;
    const void *const *pages; /* num_pages host pointers                    */
} cj_column_desc;

/* ColumnarTable (plan.h:144-147). */
typedef struct cj_table_desc {
    uint64_t num_rows;
    uint64_t num_columns;
    const cj_column_desc *columns;
} cj_table_desc;

/* One entry of PlanNode::output_attrs: (column index, declared type). */
typedef struct cj_attr {
    uint64_t index;
    int32_t type; /* cj_data_type */
    uint32_t reserved;
} cj_attr;

/* PlanNode (plan.h:62-72): a ScanNode or a JoinNode plus output_attrs. */
typedef struct cj_plan_node {
    int32_t node_type;      /* cj_node_type                                 */
    int32_t build_left;     /* JoinNode::build_left (a hint; results do not
                               depend on it)                                */
    uint64_t base_table_id; /* ScanNode::base_table_id                      */
    uint64_t left, right;   /* JoinNode children (node indices)             */
    uint64_t left_attr, right_attr; /* join keys, indices into the children's
                                       output_attrs                          */
    uint64_t num_output_attrs;
    const cj_attr *output_attrs;
} cj_plan_node;

typedef struct cj_table cj_table; /* device-resident table (see below)    */

/* Plan (plan.h:149-185). Input i is taken from resident_inputs[i] when that
 * array is non-NULL and its entry is non-NULL, else from inputs[i]. */
typedef struct cj_plan_desc {
    uint64_t num_nodes;
    const cj_plan_node *nodes;
    uint64_t num_inputs;
    const cj_table_desc *inputs;       /* may be NULL if all inputs resident */
    cj_table *const *resident_inputs;  /* may be NULL                        */
    uint64_t root;
} cj_plan_desc;

/* Contest::TimingStats (plan.h:370-378), same fields and order. */
typedef struct cj_timing_stats {
    int64_t hashtable_build_ms;
    int64_t hash_join_probe_ms;
    int64_t nested_loop_join_ms;
    int64_t materialize_ms;
    int64_t setup_ms;
    int64_t total_execution_ms;
    int64_t intermediate_ms;
} cj_timing_stats;

/* Finer-grained statistics of one cj_execute call (no reference
 * counterpart; TimingStats' millisecond integers are too coarse for a GPU). */
typedef struct cj_exec_stats {
    double upload_us;        /* host->device page copies                    */
    double decode_us;        /* page decode kernels                         */
    double build_us;         /* hash-table build kernels                    */
    double probe_us;         /* hash probe kernels                          */
    double nested_loop_us;   /* nested-loop kernels                         */
    double intermediate_us;  /* row-id gathers for non-root joins           */
    double materialize_us;   /* output page writers                         */
    double download_us;      /* device->host result copy                    */
    double total_us;         /* wall time of the call                       */
    uint64_t h2d_bytes;
    uint64_t d2h_bytes;
    uint64_t num_joins;
    uint64_t num_hash_joins;
    uint64_t num_nested_loop_joins;
    uint64_t probe_rows;     /* probe-side rows over all joins              */
    uint64_t matches;        /* match pairs over all joins                  */
    uint64_t probe_reruns;   /* probes re-run after output overflow         */
    uint64_t output_rows;
    uint64_t output_pages;
    uint64_t kernel_launches;
    uint64_t num_direct_joins; /* hash joins served by a direct-mapped table
                                  (CJ_OPT_DENSE_KEYS); within num_hash_joins */
    uint64_t num_open_joins;   /* hash joins served by an open-addressing
                                  table (unique INT32 keys too spread out for
                                  a direct-mapped one); within num_hash_joins */
    uint64_t host_syncs;       /* times the host waited for the device: one
                                  per join (its match count), one per VARCHAR
                                  result (its page counts) and the last; a
                                  root over unique build keys whose result
                                  stays in HBM (CJ_EXEC_RESULT_ON_DEVICE, no
                                  VARCHAR column) needs only the last */
} cj_exec_stats;

/* ------------------------------------------------------------------------ */
/* Context: device, streams and stream-ordered device memory pool            */
/* ------------------------------------------------------------------------ */
typedef struct cj_context cj_context;

/* Creates a context on CUDA device `device` (-1 = current device).
 * Replaces Contest::build_context() (plan.h:380), which returns nullptr in the
 * reference (src/execute.cpp:327). */
int cj_context_create(int device, cj_context **out);

/* Replaces Contest::destroy_context(void*) (plan.h:382). Frees everything the
 * context owns; results and resident tables must be freed first. */
void cj_context_destroy(cj_context *ctx);

/* Tunables, each also settable by environment variable CJ_<NAME>. */
typedef enum cj_option {
    CJ_OPT_NESTED_LOOP_MAX_BUILD = 0, /* build rows below which the nested-loop
                                         kernel is used (reference: 8,
                                         src/execute.cpp:236-238); default 64 */
    CJ_OPT_SLOTS_PER_PARTITION = 1,   /* hash directory slots per radix
                                         partition (power of two, at most
                                         16384); 0 = the autotuner's
                                         choice, else 2048                  */
    CJ_OPT_PROFILE_KERNELS = 2,       /* 1 = time every kernel with events   */
    CJ_OPT_BLOCK_THREADS = 3,         /* threads per CTA of streaming kernels;
                                         0 = auto                           */
    CJ_OPT_VARCHAR_TILE_ROWS = 4,     /* rows per VARCHAR page-packing tile  */
    CJ_OPT_CTAS_PER_SM = 5,           /* CTAs per SM of the hash probe's
                                         persistent grid and of the radix
                                         passes; 0 = the autotuner's choice,
                                         else the kernels' defaults         */
    CJ_OPT_DENSE_KEYS = 6,            /* a build side whose non-NULL keys are
                                         unique and span at most this many
                                         times its row count (and 2^28
                                         values) uses a direct-mapped table
                                         (slot = key - min) instead of the
                                         hash table; unique INT32 keys that
                                         span more use an open-addressing
                                         table; same results; 0 = both off
                                         (hash table only); default 8       */
    CJ_OPT_BUFFER_CACHE_BYTES = 7,    /* device buffers freed by a plan are
                                         kept for the next one up to this
                                         many bytes (default 16 GiB; 0 = off;
                                         always 0 for server workers)       */
    CJ_OPT_FAIL_ALLOC_AT = 8          /* fault injection on the host: the
                                         N-th device allocation of this
                                         context from now on fails as if the
                                         pool were exhausted (the call
                                         returns CJ_ERR_OUT_OF_MEMORY and the
                                         context stays usable); one-shot;
                                         0 = off (default)                  */
} cj_option;
int cj_context_set_option(cj_context *ctx, int32_t option, int64_t value);
int cj_context_get_option(const cj_context *ctx, int32_t option, int64_t *value);

/* Autotuner (no reference counterpart; the reference sizes its radix
 * partitions from the cache share per thread, include/join_execution/
 * hashtable.h:172-188): times the unchained hash table's build and probe on
 * synthetic keys of each size class (row counts split at 2^12, 2^15, 2^18,
 * 2^21 and 2^24) and keeps, per class, the fastest directory slots per
 * radix partition, radix-pass CTAs per SM and probe CTAs per SM. The table
 * goes into the context and, when `path` is not NULL, into that file.
 * Options CJ_OPT_SLOTS_PER_PARTITION / CJ_OPT_CTAS_PER_SM override it;
 * results never depend on it. A context created while the environment
 * variable CJ_TUNING_FILE names a file loads that file (and fails to be
 * created if the file is malformed or was made for another GPU). */
#define CJ_TUNE_QUICK 1u /* time only the four smaller classes (the larger
                            ones take the largest timed class's entry)    */
int cj_autotune(cj_context *ctx, const char *path, uint32_t flags);
int cj_tuning_load(cj_context *ctx, const char *path);
/* Checks a tuning file's format without a GPU. */
int cj_tuning_check_file(const char *path);
/* The context's entry for size class `size_class` (0 = untuned default). */
int cj_tuning_entry(const cj_context *ctx, uint32_t size_class, int32_t *log2_spp,
                    int32_t *part_ctas, int32_t *probe_ctas);

/* Per-kernel profile (enabled by CJ_OPT_PROFILE_KERNELS): `index`-th kernel
 * name seen since the last reset, its launch count and total device time. */
int cj_profile_reset(cj_context *ctx);
int cj_profile_count(const cj_context *ctx, uint64_t *num_kernels);
int cj_profile_entry(const cj_context *ctx, uint64_t index, const char **name,
                     uint64_t *launches, double *total_us);

/* The cudaStream_t every kernel of this context runs on (for callers that
 * time or order their own work against it). */
int cj_context_stream(const cj_context *ctx, void **stream);

/* Device memory currently held by the context's pool (bytes in use, bytes
 * reserved) — for admission control and leak tests. */
int cj_context_memory(const cj_context *ctx, uint64_t *used_bytes,
                      uint64_t *reserved_bytes);

/* ------------------------------------------------------------------------ */
/* Resident tables: pages uploaded once and kept in HBM                      */
/* ------------------------------------------------------------------------ */

/* Uploads every column of `table` into device memory. A resident table
 * may be used by every context (and server) of the same device; free it
 * after the last plan that reads it. */
int cj_table_upload(cj_context *ctx, const cj_table_desc *table,
                    cj_table **out);

/* Adopts pages that are already in device memory: column c's pages are
 * num_pages[c] consecutive CJ_PAGE_SIZE-byte pages at device_pages[c]. The
 * memory stays owned by the caller and must outlive the cj_table. */
int cj_table_from_device(cj_context *ctx, uint64_t num_rows,
                         uint64_t num_columns, const int32_t *types,
                         const uint64_t *num_pages,
                         const void *const *device_pages, cj_table **out);

/* Device pointer of a resident column's pages (for tests and tools). */
int cj_table_column_pages(const cj_table *table, uint64_t column,
                          const void **device_pages, uint64_t *num_pages);

/* Copies a resident column's pages to caller memory (dst_bytes >=
 * pages * 8192). */
int cj_table_copy_column(const cj_table *table, uint64_t column, void *dst,
                         uint64_t dst_bytes);

void cj_table_free(cj_table *table);

/* Scan-side filters on resident tables. A predicate is a tree of nodes in
 * the form of the reference's Statement (include/data_model/statement.h):
 * comparisons of one column with a literal (Comparison, statement.h:54-64)
 * combined by AND / OR / NOT (LogicalOperation). Evaluation follows the
 * reference's column-wise Comparison::eval / LogicalOperation::eval
 * (src/statement.cpp:47-241, include/data_model/inner_column.h):
 *   - a comparison is false on a NULL row; IS_NULL / IS_NOT_NULL test the
 *     validity bit; NOT flips the bit of every row (NOT (x < 5) holds on the
 *     rows where x is NULL);
 *   - INT32 columns compare with the INT64 literal cast to int32 (its low 32
 *     bits), INT64 columns with the INT64 literal, FP64 columns with the
 *     FP64 literal (an INT64 literal given for an FP64 column is converted);
 *   - VARCHAR columns compare bytewise, a shorter prefix first, like
 *     std::string_view; LIKE / NOT LIKE match the whole string, '%' any run
 *     of characters and '_' one character (a UTF-8 code point), neither of
 *     them a newline (the RE2 pattern that Comparison::like_match builds,
 *     statement.h:119-158); NOT LIKE is false on NULL rows.
 * Comparisons of mismatched types (a VARCHAR literal for a numeric column, a
 * numeric literal for VARCHAR, LIKE on a numeric column) are
 * CJ_ERR_INVALID_PLAN. */
typedef enum cj_pred_kind {
    CJ_PRED_CMP = 0,
    CJ_PRED_AND = 1,
    CJ_PRED_OR = 2,
    CJ_PRED_NOT = 3
} cj_pred_kind;

/* Values equal Comparison::Op's enumerators (statement.h:57). */
typedef enum cj_cmp_op {
    CJ_CMP_EQ = 0,
    CJ_CMP_NEQ = 1,
    CJ_CMP_LT = 2,
    CJ_CMP_GT = 3,
    CJ_CMP_LEQ = 4,
    CJ_CMP_GEQ = 5,
    CJ_CMP_LIKE = 6,
    CJ_CMP_NOT_LIKE = 7,
    CJ_CMP_IS_NULL = 8,
    CJ_CMP_IS_NOT_NULL = 9
} cj_cmp_op;

typedef struct cj_pred_node {
    int32_t kind;           /* cj_pred_kind                                  */
    int32_t op;             /* cj_cmp_op (CJ_PRED_CMP)                       */
    uint64_t column;        /* column of the input table (CJ_PRED_CMP)        */
    uint64_t left, right;   /* children (AND / OR: both; NOT: left)           */
    int32_t literal_type;   /* CJ_INT64, CJ_FP64 or CJ_VARCHAR (Literal)      */
    uint32_t reserved;
    int64_t i64;
    double f64;
    const char *str;        /* VARCHAR literal bytes (str_len of them)        */
    uint64_t str_len;
} cj_pred_node;

typedef struct cj_predicate {
    uint64_t num_nodes;
    const cj_pred_node *nodes;
    uint64_t root;
} cj_predicate;

/* Rows of the resident table `in` for which `pred` holds (all rows when
 * pred is NULL), projected to `columns` (num_columns indices into in's
 * columns, in that order), as a new resident table whose pages are written
 * as ColumnInserter<T> writes pages (include/data_model/plan.h:187-366);
 * row order is kept. `*num_rows` (may be NULL) receives its row count.
 * The GPU form of the loader's filter pass before execute()
 * (src/build_table.cpp:201-367). */
int cj_table_filter(cj_context *ctx, const cj_table *in,
                    const cj_predicate *pred, uint64_t num_columns,
                    const uint64_t *columns, cj_table **out,
                    uint64_t *num_rows);

/* The reference's `.tbl` table cache (written by DumpTable::dump,
 * include/data_access/table.h:136-221; read by Table::from_cache,
 * src/build_table.cpp:140-197): an 8 KiB header page with TableMeta
 * (table.h:30-35) and zeros, then every column's pages in column order; at
 * most 16 columns. `cj_cache_meta` mirrors TableMeta. */
typedef struct cj_cache_meta {
    uint64_t num_rows;
    uint64_t num_columns;
    int32_t types[16];
    uint64_t num_pages[16];
} cj_cache_meta;

/* Reads and checks a cache file's header (no GPU needed); a header that
 * disagrees with the file size is CJ_ERR_MALFORMED_PAGE. */
int cj_cache_read_meta(const char *path, cj_cache_meta *meta);

/* Writes host pages as a cache file (the DumpTable format). */
int cj_table_write_cache(const cj_table_desc *table, const char *path);

/* Loads a cache file into a resident table: its pages cross to HBM once.
 * Replaces Table::from_cache for callers that keep tables on the GPU. */
int cj_table_load_cache(cj_context *ctx, const char *path, cj_table **out);

/* Catalog: resident tables by name (no reference counterpart; the
 * reference's driver maps one cache file per table and query). The catalog
 * owns its tables and frees them in cj_catalog_destroy. */
typedef struct cj_catalog cj_catalog;
int cj_catalog_create(cj_context *ctx, cj_catalog **out);
void cj_catalog_destroy(cj_catalog *cat);
int cj_catalog_add(cj_catalog *cat, const char *name, cj_table *table);  /* takes ownership */
int cj_catalog_load(cj_catalog *cat, const char *name, const char *path); /* a cache file   */
int cj_catalog_get(const cj_catalog *cat, const char *name, cj_table **table);
int cj_catalog_size(const cj_catalog *cat, uint64_t *count);
int cj_catalog_name(const cj_catalog *cat, uint64_t index, const char **name);

/* ------------------------------------------------------------------------ */
/* Execution                                                                 */
/* ------------------------------------------------------------------------ */
typedef struct cj_result cj_result;

typedef enum cj_exec_flags {
    CJ_EXEC_DEFAULT = 0,
    CJ_EXEC_RESULT_ON_DEVICE = 1 /* keep output pages in HBM; no D2H copy   */
} cj_exec_flags;

/* Runs `plan` to completion and returns its root result. Replaces
 * Contest::execute(const Plan&, void*, TimingStats*) (plan.h:384;
 * src/execute.cpp:311-325). `timing` and `stats` may be NULL.
 * Semantics: inner equi-join; a NULL key never matches; output columns are
 * the root's output_attrs over (left columns ++ right columns). An INT32
 * value equal to INT32_MIN that leaves a non-root join is NULL from then on
 * (the reference's intermediate encoding, include/data_model/intermediate.h:
 * 40-63). */
int cj_execute(cj_context *ctx, const cj_plan_desc *plan, uint32_t flags,
               cj_result **out, cj_timing_stats *timing, cj_exec_stats *stats);

/* Statistics of one cj_execute_batch call. */
typedef struct cj_batch_stats {
    uint64_t num_plans, num_levels, num_joins, num_hash_joins, num_nested_loop_joins;
    uint64_t probe_rows, matches, probe_reruns;
    uint64_t kernel_launches, syncs;
    uint64_t h2d_bytes, d2h_bytes;
    double total_us;
} cj_batch_stats;

/* Runs `num_plans` independent plans together (no reference counterpart):
 * plans advance level by level (a join's level = 1 + its children's), and
 * every phase of a level (build, nested-loop collect, probe, row-id gather)
 * is one grouped launch over all joins of that level in all plans, with one
 * host synchronisation per level. results[i] equals what cj_execute would
 * return for plans[i]; statuses[i] (may be NULL) is that plan's status
 * (a plan failing validation gets a NULL result and its code). A device-
 * side error fails the whole call. */
int cj_execute_batch(cj_context *ctx, const cj_plan_desc *plans,
                     uint64_t num_plans, uint32_t flags, cj_result **results,
                     int32_t *statuses, cj_batch_stats *stats);

/* Prepared batches (no reference counterpart): a batch of plans whose
 * inputs are all device-resident (cj_table), captured once as one CUDA
 * graph and replayed as often as wanted. cj_batch_prepare runs the batch
 * once to learn every join's match count and every VARCHAR column's page
 * count, then captures the same execution with outputs sized to those
 * counts, without any host synchronisation inside, over device buffers it
 * owns. cj_batch_run launches that graph (one launch for all the plans'
 * kernels) and waits for it. The results of a run equal cj_execute's for
 * each plan; their pages live in the prepared batch's buffers and are
 * overwritten by the next run of the same batch (free them or copy them
 * before). A run whose inputs no longer give the learned counts (the
 * resident tables were changed) fails with CJ_ERR_INVALID_ARGUMENT; prepare
 * the batch again. Plans with host inputs, or with VARCHAR result columns
 * (their page count depends on the order of the rows, which differs from
 * run to run), are refused with CJ_ERR_UNSUPPORTED. */
typedef struct cj_prepared cj_prepared;
int cj_batch_prepare(cj_context *ctx, const cj_plan_desc *plans,
                     uint64_t num_plans, uint32_t flags, cj_prepared **out);
int cj_batch_run(cj_prepared *batch, cj_result **results,
                 cj_batch_stats *stats);
void cj_prepared_free(cj_prepared *batch);

/* Hash join of two INT32 key arrays already in device memory, for callers
 * that must not have a library allocate device memory (an engine whose
 * allocator or fixed budget owns all of the GPU's memory). No counterpart
 * in the reference. All pointers are device pointers except h_count (host,
 * may be NULL); valid arrays are bitmaps of ceil(n/32) u32 words, bit r set
 * when row r has a key (NULL keys never match). The matching (build row,
 * probe row) pairs are written to out_build_rows / out_probe_rows (at most
 * `capacity` of them) in an unspecified order: probe order within each
 * tile of probe rows, tiles in the order they finish counting. *d_count
 * receives the full match count, and *h_count too when given; when it
 * exceeds `capacity` the pairs written are an arbitrary subset (nothing is
 * written past `capacity`): call again with capacity >= *d_count to get
 * them all. Work runs on `stream`
 * (a cudaStream_t) and the call returns after it completes.
 * Allocates nothing: the hash table and every scratch buffer live in one
 * fixed 12 MiB device array that each GPU loading the library holds until
 * exit. Limits: n_build <= 262,144 and n_probe <= 134,217,728; larger inputs
 * get CJ_ERR_LIMIT. The first call on a device looks up that array's device
 * address, so make it before any stream capture. Calls share the array:
 * calls that overlap on the GPU race and must not be issued concurrently. */
int cj_hash_join_noalloc(const int32_t *build_keys, const uint32_t *build_valid,
                         uint32_t n_build, const int32_t *probe_keys,
                         const uint32_t *probe_valid, uint32_t n_probe,
                         uint32_t *out_build_rows, uint32_t *out_probe_rows,
                         uint64_t capacity, unsigned long long *d_count,
                         uint64_t *h_count, void *stream);

int cj_result_num_rows(const cj_result *r, uint64_t *num_rows);
int cj_result_num_columns(const cj_result *r, uint64_t *num_columns);

/* Column `c` of a result: type, page count and, unless the result was kept on
 * the device, a host pointer to its num_pages consecutive pages. */
int cj_result_column(const cj_result *r, uint64_t c, int32_t *type,
                     uint64_t *num_pages, const void **host_pages);

/* Device pointer to column `c`'s consecutive pages (valid until free). */
int cj_result_column_device(const cj_result *r, uint64_t c,
                            const void **device_pages);

/* Copies column `c`'s pages to caller memory (dst_bytes >= pages*8192). */
int cj_result_copy_column(const cj_result *r, uint64_t c, void *dst,
                          uint64_t dst_bytes);

void cj_result_free(cj_result *r);

/* ------------------------------------------------------------------------ */
/* Serving: plans run concurrently as they arrive (no reference counterpart; */
/* the reference executes one plan per execute() call)                       */
/* ------------------------------------------------------------------------ */
typedef struct cj_server cj_server;

typedef struct cj_server_config {
    int32_t device;          /* -1 = current device                          */
    uint32_t slots;          /* worker streams, each running one plan or one
                                batch of plans at a time; 0 = 4              */
    uint64_t memory_budget;  /* device bytes that admitted plans may hold by
                                estimate; 0 = 85% of the free memory         */
    uint32_t exec_flags;     /* cj_exec_flags for every result               */
    uint32_t max_batch;      /* continuous batching: a slot that frees up
                                takes up to this many queued plans that fit
                                the budget and runs them as one grouped
                                execution (cj_execute_batch); 0 = 32, 1 = one
                                plan per slot                                */
    uint64_t age_limit_us;   /* admission passes over a queued plan that
                                does not fit beside the running ones to
                                admit later plans that do, for at most this
                                long after its submission; then it goes
                                first; 0 = 20,000                            */
    uint64_t host_cache_bytes; /* page-locked host memory reserved at creation
                                for host results, which are carved from it
                                (any mix of sizes, no allocation while it has
                                room); 0 = none: blocks are allocated as
                                needed and cached by size for reuse          */
    uint64_t device_reserve_bytes; /* device memory the server's pool takes at
                                creation and keeps, so that the first large
                                batches do not wait for the pool to grow
                                (mapping new memory is slow); 0 = the pool
                                grows on demand                              */
} cj_server_config;

typedef struct cj_server_stats {
    uint64_t submitted, completed, failed, rejected, cancelled;
    uint64_t queued, running;
    uint64_t admitted_bytes, peak_admitted_bytes, memory_budget;
    double p50_us, p99_us, mean_us, max_us; /* submit -> completion         */
    double wall_s;                          /* first submit -> last finish  */
    double plans_per_s;
    uint64_t batches;                       /* executions (one plan or a
                                               grouped batch)               */
    uint64_t skipped_ahead;                 /* plans admitted ahead of an
                                               earlier one that did not fit */
    double mean_batch;                      /* plans per execution          */
    uint64_t batch_fallbacks;               /* grouped executions that failed
                                               as a whole, their plans then
                                               run one by one               */
    uint64_t pinned_allocs;                 /* page-locked host blocks
                                               allocated for results (the
                                               rest came from the cache)    */
    uint64_t pinned_alloc_bytes;
    uint64_t pool_high_bytes;               /* most device memory the server's
                                               pool has held (since creation
                                               or the last reset)          */
} cj_server_stats;

int cj_server_create(const cj_server_config *config, cj_server **out);

/* Queues a plan. The plan description and every page it points to must stay
 * valid until cj_server_wait returns for the ticket. Plans whose estimated
 * footprint (cj_server_estimate) exceeds the budget are refused with
 * CJ_ERR_REJECTED; others wait until a slot is free and their estimate fits
 * beside the running plans. Admission goes in arrival order, except that a
 * plan that does not fit may be passed over by later plans that do, for at
 * most age_limit_us. Each result equals what cj_execute returns for the
 * plan alone. */
int cj_server_submit(cj_server *server, const cj_plan_desc *plan,
                     uint64_t *ticket);

/* Waits up to timeout_us (-1 = forever) for a ticket; returns the plan's
 * status and its result (caller frees it, before cj_server_destroy), or
 * CJ_ERR_TIMEOUT if it is still queued or running. */
int cj_server_wait(cj_server *server, uint64_t ticket, int64_t timeout_us,
                   cj_result **out, cj_exec_stats *stats);

/* Cancels a queued plan (its wait returns CJ_ERR_CANCELLED). */
int cj_server_cancel(cj_server *server, uint64_t ticket);

int cj_server_get_stats(cj_server *server, cj_server_stats *out, int reset);

/* Estimated device footprint of a plan in bytes (admission control). */
int cj_server_estimate(const cj_plan_desc *plan, uint64_t *bytes);

/* Stops the workers after their running plans; queued plans are dropped. */
void cj_server_destroy(cj_server *server);

/* ------------------------------------------------------------------------ */
/* Host utilities                                                            */
/* ------------------------------------------------------------------------ */

/* Page-locked host memory for inputs whose upload should run at full PCIe
 * speed. */
int cj_host_alloc(uint64_t bytes, void **out);
void cj_host_free(void *p);

/* Number of pages ColumnInserter<T> (plan.h:187-366) produces for the given
 * column; `valid` (one byte per row, nonzero = value present) may be NULL
 * (no NULLs). For VARCHAR, `offsets` has n+1 entries delimiting the strings
 * in `chars`. */
int cj_encode_num_pages(int32_t type, const void *values,
                        const uint64_t *offsets, const uint8_t *valid,
                        uint64_t n, uint64_t *num_pages);

/* Encodes a column exactly as ColumnInserter<T>::insert / insert_null /
 * finalize would (plan.h:187-366), into `out_pages` (capacity pages). For
 * fixed-width types `values` holds n elements (entries of NULL rows are
 * ignored); for VARCHAR `values` is the character buffer. */
int cj_encode_column(int32_t type, const void *values, const uint64_t *offsets,
                     const uint8_t *valid, uint64_t n, void *out_pages,
                     uint64_t capacity, uint64_t *num_pages);

/* Message of the last failed call on this thread ("" if none). */
const char *cj_last_error(void);

/* Library and ABI version, e.g. "cj_b200 1 sm_100a". */
const char *cj_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CJ_B200_H */
