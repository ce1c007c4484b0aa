/*
 * cj_oracle.h — CPU oracle for the B200 join pipeline. TEST INFRASTRUCTURE.
 *
 * This library is the checker: a single-threaded C restatement of
 * CalamariJoins' execute() path (src/execute.cpp), its page format
 * (include/data_model/plan.h) and its page codec (src/build_table.cpp).
 * Only tests, the smoke check and the CPU-baseline leg of the benchmark may
 * load it. The product (libcj_b200.so) never links or calls it.
 *
 * Parity pinning: the restatement is checked against the 21 known-answer
 * cases of the reference's tests/unit_tests.cpp (fixtures under
 * tests/golden/) and, in the build container, against the reference's own
 * execute() compiled from its sources (oracle/_ref, built by
 * oracle/build_oracle.py).
 */
#ifndef CJ_ORACLE_H
#define CJ_ORACLE_H

#include "../include/cj_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A decoded column: one entry per row. */
typedef struct cjo_column {
    int32_t type;
    uint64_t num_rows;
    uint8_t *valid;    /* num_rows bytes, 1 = value present              */
    int32_t *i32;      /* INT32 values (0 where NULL)                    */
    int64_t *i64;      /* INT64 values                                   */
    double *f64;       /* FP64 values                                    */
    uint64_t *str_off; /* VARCHAR: num_rows+1 offsets into chars         */
    char *chars;
} cjo_column;

typedef struct cjo_table {
    uint64_t num_rows;
    uint64_t num_columns;
    cjo_column *columns;
} cjo_table;

/* Paged result of cjo_execute (ColumnInserter encoding). */
typedef struct cjo_result cjo_result;

int cjo_execute(const cj_plan_desc *plan, cjo_result **out);
uint64_t cjo_result_num_rows(const cjo_result *r);
uint64_t cjo_result_num_columns(const cjo_result *r);
int cjo_result_column(const cjo_result *r, uint64_t c, int32_t *type,
                      uint64_t *num_pages, const void **pages);
void cjo_result_free(cjo_result *r);

/* Decodes pages into rows (Table::from_columnar, build_table.cpp:520-659).
 * `pages` is an array of num_pages page pointers. Fails with
 * CJ_ERR_MALFORMED_PAGE if the pages hold a row count other than
 * expected_rows (pass UINT64_MAX to accept any). */
int cjo_decode_column(int32_t type, const void *const *pages,
                      uint64_t num_pages, uint64_t expected_rows,
                      cjo_column *out);
void cjo_column_free(cjo_column *c);

/* Same, for num_pages pages laid out consecutively at `pages`. */
int cjo_decode_column_contig(int32_t type, const void *pages,
                             uint64_t num_pages, uint64_t expected_rows,
                             cjo_column *out);

/* Structural check of one column's pages (header, bitmap popcount equals
 * n_values, VARCHAR offsets monotone and inside the page, long-string chains
 * well formed, total rows). Returns CJ_OK or CJ_ERR_MALFORMED_PAGE with a
 * message in msg. */
int cjo_validate_column(int32_t type, const void *pages, uint64_t num_pages,
                        uint64_t expected_rows, char *msg, uint64_t msg_len);

/* ColumnInserter<T> restatement (plan.h:187-366). Returns the page count in
 * *num_pages; with out_pages == NULL only counts. */
int cjo_encode_column(int32_t type, const void *values,
                      const uint64_t *offsets, const uint8_t *valid,
                      uint64_t n, void *out_pages, uint64_t capacity,
                      uint64_t *num_pages);

/* Row-multiset equality of two decoded tables (values, NULLs and VARCHAR
 * bytes; FP64 compared bitwise), the comparison of read_sql.cpp:1325-1360.
 * Returns 1 if equal, 0 if not (reason in msg). */
int cjo_tables_equal(const cjo_table *a, const cjo_table *b, char *msg,
                     uint64_t msg_len);

/* Convenience: decode two paged tables (consecutive pages per column) and
 * compare them. types/num_pages/pages describe `ncols` columns each. */
int cjo_paged_tables_equal(uint64_t ncols, const int32_t *types,
                           uint64_t rows_a, const uint64_t *num_pages_a,
                           const void *const *pages_a, uint64_t rows_b,
                           const uint64_t *num_pages_b,
                           const void *const *pages_b, char *msg,
                           uint64_t msg_len);

/* Order-insensitive 64-bit fingerprint of a paged table's row multiset
 * (sum over rows of a row hash); used for full-size property checks. */
/* Scan-side filter: rows of the host table for which `pred` holds (all
 * rows when pred is NULL), projected to `cols`, encoded as ColumnInserter
 * would, plus the selection as one byte per row in `selected` (may be
 * NULL; table->num_rows bytes). Follows the reference's column-wise
 * Comparison::eval / LogicalOperation::eval (src/statement.cpp:47-241,
 * include/data_model/inner_column.h) row by row. */
int cjo_filter(const cj_table_desc *table, const cj_predicate *pred, uint64_t ncols, const uint64_t *cols,
               cjo_result **out, uint8_t *selected);

/* Comparison::like_match's matching (statement.h:119-158): the whole
 * string, '%' any run and '_' one UTF-8 code point, neither a newline. */
int cjo_like(const char *s, uint64_t n, const char *pat, uint64_t m);

int cjo_paged_table_fingerprint(uint64_t ncols, const int32_t *types,
                                uint64_t rows, const uint64_t *num_pages,
                                const void *const *pages, uint64_t *fp);

#ifdef __cplusplus
}
#endif
#endif
