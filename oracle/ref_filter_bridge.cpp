/* Bridge to the reference's own scan-filter evaluation (TEST
 * INFRASTRUCTURE): builds InnerColumn<T>s (include/data_model/
 * inner_column.h) from decoded columns and a Comparison / LogicalOperation
 * tree (include/data_model/statement.h) from a cj_predicate, and runs the
 * reference's column-wise Statement::eval (src/statement.cpp:47-241), the
 * evaluation its loader applies before execute() (src/build_table.cpp:
 * 318-323). Compiled with src/statement.cpp by oracle/build_oracle.py. */
#include <cstring>
#include <memory>
#include <vector>

#include <data_model/inner_column.h>
#include <data_model/statement.h>

#include "../include/cj_b200.h"

namespace {

std::unique_ptr<Statement> make_stmt(const cj_predicate *p, uint64_t node) {
    const cj_pred_node &n = p->nodes[node];
    switch (n.kind) {
    case CJ_PRED_AND: return LogicalOperation::makeAnd(make_stmt(p, n.left), make_stmt(p, n.right));
    case CJ_PRED_OR: return LogicalOperation::makeOr(make_stmt(p, n.left), make_stmt(p, n.right));
    case CJ_PRED_NOT: return LogicalOperation::makeNot(make_stmt(p, n.left));
    default: break;
    }
    Literal lit;
    if (n.literal_type == CJ_INT64) lit = (int64_t)n.i64;
    else if (n.literal_type == CJ_FP64) lit = n.f64;
    else if (n.literal_type == CJ_VARCHAR) lit = std::string(n.str ? n.str : "", n.str_len);
    else lit = std::monostate{};
    return std::make_unique<Comparison>(n.column, (Comparison::Op)n.op, std::move(lit));
}

} // namespace

extern "C" int cjref_filter(uint64_t ncols, const int32_t *types, uint64_t rows, const uint8_t *const *valid,
                            const void *const *values, const uint64_t *const *offsets, const cj_predicate *pred,
                            uint8_t *selected) {
    try {
        std::vector<std::unique_ptr<InnerColumnBase>> cols;
        for (uint64_t c = 0; c < ncols; ++c) {
            switch (types[c]) {
            case CJ_INT32: {
                auto col = std::make_unique<InnerColumn<int32_t>>();
                const int32_t *v = (const int32_t *)values[c];
                for (uint64_t r = 0; r < rows; ++r) valid[c][r] ? col->push_back(v[r]) : col->push_back_null();
                cols.push_back(std::move(col));
                break;
            }
            case CJ_INT64: {
                auto col = std::make_unique<InnerColumn<int64_t>>();
                const int64_t *v = (const int64_t *)values[c];
                for (uint64_t r = 0; r < rows; ++r) valid[c][r] ? col->push_back(v[r]) : col->push_back_null();
                cols.push_back(std::move(col));
                break;
            }
            case CJ_FP64: {
                auto col = std::make_unique<InnerColumn<double>>();
                const double *v = (const double *)values[c];
                for (uint64_t r = 0; r < rows; ++r) valid[c][r] ? col->push_back(v[r]) : col->push_back_null();
                cols.push_back(std::move(col));
                break;
            }
            default: {
                auto col = std::make_unique<InnerColumn<std::string>>();
                const char *chars = (const char *)values[c];
                const uint64_t *o = offsets[c];
                for (uint64_t r = 0; r < rows; ++r) {
                    if (valid[c][r]) col->push_back(std::string_view(chars + o[r], o[r + 1] - o[r]));
                    else col->push_back_null();
                }
                cols.push_back(std::move(col));
                break;
            }
            }
        }
        std::vector<const InnerColumnBase *> view;
        for (auto &c : cols) view.push_back(c.get());
        std::vector<uint8_t> bits;
        if (pred) bits = make_stmt(pred, pred->root)->eval(view);
        for (uint64_t r = 0; r < rows; ++r) selected[r] = pred ? (bits[r / 8] >> (r % 8)) & 1 : 1;
        return 0;
    } catch (...) {
        return 1;
    }
}
