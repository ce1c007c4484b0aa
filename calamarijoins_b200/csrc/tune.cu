/*
 * tune.cu — the autotuner: launch parameters of the unchained hash table's
 * build and probe, chosen per size class of the relation by timing them on
 * this GPU, kept in the context and cached in a text file.
 *
 * The reference sizes its radix partitions from the last-level cache share
 * per thread (include/join_execution/hashtable.h:172-188) and has no other
 * tunable. Here, per size class (row counts split at 2^12, 2^15, 2^18, 2^21
 * and 2^24), the tuner times on synthetic keys of that class:
 *   - directory slots per radix partition (2^9 .. 2^13), which sets the
 *     radix fan-out and, above 12 bits, the second partitioning pass;
 *   - CTAs per SM of the radix histogram and scatter passes (2, 4, 8);
 *   - CTAs per SM of the persistent hash probe (2, 4, 6, 8);
 * and keeps the fastest of each. Results do not depend on any of them.
 *
 * File format (text, one class per line after the header):
 *   cj_b200-tuning 1 <SM count>
 *   class <c> log2_spp <v> part_ctas <v> probe_ctas <v>
 */
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"
#include "exec_common.h"

namespace cj {
namespace {

/* A 32-bit integer hash (Chris Wellons' "lowbias32": xorshift-multiply
 * rounds) used only to generate synthetic keys. */
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

/* keys[i]: drawn over [0, domain) (so the build side repeats keys), or,
 * for a `outside_permille` share, from [domain, 2 domain) (probe keys
 * without a match). */
__global__ void k_tune_keys(int32_t *keys, uint64_t n, uint32_t domain, uint32_t seed, uint32_t outside_permille) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = mix32((uint32_t)i * 2654435761u ^ seed);
        uint32_t k = mix32(x + 0x9e3779b9u) % domain;
        if (x % 1000u < outside_permille) k += domain;
        keys[i] = (int32_t)k;
    }
}

const uint64_t kClassRows[kTuneClasses] = {1ull << 11, 1ull << 14, 1ull << 17, 1ull << 20, 1ull << 23, 1ull << 25};

struct Timer {
    Context &ctx;
    cudaEvent_t a, b;
    explicit Timer(Context &c) : ctx(c) {
        a = ctx.get_event();
        b = ctx.get_event();
    }
    ~Timer() {
        ctx.put_event(a);
        ctx.put_event(b);
    }
    /* median device time of `reps` runs of f, after one untimed run */
    template <class F> float median_ms(int reps, F f) {
        f();
        std::vector<float> t;
        for (int r = 0; r < reps; ++r) {
            check_cuda(cudaEventRecord(a, ctx.stream), "event record");
            f();
            check_cuda(cudaEventRecord(b, ctx.stream), "event record");
            check_cuda(cudaEventSynchronize(b), "event synchronize");
            float ms = 0;
            check_cuda(cudaEventElapsedTime(&ms, a, b), "event time");
            t.push_back(ms);
        }
        std::sort(t.begin(), t.end());
        return t[t.size() / 2];
    }
};

TuneEntry tune_class_entry(Context &ctx, int c) {
    const uint64_t nb = kClassRows[c];
    const uint64_t npr = std::min<uint64_t>(nb * 4, 1ull << 26);
    const uint32_t domain = (uint32_t)std::max<uint64_t>(nb * 3 / 4, 1);
    DevPtr bkeys = ctx.alloc(nb * 4), pkeys = ctx.alloc(npr * 4);
    DevPtr bvalid = ctx.alloc((nb + 31) / 32 * 4), pvalid = ctx.alloc((npr + 31) / 32 * 4);
    check_cuda(cudaMemsetAsync(bvalid->ptr, 0xFF, bvalid->bytes, ctx.stream), "memset");
    check_cuda(cudaMemsetAsync(pvalid->ptr, 0xFF, pvalid->bytes, ctx.stream), "memset");
    const unsigned g = (unsigned)std::min<uint64_t>((npr + 255) / 256, (uint64_t)ctx.num_sms * 8);
    k_tune_keys<<<g, 256, 0, ctx.stream>>>(bkeys->as<int32_t>(), nb, domain, 0x51u + c, 0);
    k_tune_keys<<<g, 256, 0, ctx.stream>>>(pkeys->as<int32_t>(), npr, domain, 0xA7u + c, 300);
    check_cuda(cudaGetLastError(), "k_tune_keys");
    ColView bk{}, pk{};
    bk.values = bkeys->ptr;
    bk.valid = bvalid->as<uint32_t>();
    bk.type = CJ_INT32;
    pk.values = pkeys->ptr;
    pk.valid = pvalid->as<uint32_t>();
    pk.type = CJ_INT32;

    const int log2_slots = std::max(11, ceil_log2(nb));
    DevPtr dir = ctx.alloc(build_dir_bytes(log2_slots, 4));
    DevPtr tuples = ctx.alloc(nb * build_tuple_bytes(4));
    Timer tm(ctx);
    TuneEntry best;
    float best_ms = 1e30f;
    for (int spp : {9, 10, 11, 12, 13}) {
        if (spp > log2_slots) continue;
        for (int pc : {2, 4, 8}) {
            BuildPlan bp;
            bp.num_rows = (uint32_t)nb;
            bp.log2_slots = log2_slots;
            bp.log2_parts = log2_slots - spp;
            Launch L = ctx.launch();
            L.part_ctas_per_sm = pc;
            DevPtr tmp = ctx.alloc(build_temp_bytes(L, bp, 4));
            const float ms = tm.median_ms(3, [&] {
                check_cuda(launch_build(L, bp, bk, ctx.d_bloom, dir->as<uint64_t>(), tuples->ptr, tmp->ptr), "build");
            });
            if (ms < best_ms) {
                best_ms = ms;
                best.log2_spp = spp;
                best.part_ctas = pc;
            }
        }
    }
    /* the table of the best build, then the probe's grid */
    BuildPlan bp;
    bp.num_rows = (uint32_t)nb;
    bp.log2_slots = log2_slots;
    bp.log2_parts = log2_slots - best.log2_spp;
    Launch LB = ctx.launch();
    LB.part_ctas_per_sm = best.part_ctas;
    {
        DevPtr tmp = ctx.alloc(build_temp_bytes(LB, bp, 4));
        check_cuda(launch_build(LB, bp, bk, ctx.d_bloom, dir->as<uint64_t>(), tuples->ptr, tmp->ptr), "build");
    }
    const uint64_t cap = npr * 2;
    DevPtr ob = ctx.alloc(cap * 4), op = ctx.alloc(cap * 4), sched = ctx.alloc(probe_sched_bytes((uint32_t)npr));
    DevPtr counter = ctx.alloc(8);
    MatchOut mo;
    mo.build_rids = ob->as<uint32_t>();
    mo.probe_rids = op->as<uint32_t>();
    mo.capacity = cap;
    mo.counter = counter->as<unsigned long long>();
    best_ms = 1e30f;
    for (int ctas : {2, 4, 6, 8}) {
        Launch L = ctx.launch();
        L.ctas_per_sm = ctas;
        const float ms = tm.median_ms(3, [&] {
            check_cuda(launch_probe_tiles_hash(L, pk, (uint32_t)npr, CJ_INT32, dir->as<uint64_t>(), tuples->ptr,
                                               log2_slots, ctx.d_bloom, mo, sched->ptr),
                       "probe");
        });
        if (ms < best_ms) {
            best_ms = ms;
            best.probe_ctas = ctas;
        }
    }
    check_cuda(cudaStreamSynchronize(ctx.stream), "stream synchronize");
    return best;
}

void save_tuning(const Context &ctx, const char *path) {
    FILE *f = std::fopen(path, "w");
    if (!f) fail(CJ_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
    std::fprintf(f, "cj_b200-tuning 1 %d\n", ctx.num_sms);
    for (int c = 0; c < kTuneClasses; ++c)
        std::fprintf(f, "class %d log2_spp %d part_ctas %d probe_ctas %d\n", c, ctx.tuning.cls[c].log2_spp,
                     ctx.tuning.cls[c].part_ctas, ctx.tuning.cls[c].probe_ctas);
    const bool bad = std::ferror(f) != 0;
    std::fclose(f);
    if (bad) fail(CJ_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
}

} // namespace

/* Parses a tuning file; entries out of range, or a file for another SM
 * count, are refused (CJ_ERR_INVALID_ARGUMENT). */
Tuning load_tuning_file(const char *path, int num_sms) {
    FILE *f = std::fopen(path, "r");
    if (!f) fail(CJ_ERR_INVALID_ARGUMENT, std::string("cannot read ") + path);
    Tuning t;
    int version = 0, sms = 0;
    char line[256];
    bool ok = std::fgets(line, sizeof line, f) && std::sscanf(line, "cj_b200-tuning %d %d", &version, &sms) == 2 &&
              version == 1;
    bool seen[kTuneClasses] = {};
    while (ok && std::fgets(line, sizeof line, f)) {
        int c, spp, pc, qc;
        if (std::sscanf(line, "class %d log2_spp %d part_ctas %d probe_ctas %d", &c, &spp, &pc, &qc) != 4) {
            ok = false;
            break;
        }
        if (c < 0 || c >= kTuneClasses || spp < 0 || spp > 14 || pc < 0 || pc > 32 || qc < 0 || qc > 32) {
            ok = false;
            break;
        }
        t.cls[c] = TuneEntry{spp, pc, qc};
        seen[c] = true;
    }
    std::fclose(f);
    for (bool s : seen) ok = ok && s;
    if (!ok) fail(CJ_ERR_INVALID_ARGUMENT, std::string("malformed tuning file ") + path);
    if (num_sms > 0 && sms != num_sms)
        fail(CJ_ERR_INVALID_ARGUMENT, std::string("tuning file ") + path + " is for a GPU with " + std::to_string(sms) +
                                          " SMs");
    t.loaded = true;
    return t;
}

} // namespace cj

extern "C" {

int cj_autotune(cj_context *ctx, const char *path, uint32_t flags) {
    if (!ctx) return cj::set_last_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(ctx->device);
    try {
        cj::Tuning t;
        const int classes = (flags & CJ_TUNE_QUICK) ? 4 : cj::kTuneClasses;
        for (int c = 0; c < cj::kTuneClasses; ++c) t.cls[c] = c < classes ? cj::tune_class_entry(*ctx, c) : t.cls[c];
        /* classes left untimed (quick mode) take the largest timed one's entry */
        for (int c = classes; c < cj::kTuneClasses; ++c) t.cls[c] = t.cls[classes - 1];
        t.loaded = true;
        ctx->tuning = t;
        if (path) cj::save_tuning(*ctx, path);
    } catch (const cj::Error &e) {
        cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();
        return cj::set_last_error(e.code, e.msg);
    }
    cj::clear_last_error();
    return CJ_OK;
}

int cj_tuning_load(cj_context *ctx, const char *path) {
    if (!ctx || !path) return cj::set_last_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    try {
        ctx->tuning = cj::load_tuning_file(path, ctx->num_sms);
    } catch (const cj::Error &e) {
        return cj::set_last_error(e.code, e.msg);
    }
    cj::clear_last_error();
    return CJ_OK;
}

int cj_tuning_check_file(const char *path) {
    if (!path) return cj::set_last_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    try {
        cj::load_tuning_file(path, 0);
    } catch (const cj::Error &e) {
        return cj::set_last_error(e.code, e.msg);
    }
    cj::clear_last_error();
    return CJ_OK;
}

int cj_tuning_entry(const cj_context *ctx, uint32_t size_class, int32_t *log2_spp, int32_t *part_ctas,
                    int32_t *probe_ctas) {
    if (!ctx || !log2_spp || !part_ctas || !probe_ctas || size_class >= (uint32_t)cj::kTuneClasses)
        return cj::set_last_error(CJ_ERR_INVALID_ARGUMENT, "bad argument");
    const cj::TuneEntry &e = ctx->tuning.cls[size_class];
    *log2_spp = e.log2_spp;
    *part_ctas = e.part_ctas;
    *probe_ctas = e.probe_ctas;
    return CJ_OK;
}

} // extern "C"
