/*
 * server.cpp — serving: plans submitted as they arrive run concurrently on
 * one GPU (no reference counterpart; the reference runs one plan per
 * execute() call).
 *
 * A server owns `slots` worker threads, each with its own context (CUDA
 * stream, status block, staging) and all allocating from one shared,
 * stream-ordered memory pool. Requests queue in arrival order. A worker
 * that frees up admits queued plans whose estimated device footprint fits
 * in the memory budget next to the plans already running, and runs them
 * together (continuous batching):
 *   - up to max_batch plans per admission, and no more than an even share of
 *     the queue per idle worker, so that a short queue spreads over the
 *     workers and a long one is taken in batches;
 *   - one plan runs through the one-plan executor; several run as one
 *     grouped execution (execute_batch: every phase of a plan level is one
 *     launch over all of them), whose results equal each plan run alone;
 *   - admission goes in arrival order, but a plan that does not fit may be
 *     passed over by later ones that do until it has waited age_limit_us;
 *     after that nothing passes it, so it cannot starve.
 * Work of different workers overlaps on the device through their streams,
 * while the sum of the running plans' estimates stays within the budget. A
 * plan whose estimate alone exceeds the budget is rejected at submission
 * (CJ_ERR_REJECTED). Latency is measured from submission to completion.
 */
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace {

double now_us() {
    return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

uint64_t col_bytes_per_row(int32_t t) {
    switch (t) {
    case CJ_INT32: return 4;
    case CJ_VARCHAR: return 8;
    default: return 8;
    }
}

struct Est {
    uint64_t rows;
    uint64_t cols;
};

/* Upper-bound style footprint of a plan: uploaded pages, decoded columns,
 * per join the hash structures, match arrays and row-id vectors (join
 * output rows estimated as the larger input, the foreign-key case), and the
 * output pages. */
uint64_t estimate_bytes(const cj_plan_desc &p) {
    uint64_t bytes = 0;
    for (uint64_t t = 0; t < p.num_inputs; ++t) {
        const bool resident = p.resident_inputs && p.resident_inputs[t];
        if (resident || !p.inputs) continue;
        const cj_table_desc &td = p.inputs[t];
        for (uint64_t c = 0; c < td.num_columns; ++c) {
            bytes += td.columns[c].num_pages * CJ_PAGE_SIZE;
            bytes += td.num_rows * col_bytes_per_row(td.columns[c].type) + td.num_rows / 8 + 16 * td.columns[c].num_pages;
        }
    }
    std::vector<Est> memo(p.num_nodes, Est{0, 0});
    std::vector<int> state(p.num_nodes, 0);
    /* iterative post-order over the plan DAG */
    std::vector<uint64_t> stack{p.root};
    while (!stack.empty()) {
        uint64_t n = stack.back();
        if (n >= p.num_nodes) return UINT64_MAX;
        const cj_plan_node &node = p.nodes[n];
        if (state[n] == 2) {
            stack.pop_back();
            continue;
        }
        if (node.node_type == CJ_NODE_SCAN) {
            uint64_t rows = 0;
            if (node.base_table_id < p.num_inputs) {
                if (p.resident_inputs && p.resident_inputs[node.base_table_id])
                    rows = p.resident_inputs[node.base_table_id]->num_rows;
                else if (p.inputs)
                    rows = p.inputs[node.base_table_id].num_rows;
            }
            memo[n] = {rows, node.num_output_attrs};
            state[n] = 2;
            stack.pop_back();
            continue;
        }
        if (state[n] == 0) {
            state[n] = 1;
            stack.push_back(node.left);
            stack.push_back(node.right);
            continue;
        }
        const Est &l = memo[node.left], &r = memo[node.right];
        const uint64_t b = std::min(l.rows, r.rows), pr = std::max(l.rows, r.rows);
        uint64_t slots = 2048;
        while (slots < b) slots <<= 1;
        bytes += slots * 8 + b * 32 + pr * 8 + pr * 4 * node.num_output_attrs;
        memo[n] = {pr, node.num_output_attrs};
        state[n] = 2;
        stack.pop_back();
    }
    const cj_plan_node &root = p.nodes[p.root];
    bytes += memo[p.root].rows * 9 * root.num_output_attrs + (64u << 20);
    return bytes;
}

} // namespace

struct cj_server {
    int device = 0;
    cudaMemPool_t pool = nullptr;
    uint64_t budget = 0;
    uint32_t flags = 0;
    uint32_t max_batch = 32;
    double age_limit_us = 20000;
    std::vector<std::unique_ptr<cj::Context>> workers;
    std::vector<std::thread> threads;

    struct Req {
        const cj_plan_desc *plan = nullptr;
        uint64_t est = 0;
        int status = CJ_OK;
        std::string err;
        cj_result *res = nullptr;
        cj_exec_stats stats{};
        double t_submit = 0, t_start = 0, t_done = 0;
        bool started = false, done = false, collected = false;
    };
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, Req> reqs;
    uint64_t next_ticket = 1;
    uint64_t admitted = 0, peak_admitted = 0;
    uint32_t running = 0;      /* plans running                       */
    uint32_t busy_workers = 0; /* workers running a plan or a batch   */
    uint64_t batches = 0, batched_plans = 0, skipped_ahead = 0, batch_fallbacks = 0;
    std::shared_ptr<cj::PinnedPool> pinned; /* the workers' shared result blocks */
    uint64_t pinned_allocs0 = 0, pinned_bytes0 = 0;
    bool stop = false;
    /* statistics */
    uint64_t submitted = 0, completed = 0, failed = 0, rejected = 0, cancelled = 0;
    std::vector<double> latencies;
    double t_first = 0, t_last = 0;

    /* Takes the plans this worker runs next (lock held): queued plans that
     * fit in the budget, in arrival order, passing over one that does not
     * fit unless it has waited past the age limit. */
    bool take(std::vector<uint64_t> &out) {
        if (queue.empty()) return false;
        const double now = now_us();
        const size_t idle = std::max<size_t>(1, workers.size() - busy_workers);
        const size_t share = (queue.size() + idle - 1) / idle;
        const size_t limit = std::max<size_t>(1, std::min<size_t>(max_batch, share));
        uint64_t room = budget > admitted ? budget - admitted : 0;
        bool passed = false;
        for (auto it = queue.begin(); it != queue.end() && out.size() < limit;) {
            Req &r = reqs[*it];
            if (r.est <= room) {
                if (passed) ++skipped_ahead;
                out.push_back(*it);
                room -= r.est;
                it = queue.erase(it);
                continue;
            }
            if (now - r.t_submit > age_limit_us) break; /* aged: it goes first */
            passed = true;
            ++it;
        }
        return !out.empty();
    }

    void finish(uint64_t ticket, int status, const std::string &err, cj_result *res, const cj_exec_stats &st) {
        Req &r = reqs[ticket];
        r.status = status;
        r.err = err;
        r.res = res;
        r.stats = st;
        r.done = true;
        r.t_done = now_us();
        admitted -= r.est;
        --running;
        if (status == CJ_OK) {
            ++completed;
            latencies.push_back(r.t_done - r.t_submit);
        } else {
            ++failed;
        }
        t_last = r.t_done;
    }

    /* One plan through the one-plan executor; the status and message of a
     * failure, the context left usable. */
    static int run_one(cj::Context &ctx, const cj_plan_desc &plan, uint32_t flags, cj_result **res,
                       cj_exec_stats *st, std::string &err) {
        try {
            *res = cj::execute_plan(ctx, plan, flags, st);
            return CJ_OK;
        } catch (const cj::Error &e) {
            err = e.msg;
            cudaStreamSynchronize(ctx.stream);
            cudaGetLastError();
            return e.code;
        } catch (const std::bad_alloc &) {
            err = "host allocation failed";
            return CJ_ERR_OUT_OF_MEMORY;
        } catch (...) {
            err = "unexpected exception";
            return CJ_ERR_INTERNAL;
        }
    }

    void worker(size_t w) {
        cj::Context &ctx = *workers[w];
        cudaSetDevice(device);
        for (;;) {
            std::vector<uint64_t> tickets;
            std::vector<cj_plan_desc> plans;
            {
                std::unique_lock<std::mutex> lk(mu);
                /* wake on new work, on freed budget, and at least every
                 * millisecond so that ageing takes effect */
                while (!stop && !take(tickets)) cv_work.wait_for(lk, std::chrono::milliseconds(1));
                if (stop) return;
                ++busy_workers;
                ++batches;
                batched_plans += tickets.size();
                for (uint64_t t : tickets) {
                    Req &r = reqs[t];
                    r.started = true;
                    r.t_start = now_us();
                    admitted += r.est;
                    ++running;
                    plans.push_back(*r.plan);
                }
                peak_admitted = std::max(peak_admitted, admitted);
            }
            const size_t n = tickets.size();
            std::vector<cj_result *> res(n, nullptr);
            std::vector<int> status(n, CJ_OK);
            std::vector<std::string> err(n);
            std::vector<cj_exec_stats> st(n, cj_exec_stats{});
            bool done = false;
            if (n > 1) {
                /* one grouped execution; if it fails as a whole (a device
                 * error, memory), each plan runs alone so that one plan's
                 * failure is not every plan's */
                std::vector<int32_t> sts(n, CJ_OK);
                cj_batch_stats bst{};
                try {
                    cj::execute_batch(ctx, plans.data(), n, flags, res.data(), sts.data(), &bst);
                    for (size_t i = 0; i < n; ++i) {
                        status[i] = sts[i];
                        if (sts[i] != CJ_OK) err[i] = "plan failed validation";
                        st[i].total_us = bst.total_us;
                        st[i].kernel_launches = bst.kernel_launches;
                    }
                    done = true;
                } catch (...) {
                    for (auto &r : res) {
                        if (r) cj_result_free(r);
                        r = nullptr;
                    }
                    cudaStreamSynchronize(ctx.stream);
                    cudaGetLastError();
                    std::lock_guard<std::mutex> lk(mu);
                    ++batch_fallbacks;
                }
            }
            if (!done)
                for (size_t i = 0; i < n; ++i) status[i] = run_one(ctx, plans[i], flags, &res[i], &st[i], err[i]);
            {
                std::lock_guard<std::mutex> lk(mu);
                for (size_t i = 0; i < n; ++i) finish(tickets[i], status[i], err[i], res[i], st[i]);
                --busy_workers;
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }
};

namespace {
int serr(int code, const std::string &m) { return cj::set_last_error(code, m); }
} // namespace

extern "C" {

int cj_server_estimate(const cj_plan_desc *plan, uint64_t *bytes) {
    if (!plan || !bytes || !plan->nodes || plan->root >= plan->num_nodes)
        return serr(CJ_ERR_INVALID_ARGUMENT, "bad plan");
    *bytes = estimate_bytes(*plan);
    return CJ_OK;
}

int cj_server_create(const cj_server_config *cfg, cj_server **out) {
    if (!cfg || !out) return serr(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    auto s = std::make_unique<cj_server>();
    try {
        int dev = cfg->device;
        if (dev < 0) cj::check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        cj::check_cuda(cudaSetDevice(dev), "cudaSetDevice");
        s->device = dev;
        s->pool = cj::create_pool(dev);
        s->flags = cfg->exec_flags;
        s->max_batch = cfg->max_batch ? cfg->max_batch : 32;
        s->age_limit_us = cfg->age_limit_us ? (double)cfg->age_limit_us : 20000.0;
        size_t free_b = 0, total_b = 0;
        cj::check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
        s->budget = cfg->memory_budget ? cfg->memory_budget : (uint64_t)(free_b * 0.85);
        const uint32_t slots = cfg->slots ? cfg->slots : 4;
        s->pinned = std::make_shared<cj::PinnedPool>(); /* one cache of result blocks for all workers */
        if (cfg->host_cache_bytes) s->pinned->reserve(cfg->host_cache_bytes);
        for (uint32_t w = 0; w < slots; ++w) s->workers.emplace_back(cj::create_context(dev, s->pool, s->pinned));
        if (cfg->device_reserve_bytes) {
            /* one block of the requested size, freed at once: the pool keeps
             * the memory (release threshold = keep) and later allocations are
             * carved from it */
            const cudaStream_t st = s->workers[0]->stream;
            void *p = nullptr;
            cudaError_t e = cudaMallocFromPoolAsync(&p, cfg->device_reserve_bytes, s->pool, st);
            if (e != cudaSuccess) {
                cudaGetLastError();
                cj::fail(CJ_ERR_OUT_OF_MEMORY,
                         "device reserve of " + std::to_string(cfg->device_reserve_bytes) + " bytes failed");
            }
            cj::check_cuda(cudaFreeAsync(p, st), "cudaFreeAsync");
            cj::check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        }
    } catch (const cj::Error &e) {
        for (auto &w : s->workers) w.reset();
        if (s->pool) cudaMemPoolDestroy(s->pool);
        return serr(e.code, e.msg);
    }
    for (size_t w = 0; w < s->workers.size(); ++w) s->threads.emplace_back(&cj_server::worker, s.get(), w);
    *out = s.release();
    return CJ_OK;
}

int cj_server_submit(cj_server *s, const cj_plan_desc *plan, uint64_t *ticket) {
    if (!s || !plan || !ticket) return serr(CJ_ERR_INVALID_ARGUMENT, "null argument");
    if (!plan->nodes || plan->root >= plan->num_nodes) return serr(CJ_ERR_INVALID_PLAN, "bad plan");
    const uint64_t est = estimate_bytes(*plan);
    cj::clear_last_error();
    std::lock_guard<std::mutex> lk(s->mu);
    ++s->submitted;
    if (est > s->budget) {
        ++s->rejected;
        return serr(CJ_ERR_REJECTED, "estimated footprint " + std::to_string(est) + " bytes exceeds the budget");
    }
    const uint64_t t = s->next_ticket++;
    cj_server::Req &r = s->reqs[t];
    r.plan = plan;
    r.est = est;
    r.t_submit = now_us();
    if (s->t_first == 0) s->t_first = r.t_submit;
    s->queue.push_back(t);
    *ticket = t;
    s->cv_work.notify_one();
    return CJ_OK;
}

int cj_server_wait(cj_server *s, uint64_t ticket, int64_t timeout_us, cj_result **out, cj_exec_stats *stats) {
    if (!s || !out) return serr(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end() || it->second.collected) return serr(CJ_ERR_INVALID_ARGUMENT, "unknown ticket");
    auto pred = [&] { return s->reqs[ticket].done; };
    if (timeout_us < 0) {
        s->cv_done.wait(lk, pred);
    } else if (!s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), pred)) {
        return serr(CJ_ERR_TIMEOUT, "plan still running");
    }
    cj_server::Req r = s->reqs[ticket];
    s->reqs.erase(ticket);
    if (stats) *stats = r.stats;
    *out = r.res;
    if (r.status != CJ_OK) return serr(r.status, r.err);
    return CJ_OK;
}

int cj_server_cancel(cj_server *s, uint64_t ticket) {
    if (!s) return serr(CJ_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return serr(CJ_ERR_INVALID_ARGUMENT, "unknown ticket");
    if (it->second.started) return serr(CJ_ERR_INVALID_ARGUMENT, "plan already running");
    s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), ticket), s->queue.end());
    it->second.done = true;
    it->second.status = CJ_ERR_CANCELLED;
    it->second.err = "cancelled";
    ++s->cancelled;
    s->cv_done.notify_all();
    s->cv_work.notify_all();
    return CJ_OK;
}

int cj_server_get_stats(cj_server *s, cj_server_stats *out, int reset) {
    if (!s || !out) return serr(CJ_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    cj_server_stats st{};
    st.submitted = s->submitted;
    st.completed = s->completed;
    st.failed = s->failed;
    st.rejected = s->rejected;
    st.cancelled = s->cancelled;
    st.queued = s->queue.size();
    st.running = s->running;
    st.admitted_bytes = s->admitted;
    st.peak_admitted_bytes = s->peak_admitted;
    st.memory_budget = s->budget;
    std::vector<double> l = s->latencies;
    std::sort(l.begin(), l.end());
    if (!l.empty()) {
        auto pct = [&](double q) { return l[std::min(l.size() - 1, (size_t)(q * (l.size() - 1) + 0.5))]; };
        st.p50_us = pct(0.50);
        st.p99_us = pct(0.99);
        st.max_us = l.back();
        double sum = 0;
        for (double x : l) sum += x;
        st.mean_us = sum / l.size();
    }
    st.wall_s = s->t_last > s->t_first ? (s->t_last - s->t_first) / 1e6 : 0;
    st.plans_per_s = st.wall_s > 0 ? s->completed / st.wall_s : 0;
    st.batches = s->batches;
    st.skipped_ahead = s->skipped_ahead;
    st.mean_batch = s->batches ? (double)s->batched_plans / s->batches : 0;
    st.batch_fallbacks = s->batch_fallbacks;
    const cj::PinnedPool &pp = *s->pinned;
    st.pinned_allocs = pp.host_allocs.load() - s->pinned_allocs0;
    st.pinned_alloc_bytes = pp.host_alloc_bytes.load() - s->pinned_bytes0;
    uint64_t high = 0; /* the attribute is a 64-bit unsigned value */
    if (cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReservedMemHigh, &high) != cudaSuccess) cudaGetLastError();
    st.pool_high_bytes = high;
    *out = st;
    if (reset) {
        s->pinned_allocs0 = pp.host_allocs.load();
        uint64_t zero = 0; /* restarts the pool's high-water mark */
        if (cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReservedMemHigh, &zero) != cudaSuccess) cudaGetLastError();
        s->pinned_bytes0 = pp.host_alloc_bytes.load();
        s->latencies.clear();
        s->completed = s->failed = s->rejected = s->cancelled = s->submitted = 0;
        s->batches = s->batched_plans = s->skipped_ahead = s->batch_fallbacks = 0;
        s->t_first = s->t_last = 0;
        s->peak_admitted = s->admitted;
    }
    return CJ_OK;
}

void cj_server_destroy(cj_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->threads) t.join();
    cudaSetDevice(s->device);
    for (auto &kv : s->reqs)
        if (kv.second.res) cj_result_free(kv.second.res);
    s->workers.clear();
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
}

} /* extern "C" */
