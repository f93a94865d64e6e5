// serve.cpp — a request server over resident graphs with continuous batching.
//
// Requests (graph, query, count or first-k enumeration) are queued by
// beep_serve_submit. One scheduler thread admits them by free HBM, forms a
// batch from whatever has arrived, plans it as one multi-pair call and
// launches it on one of several streams without waiting; batches in flight
// overlap on the device, and requests that arrive meanwhile are admitted as
// soon as a stream and memory free up. A batch completes when its event
// fires; its requests get their counts (and tuples) and their latency from
// arrival to completion.
//
// The reference has no serving mode: it runs one SG_Match per query and
// graph (subgraph_matching.cuh:178-231) and keeps nothing resident.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "internal.h"

namespace beep {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    int32_t graph = 0;
    QueryPlan plan;
    uint64_t k = 0; // enumerate the first k matches (0: count only)
    Clock::time_point arrival, start, done;
    beep_status status = BEEP_OK;
    std::string error;
    uint64_t count = 0;
    uint64_t n_tuples = 0;
    std::vector<int32_t> tuples;
    bool finished = false;
};

// Grow-only pinned host buffer. Pinned allocation and release are slow and
// cudaFreeHost waits for the whole device, so a slot keeps its buffers from
// batch to batch and replaces them only to grow.
template <typename T> struct PinnedBuf {
    T *ptr = nullptr;
    size_t n = 0;
    cudaError_t reserve(size_t want) {
        if (want <= n)
            return cudaSuccess;
        if (ptr)
            cudaFreeHost(ptr);
        ptr = nullptr;
        n = 0;
        const size_t grow = std::max(want, (size_t)4096);
        cudaError_t e = cudaMallocHost(&ptr, grow * sizeof(T));
        if (e == cudaSuccess)
            n = grow;
        return e;
    }
    void release() {
        if (ptr)
            cudaFreeHost(ptr);
        ptr = nullptr;
        n = 0;
    }
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    // the slot's own side streams for the kernel tiers of its batch
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    bool busy = false;
    LaunchPlanPtr plan;
    std::vector<std::shared_ptr<Request>> reqs;
    std::vector<EnumRequest> enums;
    std::vector<void *> dbufs;     // device tuple buffers (pool)
    std::vector<size_t> hoff;      // each request's tuples in the staging buffer
    PinnedBuf<int32_t> tuples;     // pinned staging of the batch's tuples
    PinnedBuf<unsigned long long> counts; // pinned read-back of the batch's counts
    std::vector<PairSpec> specs;
    uint64_t reserved = 0;         // admission estimate of the batch in flight
};

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

} // namespace

struct Server {
    beep_ctx *uctx = nullptr;
    Ctx ctx; // planning resources; its stream is switched to the slot being planned
    std::vector<Graph *> graphs;
    std::vector<uint64_t> graph_large_bytes; // per graph: dense bitmaps of every root of degree > 1024
    std::vector<Slot> slots;
    uint32_t max_batch = 64;
    uint64_t reserve = 1ull << 30;
    uint64_t budget = 0;      // device bytes the admission may hand out: free HBM at creation - reserve
    uint64_t inflight = 0;    // estimates of the batches in flight
    uint64_t max_inflight = 0;
    uint64_t refused = 0;
    uint32_t count_options = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> pending;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> all;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread thr;
    // statistics
    std::vector<double> lat_ms;
    uint64_t batches = 0, matches = 0, completed = 0, launches = 0;
    Clock::time_point first_arrival, last_done;
    bool have_arrival = false;
    double max_batch_seen = 0;

    void loop();
    void launch(Slot &sl, std::vector<std::shared_ptr<Request>> &batch);
    void finish(Slot &sl, beep_status st, const std::string &err);
    // Device bytes a request can take while its batch runs: its tuple buffer,
    // the planning arrays over its graph's vertices and entries, and the
    // large tier's bitmap arena -- at most the dense bitmaps of all the
    // graph's roots of degree above 1024, and never more than the arena cap
    // that planning applies (min(48 GiB, half the free memory)).
    uint64_t estimate(const Request &r) const {
        const Graph *g = graphs[r.graph];
        const uint64_t arena = std::min<uint64_t>(graph_large_bytes[r.graph], std::min<uint64_t>(48ull << 30, budget / 2));
        return (uint64_t)r.k * (uint64_t)r.plan.info.K * 4ull + (uint64_t)g->n * 64ull + (uint64_t)g->m * 4ull +
               arena;
    }
};

void Server::finish(Slot &sl, beep_status st, const std::string &err_in) {
    const auto now = Clock::now();
    std::string err = err_in;
    if (st == BEEP_OK && sl.plan && (st = plan_status(sl.plan.get())) != BEEP_OK) {
        char buf[512];
        beep_last_error(buf, sizeof(buf));
        err = buf;
    }
    for (size_t i = 0; i < sl.reqs.size(); ++i) {
        Request &r = *sl.reqs[i];
        r.done = now;
        if (st != BEEP_OK) {
            r.status = st;
            r.error = err;
        } else {
            r.count = plan_count(sl.plan.get(), i);
            if (r.count == BEEP_COUNT_OVERFLOW) {
                r.status = BEEP_ERR_OVERFLOW;
                r.error = "the count is at least BEEP_COUNT_LIMIT (2^64 - 2^52)";
            } else if (r.k > 0) {
                r.n_tuples = std::min<uint64_t>(r.k, r.count);
                const int32_t *h = sl.tuples.ptr + sl.hoff[i];
                r.tuples.assign(h, h + r.n_tuples * (uint64_t)r.plan.info.K);
            }
            if (r.status == BEEP_OK)
                matches += r.count;
        }
        lat_ms.push_back(ms_between(r.arrival, r.done));
        r.finished = true;
        ++completed;
    }
    for (void *p : sl.dbufs)
        if (p)
            cudaFreeAsync(p, sl.stream);
    sl.dbufs.clear();
    sl.hoff.clear();
    inflight -= sl.reserved;
    sl.reserved = 0;
    sl.enums.clear();
    sl.specs.clear();
    sl.reqs.clear();
    sl.plan.reset();
    sl.busy = false;
    last_done = now;
}

void Server::launch(Slot &sl, std::vector<std::shared_ptr<Request>> &batch) {
    ctx.stream = sl.stream;
    ctx.side[0] = sl.side[0];
    ctx.side[1] = sl.side[1];
    ctx.ev_fork = sl.ev_fork;
    ctx.ev_join[0] = sl.ev_join[0];
    ctx.ev_join[1] = sl.ev_join[1];
    sl.reqs = batch;
    sl.enums.assign(batch.size(), EnumRequest{});
    sl.dbufs.assign(batch.size(), nullptr);
    sl.hoff.assign(batch.size(), 0);
    sl.specs.clear();
    beep_status st = BEEP_OK;
    std::string err;
    const auto start = Clock::now();
    // tuple staging: one pinned region per slot, each request at its offset
    size_t tuple_words = 0;
    for (size_t i = 0; i < batch.size(); ++i) {
        sl.hoff[i] = tuple_words;
        tuple_words += (size_t)batch[i]->k * (size_t)batch[i]->plan.info.K;
    }
    if (tuple_words) {
        cudaError_t e = sl.tuples.reserve(tuple_words);
        if (e != cudaSuccess) {
            st = BEEP_ERR_OUT_OF_MEMORY;
            err = std::string("tuple staging: ") + cudaGetErrorString(e);
        }
    }
    for (size_t i = 0; i < batch.size() && st == BEEP_OK; ++i) {
        Request &r = *batch[i];
        r.start = start;
        PairSpec ps;
        ps.g = graphs[r.graph];
        ps.plan = r.plan;
        if (r.k > 0) {
            const size_t bytes = (size_t)r.k * (size_t)r.plan.info.K * 4;
            cudaError_t e = cudaMallocFromPoolAsync(&sl.dbufs[i], bytes, ctx.pool, sl.stream);
            if (e != cudaSuccess) {
                st = BEEP_ERR_OUT_OF_MEMORY;
                err = std::string("tuple buffers: ") + cudaGetErrorString(e);
                break;
            }
            sl.enums[i].k = r.k;
            sl.enums[i].d_out = static_cast<int32_t *>(sl.dbufs[i]);
        }
        sl.specs.push_back(ps);
    }
    // spec i counts request i (closed forms allowed); a first-k request also
    // gets an enumerating spec after them, whose walk stops at k tuples
    const size_t ncount = sl.specs.size();
    for (size_t i = 0; i < ncount; ++i)
        if (batch[i]->k > 0) {
            PairSpec es = sl.specs[i];
            es.en = &sl.enums[i];
            sl.specs.push_back(es);
        }
    if (st == BEEP_OK)
        st = plan_pairs(&ctx, sl.specs, count_options, &sl.plan);
    if (st == BEEP_OK && sl.counts.reserve(plan_host_words(sl.plan.get())) != cudaSuccess) {
        st = BEEP_ERR_OUT_OF_MEMORY;
        err = "pinned read-back buffer";
    }
    if (st == BEEP_OK)
        st = launch_plan_async(&ctx, sl.plan.get(), sl.counts.ptr);
    if (st == BEEP_OK) {
        for (size_t i = 0; i < batch.size(); ++i)
            if (batch[i]->k > 0) {
                cudaError_t e = cudaMemcpyAsync(sl.tuples.ptr + sl.hoff[i], sl.dbufs[i],
                                                (size_t)batch[i]->k * (size_t)batch[i]->plan.info.K * 4,
                                                cudaMemcpyDeviceToHost, sl.stream);
                if (e != cudaSuccess) {
                    st = BEEP_ERR_CUDA;
                    err = cudaGetErrorString(e);
                }
            }
        cudaEventRecord(sl.done, sl.stream);
        launches += (uint64_t)plan_launches(sl.plan.get());
    }
    if (st != BEEP_OK && err.empty()) {
        char buf[512];
        beep_last_error(buf, sizeof(buf));
        err = buf;
    }
    sl.busy = true;
    ++batches;
    max_batch_seen = std::max(max_batch_seen, (double)batch.size());
    if (st != BEEP_OK) {
        cudaStreamSynchronize(sl.stream);
        std::lock_guard<std::mutex> lk(mu);
        finish(sl, st, err);
        cv_done.notify_all();
    }
}

void Server::loop() {
    cudaSetDevice(ctx.device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        bool progressed = false;
        // completed batches
        for (auto &sl : slots) {
            if (!sl.busy)
                continue;
            cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaSuccess) {
                finish(sl, BEEP_OK, "");
                progressed = true;
            } else if (q != cudaErrorNotReady) {
                finish(sl, BEEP_ERR_CUDA, cudaGetErrorString(q));
                progressed = true;
            }
        }
        if (progressed)
            cv_done.notify_all();
        // new batches: a free stream, pending requests and the memory to run
        // them. A request whose estimate exceeds the whole budget can never
        // run and is refused; one that does not fit beside the batches in
        // flight waits for them (back-pressure), and so do the requests
        // behind it (arrival order is kept).
        for (auto &sl : slots) {
            if (sl.busy || pending.empty())
                continue;
            std::vector<std::shared_ptr<Request>> batch;
            uint64_t need = 0;
            while (!pending.empty() && batch.size() < max_batch) {
                std::shared_ptr<Request> r = pending.front();
                const uint64_t e = estimate(*r);
                if (e > budget) {
                    pending.pop_front();
                    r->status = BEEP_ERR_OUT_OF_MEMORY;
                    r->error = "request needs an estimated " + std::to_string(e) + " device bytes, more than the " +
                               std::to_string(budget) + " the server may use (free HBM at creation minus the reserve)";
                    r->start = r->done = Clock::now();
                    r->finished = true;
                    ++refused;
                    progressed = true;
                    continue;
                }
                if (inflight + need + e > budget)
                    break;
                need += e;
                batch.push_back(r);
                pending.pop_front();
            }
            if (progressed)
                cv_done.notify_all();
            if (batch.empty())
                continue;
            sl.reserved = need;
            inflight += need;
            max_inflight = std::max(max_inflight, inflight);
            lk.unlock();
            launch(sl, batch);
            lk.lock();
            progressed = true;
        }
        bool busy = false;
        for (auto &sl : slots)
            busy |= sl.busy;
        if (stop && pending.empty() && !busy)
            break;
        if (!progressed) {
            if (busy)
                cv_work.wait_for(lk, std::chrono::microseconds(50));
            else
                cv_work.wait(lk, [&] { return stop || !pending.empty(); });
        }
    }
}

} // namespace beep

struct beep_server {
    beep::Server impl;
};

using namespace beep;

extern "C" {

beep_status beep_serve_create(beep_ctx *ctx, const beep_serve_options *opt, beep_server **out) {
    if (!ctx || !out)
        return fail(BEEP_ERR_INVALID_ARG, "beep_serve_create: bad arguments");
    *out = nullptr;
    BEEP_CUDA_TRY(cudaSetDevice(ctx->impl.device));
    auto *s = new beep_server;
    Server &S = s->impl;
    S.uctx = ctx;
    ctx->refs.fetch_add(1);
    S.ctx.device = ctx->impl.device;
    S.ctx.num_sms = ctx->impl.num_sms;
    S.ctx.smem_optin = ctx->impl.smem_optin;
    uint32_t nstreams = 4;
    if (opt) {
        if (opt->max_batch)
            S.max_batch = opt->max_batch;
        if (opt->streams)
            nstreams = opt->streams;
        if (opt->hbm_reserve_bytes)
            S.reserve = opt->hbm_reserve_bytes;
        S.count_options = opt->count_options & BEEP_OPT_REFERENCE_ROOT_CAP;
    }
    cudaError_t e = cudaMallocHost(&S.ctx.h_pinned, 64);
    // buffers come from the user context's pool (the server holds a
    // reference to that context, so the pool outlives everything built here,
    // including the views it caches in the graphs)
    S.ctx.pool = ctx->impl.pool;
    S.slots.resize(nstreams);
    for (auto &sl : S.slots) {
        if (e == cudaSuccess)
            e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
            e = cudaStreamCreateWithFlags(&sl.side[i], cudaStreamNonBlocking);
            if (e == cudaSuccess)
                e = cudaEventCreateWithFlags(&sl.ev_join[i], cudaEventDisableTiming);
        }
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&sl.ev_fork, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        beep_serve_destroy(s);
        return fail(BEEP_ERR_CUDA, std::string("server setup: ") + cudaGetErrorString(e));
    }
    S.ctx.stream = S.slots[0].stream;
    {
        size_t free_b = 0, total_b = 0;
        e = cudaMemGetInfo(&free_b, &total_b);
        if (e != cudaSuccess) {
            beep_serve_destroy(s);
            return fail(BEEP_ERR_CUDA, std::string("server setup: ") + cudaGetErrorString(e));
        }
        S.budget = free_b > S.reserve ? free_b - S.reserve : 0;
    }
    S.thr = std::thread([&S] { S.loop(); });
    *out = s;
    return BEEP_OK;
}

beep_status beep_serve_add_graph(beep_server *s, beep_graph *g, int32_t *graph_id) {
    if (!s || !g || !graph_id)
        return fail(BEEP_ERR_INVALID_ARG, "beep_serve_add_graph: bad arguments");
    if (g->impl.device != s->impl.ctx.device)
        return fail(BEEP_ERR_INVALID_ARG, "graph lives on another device");
    // the large tier's bitmap bound of this graph: rows of ceil(D / 32) words
    // for every root of degree D > 1024, plus their non-zero-word lists
    std::vector<uint32_t> rp((size_t)g->impl.n + 1);
    BEEP_CUDA_TRY(cudaSetDevice(g->impl.device));
    BEEP_CUDA_TRY(cudaMemcpy(rp.data(), g->impl.row_ptr.ptr, rp.size() * 4, cudaMemcpyDeviceToHost));
    uint64_t large = 0;
    for (size_t v = 0; v + 1 < rp.size(); ++v) {
        const uint64_t d = rp[v + 1] - rp[v];
        if (d > 1024)
            large += d * ((d + 31) / 32) * 4 + d * ((d + 31) / 32) / 2;
    }
    std::lock_guard<std::mutex> lk(s->impl.mu);
    s->impl.graphs.push_back(&g->impl);
    s->impl.graph_large_bytes.push_back(large);
    *graph_id = (int32_t)(s->impl.graphs.size() - 1);
    return BEEP_OK;
}

beep_status beep_serve_submit(beep_server *s, int32_t graph_id, const beep_query *q, beep_mode mode, uint64_t k,
                              uint64_t *request_id) {
    if (!s || !q || !request_id)
        return fail(BEEP_ERR_INVALID_ARG, "beep_serve_submit: bad arguments");
    if (mode != BEEP_MODE_SGM && mode != BEEP_MODE_SGC)
        return fail(BEEP_ERR_INVALID_ARG, "unknown mode");
    auto r = std::make_shared<Request>();
    r->arrival = Clock::now();
    BEEP_TRY(compile_plan(q->impl.qn, q->impl.row_ptr, q->impl.col, k > 0 ? BEEP_MODE_SGM : mode, &r->plan));
    r->k = k;
    r->graph = graph_id;
    {
        std::lock_guard<std::mutex> lk(s->impl.mu);
        if (graph_id < 0 || (size_t)graph_id >= s->impl.graphs.size())
            return fail(BEEP_ERR_INVALID_ARG, "unknown graph id");
        r->id = s->impl.next_id++;
        if (!s->impl.have_arrival) {
            s->impl.first_arrival = r->arrival;
            s->impl.have_arrival = true;
        }
        s->impl.pending.push_back(r);
        s->impl.all[r->id] = r;
        *request_id = r->id;
    }
    s->impl.cv_work.notify_one();
    return BEEP_OK;
}

beep_status beep_serve_wait(beep_server *s, uint64_t request_id, beep_serve_result *res, int32_t *tuples,
                            uint64_t tuples_cap) {
    if (!s || !res)
        return fail(BEEP_ERR_INVALID_ARG, "beep_serve_wait: bad arguments");
    std::unique_lock<std::mutex> lk(s->impl.mu);
    auto it = s->impl.all.find(request_id);
    if (it == s->impl.all.end())
        return fail(BEEP_ERR_INVALID_ARG, "unknown request id");
    std::shared_ptr<Request> r = it->second;
    s->impl.cv_done.wait(lk, [&] { return r->finished; });
    s->impl.all.erase(it);
    std::memset(res, 0, sizeof(*res));
    res->status = r->status;
    res->count = r->count;
    res->K = r->plan.info.K;
    res->n_tuples = r->n_tuples;
    res->latency_ms = ms_between(r->arrival, r->done);
    res->queue_ms = ms_between(r->arrival, r->start);
    if (tuples && r->n_tuples) {
        const uint64_t n = std::min<uint64_t>(r->n_tuples, tuples_cap);
        std::memcpy(tuples, r->tuples.data(), n * (uint64_t)res->K * 4);
        res->n_tuples = n;
    }
    if (r->status != BEEP_OK)
        return fail(r->status, r->error);
    return BEEP_OK;
}

beep_status beep_serve_drain(beep_server *s) {
    if (!s)
        return fail(BEEP_ERR_INVALID_ARG, "beep_serve_drain: null server");
    std::unique_lock<std::mutex> lk(s->impl.mu);
    s->impl.cv_done.wait(lk, [&] {
        bool busy = false;
        for (auto &sl : s->impl.slots)
            busy |= sl.busy;
        return s->impl.pending.empty() && !busy;
    });
    return BEEP_OK;
}

beep_status beep_serve_stats_get(beep_server *s, beep_serve_stats *out) {
    if (!s || !out)
        return fail(BEEP_ERR_INVALID_ARG, "beep_serve_stats_get: bad arguments");
    std::lock_guard<std::mutex> lk(s->impl.mu);
    std::memset(out, 0, sizeof(*out));
    Server &S = s->impl;
    out->requests = S.completed;
    out->batches = S.batches;
    out->matches = S.matches;
    out->kernel_launches = S.launches;
    out->max_batch = S.max_batch_seen;
    out->refused = S.refused;
    out->max_inflight_bytes = S.max_inflight;
    out->budget_bytes = S.budget;
    if (!S.lat_ms.empty()) {
        std::vector<double> v = S.lat_ms;
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) { return v[std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5))]; };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        out->max_ms = v.back();
        double sum = 0;
        for (double x : v)
            sum += x;
        out->mean_ms = sum / (double)v.size();
    }
    if (S.have_arrival && S.completed)
        out->span_s = std::chrono::duration<double>(S.last_done - S.first_arrival).count();
    return BEEP_OK;
}

beep_status beep_serve_destroy(beep_server *s) {
    if (!s)
        return BEEP_OK;
    Server &S = s->impl;
    {
        std::lock_guard<std::mutex> lk(S.mu);
        S.stop = true;
    }
    S.cv_work.notify_all();
    if (S.thr.joinable())
        S.thr.join();
    cudaSetDevice(S.ctx.device);
    for (auto &sl : S.slots) {
        if (sl.stream)
            cudaStreamSynchronize(sl.stream);
        sl.plan.reset();
        sl.tuples.release();
        sl.counts.release();
        if (sl.done)
            cudaEventDestroy(sl.done);
    }
    S.ctx.stream = nullptr;
    S.ctx.scratch.release();
    S.ctx.scratch2.release();
    S.ctx.arena.release();
    S.ctx.counter.release();
    if (S.ctx.h_pinned)
        cudaFreeHost(S.ctx.h_pinned);
    if (S.ctx.h_results)
        cudaFreeHost(S.ctx.h_results);
    // the context only borrowed the slots' side streams
    S.ctx.side[0] = S.ctx.side[1] = nullptr;
    S.ctx.ev_fork = S.ctx.ev_join[0] = S.ctx.ev_join[1] = nullptr;
    for (auto &sl : S.slots) {
        for (int i = 0; i < 2; ++i) {
            if (sl.side[i]) {
                cudaStreamSynchronize(sl.side[i]);
                cudaStreamDestroy(sl.side[i]);
            }
            if (sl.ev_join[i])
                cudaEventDestroy(sl.ev_join[i]);
        }
        if (sl.ev_fork)
            cudaEventDestroy(sl.ev_fork);
    }
    S.ctx.pool = nullptr; // borrowed
    for (auto &sl : S.slots)
        if (sl.stream)
            cudaStreamDestroy(sl.stream);
    beep_ctx *uctx = S.uctx;
    delete s;
    beep_ctx_destroy(uctx);
    return BEEP_OK;
}

} // extern "C"
