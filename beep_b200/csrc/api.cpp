// api.cpp — the C ABI (include/beep.h) over the device graph build and the
// counting kernels.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>

#include "internal.h"

namespace beep {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string &msg) { g_last_error = msg; }

beep_status fail(beep_status s, const std::string &msg) {
    set_error(msg);
    return s;
}

namespace {

// BEEP_ERR_OVERFLOW when a single-pair call's count reached BEEP_COUNT_LIMIT.
beep_status overflow_status(const beep_stats &st) {
    if (st.count != BEEP_COUNT_OVERFLOW)
        return BEEP_OK;
    return fail(BEEP_ERR_OVERFLOW, "the count is at least BEEP_COUNT_LIMIT (2^64 - 2^52) and is not representable "
                                   "as an exact u64");
}

beep_status bind(beep_ctx *ctx) {
    if (!ctx)
        return fail(BEEP_ERR_INVALID_ARG, "null context");
    BEEP_CUDA_TRY(cudaSetDevice(ctx->impl.device));
    return BEEP_OK;
}

// Copy a host array to a device buffer through the context's stream.
template <typename T> beep_status upload(Ctx *ctx, DevBuf &dst, const T *src, size_t count) {
    BEEP_TRY(ctx->grow(dst, std::max<size_t>(count, 1) * sizeof(T)));
    if (count)
        BEEP_CUDA_TRY(cudaMemcpyAsync(dst.ptr, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return BEEP_OK;
}

} // namespace
} // namespace beep

namespace beep {
namespace {
double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
} // namespace

bool trace_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("BEEP_TRACE");
        return e && *e && *e != '0';
    }();
    return on;
}

PhaseTrace::PhaseTrace(const char *scope_, cudaStream_t s) : scope(scope_), stream(s), t0(0) {
    if (trace_enabled()) {
        cudaStreamSynchronize(stream);
        t0 = now_ms();
    }
}

void PhaseTrace::mark(const char *phase) {
    if (!trace_enabled())
        return;
    cudaStreamSynchronize(stream);
    const double t = now_ms();
    std::fprintf(stderr, "beep-trace %s.%s %.3f ms\n", scope, phase, t - t0);
    t0 = t;
}
} // namespace beep

using namespace beep;

extern "C" {

size_t beep_last_error(char *buf, size_t len) {
    const std::string &e = g_last_error;
    if (buf && len) {
        size_t n = std::min(len - 1, e.size());
        std::memcpy(buf, e.data(), n);
        buf[n] = '\0';
    }
    return e.size();
}

const char *beep_status_string(beep_status s) {
    switch (s) {
    case BEEP_OK:
        return "ok";
    case BEEP_ERR_INVALID_ARG:
        return "invalid argument";
    case BEEP_ERR_IO:
        return "i/o error";
    case BEEP_ERR_PARSE:
        return "parse error";
    case BEEP_ERR_UNSUPPORTED:
        return "unsupported";
    case BEEP_ERR_CUDA:
        return "cuda error";
    case BEEP_ERR_OUT_OF_MEMORY:
        return "out of memory";
    case BEEP_ERR_TIMEOUT:
        return "timeout";
    case BEEP_ERR_INTERNAL:
        return "internal error";
    case BEEP_ERR_OVERFLOW:
        return "count overflow";
    }
    return "unknown";
}

beep_status beep_ctx_create(int device, void *stream, beep_ctx **out) {
    if (!out)
        return fail(BEEP_ERR_INVALID_ARG, "null output");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(BEEP_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= ndev)
        return fail(BEEP_ERR_INVALID_ARG, "device id out of range");
    auto *c = new beep_ctx;
    c->impl.device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&c->impl.num_sms, cudaDevAttrMultiProcessorCount, device);
    int optin = 0;
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    c->impl.smem_optin = (size_t)optin;
    if (e == cudaSuccess) {
        if (stream) {
            c->impl.stream = static_cast<cudaStream_t>(stream);
        } else {
            e = cudaStreamCreateWithFlags(&c->impl.stream, cudaStreamNonBlocking);
            c->impl.own_stream = true;
        }
    }
    if (e == cudaSuccess)
        e = cudaMallocHost(&c->impl.h_pinned, 64);
    if (e == cudaSuccess) {
        // per-call buffers come from a pool of this context that keeps its memory
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        e = cudaMemPoolCreate(&c->impl.pool, &props);
        if (e == cudaSuccess) {
            uint64_t keep = ~0ull;
            e = cudaMemPoolSetAttribute(c->impl.pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    if (e != cudaSuccess) {
        delete c;
        return fail(BEEP_ERR_CUDA, std::string("context setup: ") + cudaGetErrorString(e));
    }
    *out = c;
    return BEEP_OK;
}

namespace {
void ctx_free(beep_ctx *ctx) {
    cudaSetDevice(ctx->impl.device);
    cudaStreamSynchronize(ctx->impl.stream);
    ctx->impl.scratch.release();
    ctx->impl.scratch2.release();
    ctx->impl.arena.release();
    ctx->impl.counter.release();
    if (ctx->impl.h_pinned)
        cudaFreeHost(ctx->impl.h_pinned);
    if (ctx->impl.h_results)
        cudaFreeHost(ctx->impl.h_results);
    ctx->impl.release_side();
    if (ctx->impl.pool)
        cudaMemPoolDestroy(ctx->impl.pool);
    if (ctx->impl.own_stream)
        cudaStreamDestroy(ctx->impl.stream);
    delete ctx;
}
void ctx_release(beep_ctx *ctx) {
    if (ctx && ctx->refs.fetch_sub(1) == 1)
        ctx_free(ctx);
}
beep_graph *new_graph(beep_ctx *ctx) {
    auto *g = new beep_graph;
    g->ctx = ctx;
    g->impl.device = ctx->impl.device;
    ctx->refs.fetch_add(1);
    return g;
}
void graph_free(beep_graph *g) {
    beep_ctx *ctx = g->ctx;
    cudaSetDevice(g->impl.device);
    if (ctx)
        cudaStreamSynchronize(ctx->impl.stream);
    PhaseTrace tr("graph", ctx ? ctx->impl.stream : nullptr);
    delete g;
    tr.mark("destroy");
    ctx_release(ctx);
}
} // namespace

beep_status beep_ctx_destroy(beep_ctx *ctx) {
    ctx_release(ctx);
    return BEEP_OK;
}

beep_status beep_ctx_set_wait_timeout(beep_ctx *ctx, double ms) {
    if (!ctx || !(ms > 0))
        return fail(BEEP_ERR_INVALID_ARG, "bad timeout");
    ctx->impl.wait_timeout_ms = ms;
    return BEEP_OK;
}

beep_status beep_ctx_kernel_launches(const beep_ctx *ctx, uint64_t *out) {
    if (!ctx || !out)
        return fail(BEEP_ERR_INVALID_ARG, "beep_ctx_kernel_launches: bad arguments");
    *out = ctx->impl.launches;
    return BEEP_OK;
}

beep_status beep_graph_from_device_csr(beep_ctx *ctx, int64_t n, int64_t m, const int32_t *d_row_ptr,
                                       const int32_t *d_col_ind, beep_graph **out) {
    if (!out || !d_row_ptr || (m > 0 && !d_col_ind) || n < 0 || m < 0)
        return fail(BEEP_ERR_INVALID_ARG, "beep_graph_from_device_csr: bad arguments");
    *out = nullptr;
    BEEP_TRY(bind(ctx));
    beep_graph *g = new_graph(ctx);
    beep_status s = graph_build_from_device_csr(&ctx->impl, &g->impl, n, m,
                                                reinterpret_cast<const uint32_t *>(d_row_ptr),
                                                reinterpret_cast<const uint32_t *>(d_col_ind));
    if (s != BEEP_OK) {
        graph_free(g);
        return s;
    }
    *out = g;
    return BEEP_OK;
}

beep_status beep_graph_from_csr(beep_ctx *ctx, int64_t n, int64_t m, const int32_t *row_ptr, const int32_t *col_ind,
                                beep_graph **out) {
    if (!out || !row_ptr || (m > 0 && !col_ind) || n < 0 || m < 0)
        return fail(BEEP_ERR_INVALID_ARG, "beep_graph_from_csr: bad arguments");
    *out = nullptr;
    if (row_ptr[0] != 0 || row_ptr[n] != m)
        return fail(BEEP_ERR_INVALID_ARG, "row_ptr must start at 0 and end at m");
    BEEP_TRY(bind(ctx));
    beep_graph *g = new_graph(ctx);
    // Upload straight into the graph's buffers; the build keeps them when the
    // rows are already sorted and simple.
    beep_status s = upload(&ctx->impl, g->impl.row_ptr, reinterpret_cast<const uint32_t *>(row_ptr), (size_t)n + 1);
    if (s == BEEP_OK)
        s = upload(&ctx->impl, g->impl.col, reinterpret_cast<const uint32_t *>(col_ind), (size_t)m);
    if (s == BEEP_OK)
        s = graph_build_from_device_csr(&ctx->impl, &g->impl, n, m, g->impl.row_ptr.as<uint32_t>(),
                                        g->impl.col.as<uint32_t>());
    if (s != BEEP_OK) {
        graph_free(g);
        return s;
    }
    *out = g;
    return BEEP_OK;
}

beep_status beep_graph_from_edges(beep_ctx *ctx, int64_t n_edges, const uint32_t *src, const uint32_t *dst,
                                  beep_graph **out) {
    if (!out || n_edges < 0 || (n_edges > 0 && (!src || !dst)))
        return fail(BEEP_ERR_INVALID_ARG, "beep_graph_from_edges: bad arguments");
    *out = nullptr;
    BEEP_TRY(bind(ctx));
    DevBuf ds, dd;
    BEEP_TRY(upload(&ctx->impl, ds, src, (size_t)n_edges));
    BEEP_TRY(upload(&ctx->impl, dd, dst, (size_t)n_edges));
    beep_graph *g = new_graph(ctx);
    beep_status s = graph_build_from_device_edges(&ctx->impl, &g->impl, n_edges, ds.as<uint32_t>(), dd.as<uint32_t>());
    cudaStreamSynchronize(ctx->impl.stream);
    if (s != BEEP_OK) {
        graph_free(g);
        return s;
    }
    *out = g;
    return BEEP_OK;
}

beep_status beep_graph_load_bel(beep_ctx *ctx, const char *path, beep_graph **out) {
    if (!path || !out)
        return fail(BEEP_ERR_INVALID_ARG, "beep_graph_load_bel: bad arguments");
    std::vector<uint32_t> src, dst;
    BEEP_TRY(read_bel(path, src, dst));
    return beep_graph_from_edges(ctx, (int64_t)src.size(), src.data(), dst.data(), out);
}

beep_status beep_graph_info_get(const beep_graph *g, beep_graph_info *out) {
    if (!g || !out)
        return fail(BEEP_ERR_INVALID_ARG, "beep_graph_info_get: bad arguments");
    std::memset(out, 0, sizeof(*out));
    out->n = g->impl.n;
    out->m = g->impl.m;
    out->max_degree = g->impl.max_degree;
    out->cutoff = g->impl.cutoff;
    return BEEP_OK;
}

beep_status beep_graph_csr(const beep_graph *g, int32_t *row_ptr, int32_t *col_ind) {
    if (!g || !row_ptr || (g->impl.m > 0 && !col_ind))
        return fail(BEEP_ERR_INVALID_ARG, "beep_graph_csr: bad arguments");
    BEEP_TRY(bind(g->ctx));
    cudaStream_t s = g->ctx->impl.stream;
    BEEP_CUDA_TRY(cudaMemcpyAsync(row_ptr, g->impl.row_ptr.ptr, (size_t)(g->impl.n + 1) * 4, cudaMemcpyDeviceToHost, s));
    if (g->impl.m > 0)
        BEEP_CUDA_TRY(cudaMemcpyAsync(col_ind, g->impl.col.ptr, (size_t)g->impl.m * 4, cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    return BEEP_OK;
}

beep_status beep_graph_view(beep_graph *g, int32_t min_qdeg, int32_t asc, int64_t *n_out, int64_t *m_out,
                            int32_t *row_ptr, int32_t *col_ind, int32_t *orig) {
    if (!g || !n_out || !m_out || min_qdeg < 0)
        return fail(BEEP_ERR_INVALID_ARG, "beep_graph_view: bad arguments");
    BEEP_TRY(bind(g->ctx));
    Ctx *ctx = &g->ctx->impl;
    std::shared_ptr<View> v;
    BEEP_TRY(get_view(ctx, &g->impl, min_qdeg, asc ? 1 : 0, false, &v, nullptr));
    cudaStream_t s = ctx->stream;
    uint32_t m = 0;
    BEEP_CUDA_TRY(cudaMemcpyAsync(&m, v->row_ptr.as<uint32_t>() + v->n, 4, cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    *n_out = v->n;
    *m_out = m;
    if (!row_ptr && !col_ind && !orig)
        return BEEP_OK;
    if (!row_ptr || (m > 0 && !col_ind) || (v->n > 0 && !orig))
        return fail(BEEP_ERR_INVALID_ARG, "beep_graph_view: bad arguments");
    BEEP_CUDA_TRY(cudaMemcpyAsync(row_ptr, v->row_ptr.ptr, (size_t)(v->n + 1) * 4, cudaMemcpyDeviceToHost, s));
    if (m > 0)
        BEEP_CUDA_TRY(cudaMemcpyAsync(col_ind, v->col.ptr, (size_t)m * 4, cudaMemcpyDeviceToHost, s));
    if (v->n > 0)
        BEEP_CUDA_TRY(cudaMemcpyAsync(orig, v->orig.ptr, (size_t)v->n * 4, cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    return BEEP_OK;
}

beep_status beep_graph_destroy(beep_graph *g) {
    if (g)
        graph_free(g);
    return BEEP_OK;
}

beep_status beep_query_load_mtx(const char *path, beep_query **out) {
    if (!path || !out)
        return fail(BEEP_ERR_INVALID_ARG, "beep_query_load_mtx: bad arguments");
    *out = nullptr;
    std::vector<int32_t> src, dst;
    BEEP_TRY(read_mtx(path, src, dst));
    auto *q = new beep_query;
    beep_status s = query_from_edges(src, dst, &q->impl);
    if (s != BEEP_OK) {
        delete q;
        return s;
    }
    *out = q;
    return BEEP_OK;
}

beep_status beep_query_from_edges(int32_t n_edges, const int32_t *src, const int32_t *dst, beep_query **out) {
    if (!out || n_edges <= 0 || !src || !dst)
        return fail(BEEP_ERR_INVALID_ARG, "beep_query_from_edges: bad arguments");
    *out = nullptr;
    std::vector<int32_t> s(src, src + n_edges), d(dst, dst + n_edges);
    auto *q = new beep_query;
    beep_status st = query_from_edges(s, d, &q->impl);
    if (st != BEEP_OK) {
        delete q;
        return st;
    }
    *out = q;
    return BEEP_OK;
}

beep_status beep_query_destroy(beep_query *q) {
    delete q;
    return BEEP_OK;
}

beep_status beep_query_plan(const beep_query *q, beep_mode mode, beep_plan_info *out) {
    if (!q || !out)
        return fail(BEEP_ERR_INVALID_ARG, "beep_query_plan: bad arguments");
    if (mode != BEEP_MODE_SGM && mode != BEEP_MODE_SGC)
        return fail(BEEP_ERR_INVALID_ARG, "unknown mode");
    QueryPlan p;
    BEEP_TRY(compile_plan(q->impl.qn, q->impl.row_ptr, q->impl.col, mode, &p));
    *out = p.info;
    return BEEP_OK;
}

beep_status beep_count_ex(beep_ctx *ctx, beep_graph *g, const beep_query *q, beep_mode mode, uint32_t options,
                          beep_stats *stats) {
    if (!g || !q)
        return fail(BEEP_ERR_INVALID_ARG, "beep_count: null graph or query");
    if (mode != BEEP_MODE_SGM && mode != BEEP_MODE_SGC)
        return fail(BEEP_ERR_INVALID_ARG, "unknown mode");
    if (ctx && g->ctx && ctx->impl.device != g->impl.device)
        return fail(BEEP_ERR_INVALID_ARG, "graph lives on another device");
    if (!ctx)
        ctx = g->ctx;
    BEEP_TRY(bind(ctx));
    QueryPlan p;
    BEEP_TRY(compile_plan(q->impl.qn, q->impl.row_ptr, q->impl.col, mode, &p));
    beep_stats st;
    BEEP_TRY(run_count(&ctx->impl, &g->impl, p, options, nullptr, &st));
    ctx->impl.launches += (uint64_t)st.kernel_launches;
    if (stats)
        *stats = st;
    return overflow_status(st);
}

beep_status beep_count_shard(beep_ctx *ctx, beep_graph *g, const beep_query *q, beep_mode mode, uint32_t options,
                             uint32_t shard, uint32_t nshards, beep_stats *stats) {
    if (!g || !q || nshards == 0 || shard >= nshards)
        return fail(BEEP_ERR_INVALID_ARG, "beep_count_shard: bad arguments");
    if (mode != BEEP_MODE_SGM && mode != BEEP_MODE_SGC)
        return fail(BEEP_ERR_INVALID_ARG, "unknown mode");
    if (!ctx)
        ctx = g->ctx;
    if (ctx->impl.device != g->impl.device)
        return fail(BEEP_ERR_INVALID_ARG, "graph lives on another device");
    BEEP_TRY(bind(ctx));
    QueryPlan p;
    BEEP_TRY(compile_plan(q->impl.qn, q->impl.row_ptr, q->impl.col, mode, &p));
    beep_stats st;
    BEEP_TRY(run_count(&ctx->impl, &g->impl, p, options, nullptr, &st, shard, nshards));
    ctx->impl.launches += (uint64_t)st.kernel_launches;
    if (stats)
        *stats = st;
    return overflow_status(st);
}

beep_status beep_count(beep_ctx *ctx, beep_graph *g, const beep_query *q, beep_mode mode, uint64_t *out_count) {
    if (!out_count)
        return fail(BEEP_ERR_INVALID_ARG, "beep_count: null output");
    beep_stats st;
    const beep_status rc = beep_count_ex(ctx, g, q, mode, 0, &st);
    if (rc == BEEP_OK || rc == BEEP_ERR_OVERFLOW)
        *out_count = st.count;
    return rc;
}

beep_status beep_enumerate(beep_ctx *ctx, beep_graph *g, const beep_query *q, uint64_t k, int32_t *out_tuples,
                           uint64_t *n_out, uint64_t *total_count) {
    if (!g || !q || !n_out || (k > 0 && !out_tuples))
        return fail(BEEP_ERR_INVALID_ARG, "beep_enumerate: bad arguments");
    if (!ctx)
        ctx = g->ctx;
    BEEP_TRY(bind(ctx));
    QueryPlan p;
    BEEP_TRY(compile_plan(q->impl.qn, q->impl.row_ptr, q->impl.col, BEEP_MODE_SGM, &p));
    const size_t K = (size_t)p.info.K;
    DevBuf dout;
    BEEP_TRY(dout.reserve(std::max<uint64_t>(k, 1) * K * 4));
    EnumRequest er;
    er.k = k;
    er.d_out = dout.as<int32_t>();
    // two pairs in one call: the exact count (closed forms allowed) and the
    // enumerating walk, which stops once k tuples are written
    std::vector<PairSpec> specs(k > 0 ? 2 : 1);
    for (auto &ps : specs) {
        ps.g = &g->impl;
        ps.plan = p;
    }
    if (k > 0)
        specs[1].en = &er;
    uint64_t counts[2] = {0, 0};
    beep_stats st;
    BEEP_TRY(run_pairs(&ctx->impl, specs, 0, &st, counts));
    ctx->impl.launches += (uint64_t)st.kernel_launches;
    st.count = counts[0];
    if (st.count == BEEP_COUNT_OVERFLOW) {
        *n_out = 0;
        if (total_count)
            *total_count = st.count;
        return overflow_status(st);
    }
    const uint64_t got = std::min<uint64_t>(k, st.count);
    if (got)
        BEEP_CUDA_TRY(cudaMemcpyAsync(out_tuples, dout.ptr, got * K * 4, cudaMemcpyDeviceToHost, ctx->impl.stream));
    BEEP_CUDA_TRY(cudaStreamSynchronize(ctx->impl.stream));
    *n_out = got;
    if (total_count)
        *total_count = st.count;
    return BEEP_OK;
}

struct beep_batch {
    beep_ctx *ctx = nullptr;
    std::vector<beep::PairSpec> specs;
    beep::LaunchPlanPtr plan;
    uint32_t planned_options = 0;
    beep::TierCfg tiers;
};

beep_status beep_batch_create(beep_ctx *ctx, beep_batch **out) {
    if (!ctx || !out)
        return fail(BEEP_ERR_INVALID_ARG, "beep_batch_create: bad arguments");
    auto *b = new beep_batch;
    b->ctx = ctx;
    ctx->refs.fetch_add(1);
    *out = b;
    return BEEP_OK;
}

beep_status beep_batch_add(beep_batch *b, beep_graph *g, const beep_query *q, beep_mode mode, uint32_t *index) {
    if (!b || !g || !q)
        return fail(BEEP_ERR_INVALID_ARG, "beep_batch_add: bad arguments");
    if (mode != BEEP_MODE_SGM && mode != BEEP_MODE_SGC)
        return fail(BEEP_ERR_INVALID_ARG, "unknown mode");
    if (g->impl.device != b->ctx->impl.device)
        return fail(BEEP_ERR_INVALID_ARG, "graph lives on another device");
    PairSpec ps;
    ps.g = &g->impl;
    BEEP_TRY(compile_plan(q->impl.qn, q->impl.row_ptr, q->impl.col, mode, &ps.plan));
    b->specs.push_back(ps);
    b->plan.reset(); // re-plan on the next run
    if (index)
        *index = (uint32_t)(b->specs.size() - 1);
    return BEEP_OK;
}

beep_status beep_batch_size(const beep_batch *b, uint32_t *out) {
    if (!b || !out)
        return fail(BEEP_ERR_INVALID_ARG, "beep_batch_size: bad arguments");
    *out = (uint32_t)b->specs.size();
    return BEEP_OK;
}

beep_status beep_batch_run(beep_batch *b, uint32_t options, uint64_t *counts, beep_stats *stats) {
    if (!b || (!counts && !b->specs.empty()))
        return fail(BEEP_ERR_INVALID_ARG, "beep_batch_run: bad arguments");
    BEEP_TRY(bind(b->ctx));
    Ctx *ctx = &b->ctx->impl;
    const uint32_t plan_opts = options & (BEEP_OPT_REFERENCE_ROOT_CAP | BEEP_OPT_NO_VIEW_CACHE | BEEP_OPT_NO_NBHD);
    double prep_ms = 0;
    if (!b->plan || b->planned_options != plan_opts) {
        b->plan.reset();
        cudaEvent_t p0, p1;
        cudaEventCreate(&p0);
        cudaEventCreate(&p1);
        cudaEventRecord(p0, ctx->stream);
        BEEP_TRY(plan_pairs(ctx, b->specs, plan_opts, &b->plan, b->tiers));
        b->planned_options = plan_opts;
        cudaEventRecord(p1, ctx->stream);
        cudaEventSynchronize(p1);
        float ms = 0;
        cudaEventElapsedTime(&ms, p0, p1);
        prep_ms = ms;
        cudaEventDestroy(p0);
        cudaEventDestroy(p1);
    }
    if (!(options & BEEP_OPT_NO_GRAPH) && !(options & BEEP_OPT_TIMING))
        BEEP_TRY(capture_plan(ctx, b->plan.get()));
    beep_stats st;
    BEEP_TRY(execute_plan(ctx, b->plan.get(), options, &b->specs, counts, b->specs.size(), &st));
    st.prep_ms = prep_ms;
    ctx->launches += (uint64_t)st.kernel_launches;
    if (stats)
        *stats = st;
    return BEEP_OK;
}

beep_status beep_batch_set_tiers(beep_batch *b, const beep_tier_cfg *cfg) {
    if (!b || !cfg)
        return fail(BEEP_ERR_INVALID_ARG, "beep_batch_set_tiers: bad arguments");
    BEEP_TRY(bind(b->ctx));
    cudaStreamSynchronize(b->ctx->impl.stream);
    b->tiers = TierCfg{cfg->tiny_max, cfg->small_max, cfg->med_a_max, cfg->med_max, cfg->donate_min_iters};
    b->plan.reset(); // the next run plans (and captures) with the new limits
    return BEEP_OK;
}

beep_status beep_batch_autotune(beep_batch *b, uint32_t options, beep_tier_cfg *chosen, double *best_count_ms) {
    if (!b)
        return fail(BEEP_ERR_INVALID_ARG, "beep_batch_autotune: bad arguments");
    BEEP_TRY(bind(b->ctx));
    Ctx *ctx = &b->ctx->impl;
    const uint32_t plan_opts = options & BEEP_OPT_REFERENCE_ROOT_CAP;
    std::vector<uint64_t> counts(std::max<size_t>(b->specs.size(), 1));
    auto measure = [&](const TierCfg &cfg, double *ms) -> beep_status {
        LaunchPlanPtr lp;
        BEEP_TRY(plan_pairs(ctx, b->specs, plan_opts, &lp, cfg));
        beep_stats st;
        BEEP_TRY(execute_plan(ctx, lp.get(), BEEP_OPT_TIMING, &b->specs, counts.data(), b->specs.size(), &st));
        ctx->launches += (uint64_t)st.kernel_launches;
        *ms = st.count_ms;
        return BEEP_OK;
    };
    TierCfg best = b->tiers;
    double best_ms = 0;
    BEEP_TRY(measure(best, &best_ms)); // also builds the views, so later candidates time only the counting
    BEEP_TRY(measure(best, &best_ms));
    const std::vector<uint32_t> cand[5] = {{0, 8, 16}, {32, 64}, {128, 256}, {512, 1024}, {2, 4, 16}};
    for (int k = 0; k < 5; ++k)
        for (uint32_t val : cand[k]) {
            TierCfg c = best;
            uint32_t *f[5] = {&c.tiny_max, &c.small_max, &c.med_a_max, &c.med_max, &c.donate_min_iters};
            if (*f[k] == val)
                continue;
            *f[k] = val;
            double ms = 0;
            BEEP_TRY(measure(c, &ms));
            if (ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
    b->tiers = best;
    b->plan.reset();
    if (chosen)
        *chosen = beep_tier_cfg{best.tiny_max, best.small_max, best.med_a_max, best.med_max, best.donate_min_iters};
    if (best_count_ms)
        *best_count_ms = best_ms;
    return BEEP_OK;
}

beep_status beep_batch_destroy(beep_batch *b) {
    if (!b)
        return BEEP_OK;
    beep_ctx *ctx = b->ctx;
    cudaSetDevice(ctx->impl.device);
    cudaStreamSynchronize(ctx->impl.stream);
    b->plan.reset();
    delete b;
    ctx_release(ctx);
    return BEEP_OK;
}

} // extern "C"
