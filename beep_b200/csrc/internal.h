// internal.h — shared host/device declarations of the B200 subgraph library.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/beep.h"

namespace beep {

// ---------------------------------------------------------------------------
// host phase trace: with BEEP_TRACE=1 in the environment, each marked phase
// synchronises its stream and prints its wall-clock time to stderr
// ---------------------------------------------------------------------------
bool trace_enabled();
struct PhaseTrace {
    const char *scope;
    cudaStream_t stream;
    double t0;
    PhaseTrace(const char *scope_, cudaStream_t s);
    void mark(const char *phase);
};

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
void set_error(const std::string &msg);
beep_status fail(beep_status s, const std::string &msg);

#define BEEP_CUDA_TRY(expr)                                                                        \
    do {                                                                                           \
        cudaError_t e__ = (expr);                                                                  \
        if (e__ != cudaSuccess) {                                                                  \
            return ::beep::fail(e__ == cudaErrorMemoryAllocation ? BEEP_ERR_OUT_OF_MEMORY            \
                                                                 : BEEP_ERR_CUDA,                  \
                                std::string(#expr) + ": " + cudaGetErrorString(e__));              \
        }                                                                                          \
    } while (0)

#define BEEP_TRY(expr)                                                                             \
    do {                                                                                           \
        beep_status s__ = (expr);                                                                  \
        if (s__ != BEEP_OK)                                                                        \
            return s__;                                                                            \
    } while (0)

// ---------------------------------------------------------------------------
// compiled query plan
// ---------------------------------------------------------------------------
constexpr int kMaxQ = BEEP_MAX_QUERY;

// The plan as the kernels consume it (passed by value as a kernel argument).
struct DevPlan {
    int32_t K;               // query vertices
    int32_t dend;            // positions matched: K (sgm) or K - LUNMAT (sgc)
    uint32_t back[kMaxQ];    // bit q (q >= 1): position q is a back edge of position p
    uint32_t sym[kMaxQ];     // bit s (s >= 1): x_p > x_s is required
    int32_t order[kMaxQ];    // query vertex at each position
    int32_t pos1_after_root; // position 1 must follow the root in the priority order
    int32_t restricted;      // every position follows the root: search only the out-list
    int32_t asc;             // ascending (degree, id) priority order
    int32_t free_from;       // positions [free_from, dend) share one back-edge set and form a symmetry chain
    uint32_t free_back;      // that back-edge set (bits q >= 1; 0: only the root)
    int32_t rows_needed;     // adjacency rows the DFS reads: 0 none, 1 only position 1's, 2 any
    int32_t central;         // position 0 adjacent to every position (else: list walker)
    uint32_t adj0;           // bit p: position p is adjacent to position 0
    uint32_t sym0;           // bit p: position p must follow position 0
    int32_t wheel4;          // the 4-wheel's plan: counted per (x1, x3) pair in closed form
    int32_t nbhd;            // NbhdForm: in the large tier, counted from neighbourhood statistics
};

// Five-vertex central queries whose count at a root v follows from statistics
// of the neighbourhood graph G[N(v)] (each is a cone over a 4-vertex graph H;
// a copy counts at v when v is its earliest universal vertex, as the walk's
// symmetry breaking counts it). d_u: degree of u in G[N(v)], E: its edges,
// c(u, w): common neighbours of u and w in it, D = |N(v)|.
enum NbhdForm : int32_t {
    kNbNone = 0,
    kNbWedgeIso = 1, // H = wedge + isolated vertex: sum_u C(d_u, 2) (D - 3)
    kNbTwoEdges = 2, // H = two disjoint edges:     C(E, 2) - sum_u C(d_u, 2)
    kNbTriIso = 3,   // H = triangle + isolated:    T (D - 3), T the triangles
    kNbPath4 = 4,    // H = path on 4 vertices:     sum over edges (d_u - 1)(d_w - 1) - 3T
    kNbPaw = 5,      // H = paw (universal vertex u after v): sum_u t_u (d_u - 2), t_u triangles at u
    kNbDiamond = 6   // H = diamond (both universal vertices after v): sum over edges C(c(u, w), 2)
};

struct QueryPlan {
    beep_plan_info info;     // the reference-visible plan (per mode)
    DevPlan dev;
};

// Compile the plan of a query CSR (qn vertices) for a mode.
beep_status compile_plan(int32_t qn, const std::vector<int32_t> &qrow_ptr, const std::vector<int32_t> &qcol,
                         beep_mode mode, QueryPlan *out);

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    bool pooled = false; // from a context's stream-ordered pool
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    // Owners release a buffer only after the work that uses it has completed
    // (they synchronise its stream first), so a pooled buffer goes back to
    // its pool at once.
    void release() {
        if (ptr) {
            if (pooled)
                cudaFreeAsync(ptr, cudaStreamPerThread);
            else
                cudaFree(ptr);
        }
        ptr = nullptr;
        bytes = 0;
        pooled = false;
    }
    // Grow-only: keeps the allocation when it is already large enough.
    beep_status reserve(size_t b) {
        if (b <= bytes && ptr)
            return BEEP_OK;
        release();
        if (b == 0)
            b = 16;
        cudaError_t e = cudaMalloc(&ptr, b);
        if (e != cudaSuccess) {
            ptr = nullptr;
            return fail(BEEP_ERR_OUT_OF_MEMORY, std::string("cudaMalloc ") + std::to_string(b) + " bytes: " +
                                                    cudaGetErrorString(e));
        }
        bytes = b;
        return BEEP_OK;
    }
    // Grow-only, from a stream-ordered pool: the old buffer is freed in the
    // order of stream s (work already queued on s may still read it) and the
    // new one is usable on s at once. Pool allocations cost microseconds where
    // cudaMalloc/cudaFree cost up to milliseconds and synchronise the device.
    beep_status reserve(size_t b, cudaMemPool_t pool, cudaStream_t s) {
        if (b <= bytes && ptr)
            return BEEP_OK;
        if (!pool)
            return reserve(b);
        if (ptr) {
            if (pooled)
                cudaFreeAsync(ptr, s);
            else
                cudaFree(ptr);
        }
        ptr = nullptr;
        bytes = 0;
        pooled = false;
        if (b == 0)
            b = 16;
        cudaError_t e = cudaMallocFromPoolAsync(&ptr, b, pool, s);
        if (e != cudaSuccess) {
            ptr = nullptr;
            return fail(BEEP_ERR_OUT_OF_MEMORY, std::string("device pool allocation of ") + std::to_string(b) +
                                                    " bytes: " + cudaGetErrorString(e));
        }
        bytes = b;
        pooled = true;
        return BEEP_OK;
    }
    template <typename T> T *as() const { return static_cast<T *>(ptr); }
};

// A peeled, priority-relabelled copy of the graph for one (min_qdeg, order).
// New ids follow the reference's priority order, so each sorted row is the
// reference's oriented_colInd row (subgraph_matching.cuh:1282-1336).
struct View {
    int32_t min_qdeg = 0;
    int32_t asc = 1;
    int64_t n = 0;           // vertices with degree > 0 after peeling
    int32_t peel_rounds = 0;
    DevBuf row_ptr;          // u32[n+1]
    DevBuf col;              // u32[row_ptr[n]] (sized for the graph's m), new ids, rows ascending
    DevBuf orig;             // u32[n]: new id -> input id
    DevBuf split;            // u32[n]: neighbours with a smaller new id
};

struct Graph {
    int device = 0;
    int64_t n = 0, m = 0;
    int64_t max_degree = 0;
    uint32_t cutoff = 0;
    DevBuf row_ptr; // u32[n+1]
    DevBuf col;     // u32[m]
    std::map<std::pair<int, int>, std::shared_ptr<View>> views;
};

struct Query {
    int32_t qn = 0;
    std::vector<int32_t> row_ptr, col; // query CSR as CSRCOO::from_edgelist builds it
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    double wait_timeout_ms = 1000.0;
    int num_sms = 148;
    size_t smem_optin = 0;
    DevBuf scratch;      // CUB temp storage and small per-call arrays
    DevBuf scratch2;
    DevBuf arena;        // neighbourhood bitmaps of large roots
    DevBuf counter;      // u64 counters
    unsigned long long *h_pinned = nullptr; // pinned host mirror of small results
    uint64_t launches = 0; // kernels of this library launched on the context
    cudaMemPool_t pool = nullptr; // stream-ordered pool for per-call buffers
    // grow b (a buffer of this context or of an object it builds) from the pool on the context's stream
    beep_status grow(DevBuf &b, size_t bytes) { return b.reserve(bytes, pool, stream); }
    // side streams and events that let the kernel tiers of one call overlap
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    beep_status ensure_side() {
        for (int i = 0; i < 2; ++i)
            if (!side[i]) {
                cudaError_t e = cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking);
                if (e == cudaSuccess)
                    e = cudaEventCreateWithFlags(&ev_join[i], cudaEventDisableTiming);
                if (e != cudaSuccess)
                    return fail(BEEP_ERR_CUDA, std::string("side stream: ") + cudaGetErrorString(e));
            }
        if (!ev_fork) {
            cudaError_t e = cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming);
            if (e != cudaSuccess)
                return fail(BEEP_ERR_CUDA, std::string("fork event: ") + cudaGetErrorString(e));
        }
        return BEEP_OK;
    }
    void release_side() {
        for (int i = 0; i < 2; ++i) {
            if (side[i])
                cudaStreamDestroy(side[i]);
            if (ev_join[i])
                cudaEventDestroy(ev_join[i]);
            side[i] = nullptr;
            ev_join[i] = nullptr;
        }
        if (ev_fork)
            cudaEventDestroy(ev_fork);
        ev_fork = nullptr;
    }
    // grow-only pinned host buffer for results read back by a call
    unsigned long long *h_results = nullptr;
    size_t h_results_n = 0;
    beep_status host_results(size_t n, unsigned long long **out) {
        if (n > h_results_n) {
            if (h_results)
                cudaFreeHost(h_results);
            h_results = nullptr;
            h_results_n = 0;
            cudaError_t e = cudaMallocHost(&h_results, std::max<size_t>(n, 1024) * sizeof(unsigned long long));
            if (e != cudaSuccess)
                return fail(BEEP_ERR_OUT_OF_MEMORY, std::string("cudaMallocHost: ") + cudaGetErrorString(e));
            h_results_n = std::max<size_t>(n, 1024);
        }
        *out = h_results;
        return BEEP_OK;
    }
};

// device entry points (device.cu)
beep_status graph_build_from_device_csr(Ctx *ctx, Graph *g, int64_t n, int64_t m, const uint32_t *d_row_ptr,
                                        const uint32_t *d_col);
beep_status graph_build_from_device_edges(Ctx *ctx, Graph *g, int64_t n_edges, const uint32_t *d_src,
                                          const uint32_t *d_dst);
beep_status get_view(Ctx *ctx, Graph *g, int32_t min_qdeg, int32_t asc, bool no_cache,
                     std::shared_ptr<View> *out, bool *built);

struct EnumRequest {
    uint64_t k = 0;
    int32_t *d_out = nullptr;  // k*K ints on the device
};

beep_status run_count(Ctx *ctx, Graph *g, const QueryPlan &plan, uint32_t options, const EnumRequest *en,
                      beep_stats *stats, uint32_t shard = 0, uint32_t nshards = 1);

// One (graph, compiled query) of a multi-pair call.
struct PairSpec {
    Graph *g = nullptr;
    QueryPlan plan;
    const EnumRequest *en = nullptr;
    uint32_t shard = 0, nshards = 1; // roots with input id % nshards == shard
};
// Count every pair in one set of launches; counts[i] receives pair i's count.
beep_status run_pairs(Ctx *ctx, const std::vector<PairSpec> &specs, uint32_t options, beep_stats *stats,
                      uint64_t *counts);

// A planned multi-pair call: its launches and the buffers they use.
struct LaunchPlan;
struct LaunchPlanDeleter {
    void operator()(LaunchPlan *p) const;
};
using LaunchPlanPtr = std::unique_ptr<LaunchPlan, LaunchPlanDeleter>;
// Domain-size limits of the kernel tiers (each at most the compile-time
// bound of its kernel): 8-lane small groups up to tiny_max, warp groups up to
// small_max (<= 64), thread-walker blocks up to med_a_max (<= 256), warp-walker
// blocks up to med_max (<= 1024), the global-arena tier above.
struct TierCfg {
    uint32_t tiny_max = 8, small_max = 64, med_a_max = 256, med_max = 1024; // tiny_max 8: the tuner's pick on C2
    // large tier: a walk hands half of its remaining iterations to a waiting
    // warp when at least this many remain (0: no donation)
    uint32_t donate_min_iters = 2;
};
beep_status plan_pairs(Ctx *ctx, const std::vector<PairSpec> &specs, uint32_t options, LaunchPlanPtr *out,
                       const TierCfg &tiers = TierCfg());
// Capture the plan's launches into a CUDA graph (relaunched by execute_plan).
beep_status capture_plan(Ctx *ctx, LaunchPlan *lp);
beep_status execute_plan(Ctx *ctx, LaunchPlan *lp, uint32_t options, const std::vector<PairSpec> *specs,
                         uint64_t *counts, size_t ncounts, beep_stats *stats);
// Issue the plan and its count read-back on ctx->stream without waiting; the
// read-back lands in h_buf, a pinned buffer of plan_host_words(lp) words that
// the caller owns and keeps until the stream has passed the launch.
beep_status launch_plan_async(Ctx *ctx, LaunchPlan *lp, unsigned long long *h_buf);
size_t plan_host_words(const LaunchPlan *lp);
// After the stream passed the launch: BEEP_ERR_TIMEOUT if a bounded wait ran out.
beep_status plan_status(const LaunchPlan *lp);
// After the stream passed the launch: the count of the spec_index-th pair.
uint64_t plan_count(const LaunchPlan *lp, size_t spec_index);
// Kernel launches of planning plus one execution.
int plan_launches(const LaunchPlan *lp);

// host helpers (io.cpp)
beep_status read_bel(const char *path, std::vector<uint32_t> &src, std::vector<uint32_t> &dst);
beep_status read_mtx(const char *path, std::vector<int32_t> &src, std::vector<int32_t> &dst);
beep_status query_from_edges(const std::vector<int32_t> &src, const std::vector<int32_t> &dst, Query *q);

} // namespace beep

// A context lives until its handle and every graph built on it are destroyed.
struct beep_ctx {
    beep::Ctx impl;
    std::atomic<int> refs{1};
};
struct beep_graph {
    beep::Graph impl;
    beep_ctx *ctx = nullptr;
};
struct beep_query {
    beep::Query impl;
};
