/*
 * beep.h — C ABI of the B200 subgraph counting / enumeration library.
 *
 * This is the drop-in boundary for BEEP's `-m sgm` / `-m sgc` path. The
 * reference exposes that path as a C++ template class
 *   graph::SG_Match<uint>(MAINTASK task, ProcessBy by, int dev, uint cutoff, int ndev)
 *   void SG_Match::run(COOCSRGraph_d<uint>& data, COOCSRGraph<uint>& query)
 * (subgraph_matching/subgraph_matching.cuh:113-231) behind the CLI in
 * src/main.cu:27-344, which loads the data graph from .bel
 * (include/FIleReader.cuh:51-95), the query from .mtx
 * (include/FIleReader.cuh:130-212, 299-353) and prints
 * "------------- Counter = N" (subgraph_matching.cuh:1277).
 *
 * Conventions of this ABI:
 *   - every call returns a beep_status; nothing exits, traps or aborts;
 *     beep_last_error() gives the message of the last failure on the thread;
 *   - device objects live behind opaque handles freed by *_destroy;
 *   - inputs are never mutated (the reference frees and replaces the caller's
 *     device CSR during peeling, subgraph_matching.cuh:746-756);
 *   - one beep_ctx per host thread; all work of a context is ordered on its
 *     CUDA stream.
 */
#ifndef BEEP_H
#define BEEP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BEEP_MAX_QUERY 10 /* subgraph_matching/include/host_utils.cuh:10 (DEPTH) */

typedef enum beep_status {
    BEEP_OK = 0,
    BEEP_ERR_INVALID_ARG = 1,   /* null pointer, bad size */
    BEEP_ERR_IO = 2,            /* file cannot be opened / read */
    BEEP_ERR_PARSE = 3,         /* malformed .mtx / .bel */
    BEEP_ERR_UNSUPPORTED = 4,   /* query outside the supported class (no central vertex, K>10, ...) */
    BEEP_ERR_CUDA = 5,          /* CUDA runtime error (message has the CUDA error string) */
    BEEP_ERR_OUT_OF_MEMORY = 6, /* device or host allocation failed / admission refused */
    BEEP_ERR_TIMEOUT = 7,       /* a bounded device wait ran out */
    BEEP_ERR_INTERNAL = 8,
    BEEP_ERR_OVERFLOW = 9       /* the count is BEEP_COUNT_LIMIT or more: not representable */
} beep_status;

/* Counts are exact below BEEP_COUNT_LIMIT = 2^64 - 2^52. A count at or above
 * it is reported as overflow (BEEP_ERR_OVERFLOW from the single-pair calls,
 * BEEP_COUNT_OVERFLOW in a batch's count slot) rather than reduced mod 2^64
 * as the reference's u64 counter is (subgraph_matching.cuh:1277). */
#define BEEP_COUNT_LIMIT 0xFFF0000000000000ull
#define BEEP_COUNT_OVERFLOW 0xFFFFFFFFFFFFFFFFull

/* MAINTASK values GRAPH_MATCH ("sgm") and GRAPH_COUNT ("sgc")
 * (include/defs.cuh:78-95, include/Config.h:80-84). */
typedef enum beep_mode {
    BEEP_MODE_SGM = 0, /* count every match (embeddings / |Aut(Q)|) */
    BEEP_MODE_SGC = 1  /* reference sgc: when the last query position is not adjacent to
                          the one before it (LUNMAT = 1), the count stops one level early
                          (subgraph_matching.cuh:612-631, device_utils.cuh:253,303) */
} beep_mode;

typedef struct beep_ctx beep_ctx;
typedef struct beep_graph beep_graph;
typedef struct beep_query beep_query;

/* ---- errors ------------------------------------------------------------ */

/* Copies the last error message of the calling thread into buf (NUL
 * terminated, truncated to len). Returns the full message length.
 * Replaces the reference's fprintf + exit(1) in CUDA_RUNTIME
 * (include/utils.cuh:27-40). */
size_t beep_last_error(char *buf, size_t len);
const char *beep_status_string(beep_status s);

/* ---- context ----------------------------------------------------------- */

/* Binds device `device` and a stream (NULL: the context creates its own).
 * Replaces SG_Match's `dev` argument and cudaSetDevice
 * (subgraph_matching.cuh:113, :180). */
beep_status beep_ctx_create(int device, void *cuda_stream, beep_ctx **out);
beep_status beep_ctx_destroy(beep_ctx *ctx);
/* Bound (milliseconds, default 1000) on every device-side wait of the
 * context's kernels: the large tier's warps that wait for donated work give
 * up after this long without progress anywhere on the GPU (no donation, no
 * finished task, no heartbeat of a running walk); the call then returns
 * BEEP_ERR_TIMEOUT and the context stays usable. Applies to calls planned
 * after it is set. */
beep_status beep_ctx_set_wait_timeout(beep_ctx *ctx, double ms);
/* Number of the library's own kernels launched on this context so far. */
beep_status beep_ctx_kernel_launches(const beep_ctx *ctx, uint64_t *out);

/* ---- data graph -------------------------------------------------------- */

/* Load a .bel edge list: 24-byte records {u64 dst, u64 src, u64 weight}
 * (include/FIleReader.cuh:51-95 read_bel; src/main.cu:72-130,283-300).
 * Self loops are dropped; duplicate edges are removed on the device. */
beep_status beep_graph_load_bel(beep_ctx *ctx, const char *path, beep_graph **out);

/* Build from a host CSR (both edge directions). Rows need not be sorted and
 * may hold duplicates or self loops: the device build sorts, dedups and drops
 * them. Replaces CSRCOO::from_edgelist + GPUArray::switch_to_gpu
 * (include/CSRCOO.cuh:37-80, src/main.cu:106-126, 283-300). */
beep_status beep_graph_from_csr(beep_ctx *ctx, int64_t n, int64_t m, const int32_t *row_ptr,
                                const int32_t *col_ind, beep_graph **out);
/* Same, from device pointers (copied into the graph; the caller keeps them). */
beep_status beep_graph_from_device_csr(beep_ctx *ctx, int64_t n, int64_t m, const int32_t *d_row_ptr,
                                       const int32_t *d_col_ind, beep_graph **out);
/* Build from a host edge list (src[i] -> dst[i]); self loops dropped,
 * duplicates removed, n = max id + 1 (include/CSRCOO.cuh:37-80). */
beep_status beep_graph_from_edges(beep_ctx *ctx, int64_t n_edges, const uint32_t *src, const uint32_t *dst,
                                  beep_graph **out);

typedef struct beep_graph_info {
    int64_t n;           /* vertices */
    int64_t m;           /* directed edges after dedup */
    int64_t max_degree;
    uint32_t cutoff;     /* ceil(mean + 6*sd) of the degree (include/utils.cuh:186-261, src/main.cu:132) */
    int32_t reserved;
} beep_graph_info;
beep_status beep_graph_info_get(const beep_graph *g, beep_graph_info *out);
/* Copy the deduped CSR back to the host (row_ptr[n+1], col_ind[m]). */
beep_status beep_graph_csr(const beep_graph *g, int32_t *row_ptr, int32_t *col_ind);
/* The graph as the counting kernels read it for one peel threshold and order
 * (built and cached as a count would): the iterated peel of the vertices of
 * degree in [1, min_qdeg) (subgraph_matching.cuh:685-764), then every vertex
 * that kept an edge, in priority order -- ascending (degree, id) when asc,
 * else descending degree with ties by ascending id -- and each row the sorted
 * new ids of its surviving neighbours (subgraph_matching.cuh:1282-1336).
 * With NULL arrays only *n_out and *m_out are written; otherwise row_ptr[n+1],
 * col_ind[m] and orig[n] (the input id of every new vertex) are filled too. */
beep_status beep_graph_view(beep_graph *g, int32_t min_qdeg, int32_t asc, int64_t *n_out, int64_t *m_out,
                            int32_t *row_ptr, int32_t *col_ind, int32_t *orig);
beep_status beep_graph_destroy(beep_graph *g);

/* ---- query ------------------------------------------------------------- */

/* Load a .mtx query: '%' lines (a '%%' banner may say "symmetric"), a
 * "rows cols nnz" line, then 0-based "row col" lines
 * (include/FIleReader.cuh:130-212, 299-353; src/main.cu:310-334). */
beep_status beep_query_load_mtx(const char *path, beep_query **out);
/* From a directed edge list as the .mtx lists it (both directions). */
beep_status beep_query_from_edges(int32_t n_edges, const int32_t *src, const int32_t *dst, beep_query **out);
beep_status beep_query_destroy(beep_query *q);

/* The compiled query plan (SG_Match::preprocess_query, detect_symmetry,
 * check_unmat, detect_reuse's first_sym_level: subgraph_matching.cuh:257-631). */
typedef struct beep_plan_info {
    int32_t K;
    int32_t order[BEEP_MAX_QUERY];                      /* query vertex at each position */
    int32_t qdeg[BEEP_MAX_QUERY];
    int32_t qedge_ptr[BEEP_MAX_QUERY + 1];              /* back edges (QEDGE / QEDGE_PTR) */
    int32_t qedge[BEEP_MAX_QUERY * (BEEP_MAX_QUERY - 1) / 2];
    int32_t sym_ptr[BEEP_MAX_QUERY + 1];                /* symmetry reps (SYMNODE / SYMNODE_PTR) */
    int32_t sym[BEEP_MAX_QUERY * (BEEP_MAX_QUERY - 1) / 2];
    int32_t unmat;                                      /* LUNMAT for the requested mode */
    int32_t first_sym_level;
    int32_t min_qdeg, max_qdeg;
    int32_t aut_order;                                  /* |Aut(Q)| */
    int32_t restricted;    /* 1: every position is ordered after the root, so only the
                              root's higher-priority neighbours are searched */
    int32_t central;       /* 1: position 0 is adjacent to every other position (the
                              reference's requirement, README.md:51-53); 0: counted by the
                              list-intersection walker (sgm, or sgc without an unmatched
                              last position) */
    int32_t wheel4;        /* 1: the 4-wheel's plan (positions 1-4 a 4-cycle around the
                              root); counts are summed once per (x1, x3) pair in closed form */
    int32_t nbhd;          /* > 0: a five-vertex query counted at the large tier's roots from
                              statistics of the root's neighbourhood graph (degrees, edges,
                              common neighbours per edge); 1 wedge + isolated vertex, 2 two
                              disjoint edges, 3 triangle + isolated vertex, 4 path, 5 paw,
                              6 diamond (the query minus its root) */
} beep_plan_info;
beep_status beep_query_plan(const beep_query *q, beep_mode mode, beep_plan_info *out);

/* ---- counting / enumeration -------------------------------------------- */

enum {
    /* Skip roots with degree >= 100*cutoff as the reference does
     * (subgraph_matching.cuh:1052, 1098). Off by default: those roots are counted. */
    BEEP_OPT_REFERENCE_ROOT_CAP = 1u << 0,
    /* Record per-phase device times with CUDA events (beep_stats). */
    BEEP_OPT_TIMING = 1u << 1,
    /* Drop the graph's cached peeled/ordered views before running. */
    BEEP_OPT_NO_VIEW_CACHE = 1u << 2,
    /* Compute the adjacency bytes of the searched roots (an extra pass). */
    BEEP_OPT_ALG_BYTES = 1u << 3,
    /* Launch the kernel tiers one after another on the call's stream instead
     * of overlapping them on side streams (with BEEP_OPT_TIMING: per-kernel
     * times that are each kernel's own). */
    BEEP_OPT_SERIAL_TIERS = 1u << 5,
    /* Test of the bounded device waits: the large tier's walk launches start
     * with one donated task that no donor ever publishes, so every warp that
     * waits for donated work runs out its wait (beep_ctx_set_wait_timeout)
     * and the call returns BEEP_ERR_TIMEOUT. No effect without large roots. */
    BEEP_OPT_WAIT_STALL_TEST = 1u << 6,
    /* Count the large tier's roots of every query by walking, even where the
     * plan has a neighbourhood-statistics form (beep_plan_info.nbhd). */
    BEEP_OPT_NO_NBHD = 1u << 7
};

typedef struct beep_stats {
    uint64_t count;
    int64_t roots;              /* roots searched */
    int64_t roots_small;        /* roots by kernel tier */
    int64_t roots_medium;
    int64_t roots_large;
    int32_t peel_rounds;
    int32_t ascending;          /* priority order used */
    uint32_t cutoff;
    int32_t kernel_launches;    /* kernels this call launched */
    double prep_ms;             /* device time: peel + ordering (BEEP_OPT_TIMING) */
    double count_ms;            /* device time: counting kernels */
    /* per tier (BEEP_OPT_TIMING); large_encode: row builds and word lists,
     * large_dfs: the large tier's walks and 4-wheel kernels */
    double small_ms, medium_ms, large_encode_ms, large_dfs_ms;
    int32_t small_launches, medium_launches, large_encode_launches, large_dfs_launches;
    uint64_t adjacency_bytes;   /* adjacency bytes the kernels must read (BEEP_OPT_ALG_BYTES) */
    uint64_t bitmap_bytes;      /* bitmap arena bytes of the large tier (rows and word lists) */
    uint64_t small_bytes, medium_bytes, large_bytes; /* adjacency_bytes by tier (BEEP_OPT_ALG_BYTES) */
    int64_t roots_general;      /* roots of non-central queries (list walker) */
    double general_ms;
    int32_t general_launches;
    int32_t overflow_pairs;     /* pairs whose count reached BEEP_COUNT_LIMIT (count is then
                                   BEEP_COUNT_OVERFLOW, also in the aggregate) */
    /* BEEP_OPT_ALG_BYTES: algorithmic bytes of the searched roots by tier,
     * 4 * (deg r + sum of deg v over v in N(r)) on the input CSR -- the
     * adjacency traffic of building each root's neighbourhood bitmap from the
     * CSR, whatever the kernels actually read */
    uint64_t alg_small_bytes, alg_medium_bytes, alg_large_bytes;
    /* BEEP_OPT_TIMING: per tier, the longest time of a launch from its first
     * to its last warp's exit -- from "every item taken" to "every item done",
     * the load-imbalance tail */
    double small_tail_ms, medium_tail_ms, large_tail_ms;
    uint64_t donated_tasks;     /* subtrees the large tier's walks handed to waiting warps */
} beep_stats;

/* Count matches. Replaces SG_Match::run + count_subgraphs + final_counter
 * (subgraph_matching.cuh:178-231, 1038-1279; host_utils.cuh:318-321).
 * stats may be NULL. */
beep_status beep_count(beep_ctx *ctx, beep_graph *g, const beep_query *q, beep_mode mode, uint64_t *out_count);
beep_status beep_count_ex(beep_ctx *ctx, beep_graph *g, const beep_query *q, beep_mode mode, uint32_t options,
                          beep_stats *stats);

/* Count only the roots whose input vertex id % nshards == shard. Roots are
 * independent, so the counts of shards 0..nshards-1 sum to beep_count's
 * count: one process per GPU can each count one shard of a replicated graph
 * and add the results (the reference's multi-device mode splits the level-1
 * work of heavy roots across devices instead, sgm_kernelsLD.cuh:60,
 * subgraph_matching.cuh:1149-1160). */
beep_status beep_count_shard(beep_ctx *ctx, beep_graph *g, const beep_query *q, beep_mode mode, uint32_t options,
                             uint32_t shard, uint32_t nshards, beep_stats *stats);

/* Enumerate up to k full matches (sgm semantics) as int32 tuples of data
 * vertex ids in ORIGINAL query-vertex order: out_tuples[i*K + v] is the data
 * vertex matched to query vertex v. *n_out = min(k, total); *total_count
 * (may be NULL) = the exact number of matches. Which matches are returned
 * when k < total is unspecified. The reference only counts (its last level
 * is a popcount, device_utils.cuh:303-306); this extends the same DFS. */
beep_status beep_enumerate(beep_ctx *ctx, beep_graph *g, const beep_query *q, uint64_t k, int32_t *out_tuples,
                           uint64_t *n_out, uint64_t *total_count);

/* ---- batched counting -------------------------------------------------- */

/* Many (graph, query, mode) pairs counted by one set of launches: the roots
 * of every pair are classified together, each kernel tier runs once over the
 * roots of all pairs, and the launch sequence is captured into a CUDA graph
 * on the first run and replayed afterwards. Replaces looping the plain count
 * over the pairs (the reference runs one SG_Match per query and graph,
 * subgraph_matching.cuh:178-231). The graphs and queries must outlive the
 * batch; adding a pair after a run re-plans the batch. */
typedef struct beep_batch beep_batch;
enum {
    /* Run the planned launches directly instead of through the CUDA graph. */
    BEEP_OPT_NO_GRAPH = 1u << 4
};
/* Domain-size limits of the kernel tiers a batch plans with (each clamped to
 * its kernel's bound: 16, 64, 256, 1024; defaults 8, 64, 256, 1024), and the
 * large tier's donation threshold. A root whose search domain has D vertices
 * goes to 8-lane groups if D <= tiny_max, warp groups if D <= small_max,
 * thread-walker blocks if D <= med_a_max, warp-walker blocks if D <= med_max,
 * and the global-arena tier above. In the global-arena tier a warp walking a
 * level hands the upper half of its remaining iterations (32 bitmap words
 * each) to a waiting warp when at least donate_min_iters remain (default 2;
 * 0 turns donation off). */
typedef struct beep_tier_cfg {
    uint32_t tiny_max, small_max, med_a_max, med_max;
    uint32_t donate_min_iters;
} beep_tier_cfg;
beep_status beep_batch_create(beep_ctx *ctx, beep_batch **out);
beep_status beep_batch_add(beep_batch *b, beep_graph *g, const beep_query *q, beep_mode mode, uint32_t *index);
/* counts[i] receives the count of the i-th added pair (array of at least
 * beep_batch_size entries); stats (may be NULL) aggregates the run. */
beep_status beep_batch_run(beep_batch *b, uint32_t options, uint64_t *counts, beep_stats *stats);
beep_status beep_batch_size(const beep_batch *b, uint32_t *out);
beep_status beep_batch_destroy(beep_batch *b);
/* Pick the batch's tier limits by measurement: coordinate descent over
 * tiny_max {0, 8, 16}, small_max {32, 64}, med_a_max {128, 256}, med_max
 * {512, 1024} and donate_min_iters {2, 4, 16}, each candidate planned and run
 * once (no CUDA graph) with its counting kernels timed by CUDA events; later
 * runs plan with the fastest. Counts do not depend on the choice. chosen and
 * best_count_ms may be NULL. */
beep_status beep_batch_autotune(beep_batch *b, uint32_t options, beep_tier_cfg *chosen, double *best_count_ms);
beep_status beep_batch_set_tiers(beep_batch *b, const beep_tier_cfg *cfg);

/* ---- serving ------------------------------------------------------------ */

/* A request server over resident graphs with continuous batching. Requests
 * are queued by beep_serve_submit and return at once; a scheduler thread
 * admits them in arrival order while the estimates of the batches in flight
 * fit the budget (free HBM at creation minus the reserve; the estimate covers
 * a request's tuple buffer, planning arrays and the large tier's bitmap
 * arena): a request that does not fit waits for running batches to finish,
 * and one that exceeds the whole budget is refused with
 * BEEP_ERR_OUT_OF_MEMORY instead of running out of memory. It plans whatever has
 * arrived as one multi-pair call and launches it on one of several streams
 * without waiting, so batches overlap on the device and requests arriving
 * meanwhile join the next batch as soon as a stream frees up. The reference
 * has no counterpart: it runs one SG_Match per query and graph
 * (subgraph_matching.cuh:178-231). Graphs added to a server must outlive it
 * and must not be used by other calls while it runs. */
typedef struct beep_server beep_server;
typedef struct beep_serve_options {
    uint32_t max_batch;         /* requests per batch (0: 64) */
    uint32_t streams;           /* batches in flight (0: 4) */
    uint64_t hbm_reserve_bytes; /* free HBM the admission keeps (0: 1 GiB) */
    uint32_t count_options;     /* BEEP_OPT_REFERENCE_ROOT_CAP or 0 */
    uint32_t reserved;
} beep_serve_options;
typedef struct beep_serve_result {
    beep_status status;
    int32_t K;                  /* query vertices (tuple width) */
    uint64_t count;             /* exact number of matches */
    uint64_t n_tuples;          /* tuples returned (first-k requests) */
    double latency_ms;          /* arrival to completion */
    double queue_ms;            /* arrival to launch of its batch */
} beep_serve_result;
typedef struct beep_serve_stats {
    uint64_t requests, batches, matches, kernel_launches;
    double p50_ms, p99_ms, mean_ms, max_ms;
    double span_s;              /* first arrival to last completion */
    double max_batch;
    uint64_t refused;           /* requests whose estimate exceeds the budget (BEEP_ERR_OUT_OF_MEMORY) */
    uint64_t max_inflight_bytes;/* largest sum of estimates of the batches in flight at once */
    uint64_t budget_bytes;      /* device bytes admission may hand out: free HBM at creation - reserve */
} beep_serve_stats;
beep_status beep_serve_create(beep_ctx *ctx, const beep_serve_options *opt, beep_server **out);
beep_status beep_serve_add_graph(beep_server *s, beep_graph *g, int32_t *graph_id);
/* k = 0: count (mode sgm or sgc); k > 0: also return the first k matches
 * (sgm semantics). */
beep_status beep_serve_submit(beep_server *s, int32_t graph_id, const beep_query *q, beep_mode mode, uint64_t k,
                              uint64_t *request_id);
/* Blocks until the request is done; consumes it. tuples (may be NULL) gets
 * up to tuples_cap tuples of K int32 in original query-vertex order. */
beep_status beep_serve_wait(beep_server *s, uint64_t request_id, beep_serve_result *res, int32_t *tuples,
                            uint64_t tuples_cap);
beep_status beep_serve_drain(beep_server *s);
beep_status beep_serve_stats_get(beep_server *s, beep_serve_stats *out);
beep_status beep_serve_destroy(beep_server *s);

/* ---- counting without allocation --------------------------------------- */

/* Size of the device scratch array the allocation-free path uses (64 MiB per
 * device, held from the first call until the process exits). */
#define BEEP_NOALLOC_SCRATCH_BYTES (64u << 20)
/* Largest search domain (vertices) whose bitmap fits that array: D rows of
 * ceil(D / 32) words must fit (64 MiB - 256 B) / 4 words. */
#define BEEP_NOALLOC_MAX_DOMAIN 23168u

/* Count matches without allocating any device memory. No counterpart in the
 * reference: it exists for callers that cannot let a library call cudaMalloc
 * -- processes whose device memory belongs to their own pool or caching
 * allocator (a library allocation can fail there or fragment the pool) and
 * latency-critical loops that cannot afford the device-wide synchronisation
 * of cudaMalloc/cudaFree.
 *
 * Input: the caller's CSR in device memory on `device` (rows sorted
 * ascending, no duplicate edge, no self loop, both directions -- the form
 * beep_graph_csr returns); output: the count written to *out_count (host).
 * The CSR is checked on the device before it is used: row pointers that are
 * not non-decreasing within [0, m], entries at or above n, rows that are not
 * strictly increasing and self loops are refused with BEEP_ERR_INVALID_ARG
 * before any counting work. Work is ordered on cuda_stream (NULL: the legacy
 * default stream) and the call waits for it: it returns when the count is on
 * the host. It calls no cudaMalloc, cudaFree or other
 * allocating routine: its only scratch is a file-scope device array of
 * BEEP_NOALLOC_SCRATCH_BYTES. The first call on a device looks up that array's
 * device address; make that first call before any stream capture.
 *
 * The graph is neither peeled nor relabelled: vertex ids give the symmetry-
 * breaking order, which leaves sgm counts unchanged. sgc queries whose last
 * level is unmaterialised (LUNMAT = 1) depend on the reference's degree order
 * and are refused with BEEP_ERR_UNSUPPORTED. Roots whose search domain exceeds
 * 1024 vertices keep their bitmap in the scratch array, so the largest domain
 * (a root's neighbours, or its higher-id neighbours for clique-like queries)
 * is limited to BEEP_NOALLOC_MAX_DOMAIN (23168) vertices; larger inputs are
 * refused with BEEP_ERR_UNSUPPORTED before any counting work; the fewer such
 * slices fit, the fewer blocks run. A count of BEEP_COUNT_LIMIT or more
 * returns BEEP_ERR_OVERFLOW. All calls on a device share the scratch array, which keeps the
 * last call's contents (each call clears what must start at zero); calls that
 * overlap on the GPU, from other streams or host threads, race on it. */
beep_status beep_count_noalloc(int device, void *cuda_stream, int64_t n, int64_t m, const int32_t *d_row_ptr,
                               const int32_t *d_col_ind, const beep_query *q, beep_mode mode, uint64_t *out_count);

/* ---- synthetic inputs and files ---------------------------------------- */

/* Deterministic generators (splitmix64 streams keyed by seed and edge index).
 * Each writes an undirected simple graph as a CSR with both directions, rows
 * sorted. Two-phase: call with row_ptr/col_ind NULL to get n and m, then
 * with buffers of n+1 and m entries. */
beep_status beep_gen_erdos_renyi(int64_t n, double p, uint64_t seed, int64_t *n_out, int64_t *m_out,
                                 int32_t *row_ptr, int32_t *col_ind);
beep_status beep_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                          int64_t *n_out, int64_t *m_out, int32_t *row_ptr, int32_t *col_ind);
beep_status beep_gen_chung_lu(int64_t n, double avg_degree, double exponent, uint64_t seed, int64_t *n_out,
                              int64_t *m_out, int32_t *row_ptr, int32_t *col_ind);

/* Write a CSR as .bel (src-sorted, both directions) — the byte format
 * read_bel consumes (include/FIleReader.cuh:63-89). */
beep_status beep_write_bel(const char *path, int64_t n, const int32_t *row_ptr, const int32_t *col_ind);

/* ---- file converters (the reference's -m txt-bel | mtx-bel | tsv-bel |
 * tsv-mtx | bel-mtx, src/main.cu:40-67 over graph::MtB_Writer,
 * include/FIleReader.cuh:456-912) ----------------------------------------- */
typedef enum beep_convert_task {
    BEEP_CONV_TXT_BEL = 0, /* "a b" lines, '%' comments -> both directions, sorted, unique */
    BEEP_CONV_MTX_BEL = 1, /* Matrix Market -> sorted records, mirrored when symmetric */
    BEEP_CONV_TSV_BEL = 2, /* "dst src weight" triples -> records in file order */
    BEEP_CONV_TSV_MTX = 3, /* "dst src weight" triples -> Matrix Market */
    BEEP_CONV_BEL_MTX = 4  /* .bel records -> Matrix Market */
} beep_convert_task;
/* Converts src_path into dst_path with the bytes the reference's converter
 * writes; *records_out (may be NULL) receives the records or entries written.
 * Inputs the reference cannot finish (no edges for a Matrix Market output, a
 * missing size line) return BEEP_ERR_PARSE instead. */
beep_status beep_convert(beep_convert_task task, const char *src_path, const char *dst_path, uint64_t *records_out);

#ifdef __cplusplus
}
#endif
#endif /* BEEP_H */
