// graph.cu — on-device CSR build, dedup, iterated peeling and priority
// relabelling.
//
// The reference builds the CSR on the host (include/CSRCOO.cuh:37-80), peels
// with many synchronous launches and managed-memory reads
// (subgraph_matching.cuh:685-764) and orders every adjacency list with two
// global thrust::stable_sort passes over a triplet array
// (subgraph_matching.cuh:1282-1336). Here the whole graph is relabelled once
// per (peel threshold, order) by the same priority, so every sorted row of the
// relabelled CSR is the reference's oriented row and the split point is a
// lower_bound.
#include <cmath>

#include <cooperative_groups.h>
#include <cub/cub.cuh>

#include "internal.h"

namespace beep {

namespace {

constexpr unsigned kFull = 0xffffffffu;

// Rows are processed in two passes so that a few very long rows (hubs, which
// the priority order and R-MAT-like inputs put next to each other) cannot
// serialise on one warp: rows of up to kSerialMax entries are handled by one
// lane each; longer rows are cut into chunks of kChunk entries that the first
// pass appends to a list, and a second kernel spreads the chunks over every
// warp of the GPU.
constexpr uint32_t kSerialMax = 32;
constexpr uint32_t kChunk = 1024;

struct RowChunk {
    uint32_t row, b, e, pad;
};

// Warp-collective: lane l appends the chunks of [b, e) of row `row` when
// `big` (one atomic per warp).
// Entries past `cap` are dropped (only an invalid CSR, whose rows overlap, can
// have more chunks than a valid one); readers clamp the count to `cap`.
__device__ __forceinline__ void push_chunks(bool big, uint32_t row, uint32_t b, uint32_t e, RowChunk *list,
                                            unsigned *n_list, uint32_t cap, int lane) {
    const uint32_t nc = big ? (uint32_t)(((uint64_t)e - b + kChunk - 1) / kChunk) : 0u;
    uint32_t inc = nc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, inc, o);
        if (lane >= o)
            inc += t;
    }
    const uint32_t total = __shfl_sync(kFull, inc, 31);
    if (total == 0)
        return;
    uint32_t base = 0;
    if (lane == 31)
        base = atomicAdd(n_list, total);
    base = __shfl_sync(kFull, base, 31);
    const uint32_t pos = base + inc - nc;
    for (uint32_t c = 0; c < nc && pos + c < cap; ++c) {
        const uint32_t cb = b + c * kChunk;
        list[pos + c] = RowChunk{row, cb, min(cb + kChunk, e), 0u};
    }
}

// Capacity of a chunk list for a CSR of n rows and m entries.
inline size_t chunk_capacity(int64_t n, int64_t m) { return (size_t)n + (size_t)m / kChunk + 64; }

__global__ void k_check_csr(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, int64_t n, int64_t m,
                            unsigned *bad, RowChunk *chunks, unsigned *n_chunks, uint32_t cap) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    unsigned flag = 0;
    for (int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n; base += warps * 32) {
        const int64_t v = base + lane;
        bool big = false;
        uint32_t b = 0, e = 0;
        if (v < n) {
            b = rp[v];
            e = rp[v + 1];
            if (e < b || e > m)
                flag |= 2u; // row pointers unusable
            else if (e - b > kSerialMax)
                big = true;
            else
                for (uint32_t i = b; i < e; ++i) {
                    const uint32_t w = col[i];
                    if (!(w < n && w != (uint32_t)v && (i == b || col[i - 1] < w)))
                        flag |= 1u;
                }
        }
        push_chunks(big, (uint32_t)v, b, e, chunks, n_chunks, cap, lane);
    }
    flag = __reduce_or_sync(kFull, flag);
    if (lane == 0 && flag)
        atomicOr(bad, flag);
}

__global__ void k_check_chunks(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, int64_t n,
                               const RowChunk *__restrict__ chunks, const unsigned *__restrict__ n_chunks,
                               uint32_t cap, unsigned *bad) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t nc = min(*n_chunks, cap);
    unsigned flag = 0;
    for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nc; c += warps) {
        const RowChunk ch = chunks[c];
        const uint32_t rb = rp[ch.row];
        for (uint32_t i = ch.b + lane; i < ch.e; i += 32) {
            const uint32_t w = col[i];
            if (!(w < n && w != ch.row && (i == rb || col[i - 1] < w)))
                flag |= 1u;
        }
    }
    flag = __reduce_or_sync(kFull, flag);
    if (lane == 0 && flag)
        atomicOr(bad, flag);
}

__global__ void k_csr_keys(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, int64_t n,
                           uint64_t *keys) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        const uint32_t b = rp[v], e = rp[v + 1];
        for (uint32_t i = b + lane; i < e; i += 32) {
            const uint32_t w = col[i];
            keys[i] = (w == (uint32_t)v) ? ~0ull : (((uint64_t)v << 32) | w);
        }
    }
}

__global__ void k_edge_keys(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, int64_t ne,
                            uint64_t *keys, unsigned *max_id) {
    uint32_t mx = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t s = src[i], d = dst[i];
        keys[i] = (s == d) ? ~0ull : (((uint64_t)s << 32) | d);
        mx = max(mx, max(s, d));
    }
    for (int o = 16; o > 0; o >>= 1)
        mx = max(mx, __shfl_xor_sync(kFull, mx, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(max_id, mx);
}

// Keys are sorted and unique; the self-loop sentinel (~0) sorts last.
__global__ void k_keys_to_coo(const uint64_t *__restrict__ keys, int64_t m, uint32_t *col, uint32_t *deg) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        col[i] = (uint32_t)k;
        atomicAdd(&deg[k >> 32], 1u);
    }
}

__global__ void k_degree_stats(const uint32_t *__restrict__ rp, int64_t n, unsigned long long *sumsq,
                               unsigned *maxdeg) {
    unsigned long long s = 0;
    uint32_t mx = 0;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t d = rp[v + 1] - rp[v];
        s += (unsigned long long)d * d;
        mx = max(mx, d);
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(kFull, s, o);
        mx = max(mx, __shfl_xor_sync(kFull, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(sumsq, s);
        atomicMax(maxdeg, mx);
    }
}

// ---- peeling --------------------------------------------------------------

__global__ void k_peel_init(const uint32_t *__restrict__ rp, int64_t n, uint32_t *deg, uint8_t *alive) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        deg[v] = rp[v + 1] - rp[v];
        alive[v] = 1;
    }
}

// All peel rounds in one cooperative launch (every block resident; grid-wide
// barriers between the phases of a round). A round removes together every
// vertex whose degree is in [1, min_qdeg) (bucket_scan window,
// subgraph_matching.cuh:66-109, 703) and lowers the degree of each surviving
// neighbour once per removed neighbour, which leaves every degree equal to the
// count of surviving neighbours -- what the reference's full recount gives
// (remove_edges_connected_to_node + warp_detect_deleted_edges,
// common_utils.cuh:99-133, 217-246). Rounds go on while one removes more than
// 5% of n (subgraph_matching.cuh:699-758), so there are at most 21;
// removed[r] counts round r (zeroed by the caller, kPeelMaxRounds entries).
constexpr int kPeelMaxRounds = 32;

__global__ void k_peel_fused(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, int64_t n,
                             uint32_t min_qdeg, uint32_t *deg, uint8_t *alive, uint32_t *list,
                             unsigned long long *removed, int *rounds_out) {
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    const int lane = threadIdx.x & 31;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = nth >> 5;
    const double limit = 0.05 * (double)n;
    int round = 0;
    for (;;) {
        unsigned long long *cnt = removed + round;
        // mark: threads of a warp take 32 consecutive vertices; one atomic per warp
        for (int64_t base = warp * 32; base < n; base += nwarps * 32) {
            const int64_t v = base + lane;
            bool out = false;
            if (v < n) {
                const uint32_t d = deg[v];
                out = d >= 1 && d < min_qdeg;
                if (out)
                    alive[v] = 0;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, out);
            if (!bal)
                continue;
            unsigned long long at = 0;
            if (lane == 0)
                at = atomicAdd(cnt, (unsigned long long)__popc(bal));
            at = __shfl_sync(0xffffffffu, at, 0);
            if (out)
                list[at + __popc(bal & ((1u << lane) - 1u))] = (uint32_t)v;
        }
        grid.sync();
        const unsigned long long R = *(volatile unsigned long long *)cnt;
        // lower the surviving neighbours' degrees: a warp per removed vertex
        for (unsigned long long i = (unsigned long long)warp; i < R; i += (unsigned long long)nwarps) {
            const uint32_t w = list[i];
            if (lane == 0)
                deg[w] = 0;
            const uint32_t b = rp[w], e = rp[w + 1];
            for (uint32_t k = b + lane; k < e; k += 32) {
                const uint32_t u = col[k];
                if (alive[u])
                    atomicSub(&deg[u], 1u);
            }
        }
        grid.sync();
        ++round;
        if (!((double)R > limit) || round >= kPeelMaxRounds)
            break;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        *rounds_out = round;
}

// ---- relabelling -----------------------------------------------------------

// Priority key (subgraph_matching.cuh:1299-1331, host_utils.cuh:230-246):
// ascending (degree, id) or descending degree with ties by ascending id.
// Vertices left with no edge get the largest key and are dropped.
// The key is the degree part alone; a stable radix sort of (key, id) pairs
// with ids in increasing order keeps ties by ascending id.
__global__ void k_prio_keys(const uint32_t *__restrict__ deg, int64_t n, uint32_t maxdeg, int asc,
                            uint32_t *keys, uint32_t *ids, unsigned long long *n_alive) {
    unsigned long long c = 0;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t d = deg[v];
        uint32_t k;
        if (d == 0) {
            k = maxdeg;
        } else {
            k = asc ? d - 1 : maxdeg - d;
            ++c;
        }
        keys[v] = k;
        ids[v] = (uint32_t)v;
    }
    for (int o = 16; o > 0; o >>= 1)
        c += __shfl_xor_sync(kFull, c, o);
    if ((threadIdx.x & 31) == 0 && c)
        atomicAdd(n_alive, c);
}

__global__ void k_rank(const uint32_t *__restrict__ sorted_ids, int64_t n_alive, uint32_t *orig, uint32_t *rank,
                       const uint32_t *__restrict__ deg, uint32_t *new_deg) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_alive;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t v = sorted_ids[i];
        orig[i] = v;
        rank[v] = (uint32_t)i;
        new_deg[i] = deg[v];
    }
}

// The relabelled rows are produced by one sort: every input entry (v, w)
// becomes the key (rank v) << rb | rank w (ranks < 2^rb), or ~0 when either
// end was dropped,
// written at the entry's own position; sorting the keys leaves the new rows
// in order, each sorted, with the dropped entries after them. No per-row
// sort, so a few very long rows (hubs) cannot hold up the rest.
__device__ __forceinline__ uint64_t view_key(uint32_t rv, uint32_t rw, int rb) {
    return (rv == 0xffffffffu || rw == 0xffffffffu) ? ~0ull : (((uint64_t)rv << rb) | rw);
}

__global__ void k_fill_keys(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col,
                            const uint32_t *__restrict__ rank, int64_t n, int rb, uint64_t *keys,
                            RowChunk *chunks, unsigned *n_chunks, uint32_t cap) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n; base += warps * 32) {
        const int64_t v = base + lane;
        bool big = false;
        uint32_t b = 0, e = 0;
        if (v < n) {
            b = rp[v];
            e = rp[v + 1];
            if (e - b > kSerialMax) {
                big = true;
            } else {
                const uint32_t rv = rank[v];
                for (uint32_t k = b; k < e; ++k)
                    keys[k] = view_key(rv, rank[col[k]], rb);
            }
        }
        push_chunks(big, (uint32_t)v, b, e, chunks, n_chunks, cap, lane);
    }
}

__global__ void k_fill_key_chunks(const uint32_t *__restrict__ col, const uint32_t *__restrict__ rank,
                                  const RowChunk *__restrict__ chunks, const unsigned *__restrict__ n_chunks,
                                  uint32_t cap, int rb, uint64_t *keys) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t nc = min(*n_chunks, cap);
    for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nc; c += warps) {
        const RowChunk ch = chunks[c];
        const uint32_t rv = rank[ch.row];
        for (uint32_t k = ch.b + lane; k < ch.e; k += 32)
            keys[k] = view_key(rv, rank[col[k]], rb);
    }
}

// The first *m_live sorted keys are the view's entries (the dropped ones,
// all ones, sort last).
__global__ void k_keys_low(const uint64_t *__restrict__ keys, const uint32_t *__restrict__ m_live, int rb,
                           uint32_t *col) {
    const uint64_t mask = ((uint64_t)1 << rb) - 1;
    const int64_t m = *m_live;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        col[i] = (uint32_t)(keys[i] & mask);
}

// split[i] = number of neighbours with a smaller new id (lower_bound of i).
__global__ void k_split(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, int64_t n,
                        uint32_t *split) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t lo = rp[i], hi = rp[i + 1];
        const uint32_t b = lo;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (col[mid] < (uint32_t)i)
                lo = mid + 1;
            else
                hi = mid;
        }
        split[i] = lo - b;
    }
}

inline int grid_for(int64_t items, int block, int num_sms) {
    int64_t g = (items + block - 1) / block;
    int64_t cap = (int64_t)num_sms * 32;
    if (g > cap)
        g = cap;
    if (g < 1)
        g = 1;
    return (int)g;
}

// Bump allocator over a grow-only buffer.
struct Carve {
    char *base;
    size_t off = 0;
    explicit Carve(void *b) : base(static_cast<char *>(b)) {}
    template <typename T> T *take(size_t count) {
        off = (off + 255) & ~(size_t)255;
        T *p = reinterpret_cast<T *>(base + off);
        off += count * sizeof(T);
        return p;
    }
    static size_t need(std::initializer_list<size_t> bytes) {
        size_t s = 0;
        for (size_t b : bytes)
            s += ((b + 255) & ~(size_t)255) + 256;
        return s;
    }
};

// Sorted unique u64 keys -> CSR in g.
beep_status keys_to_graph(Ctx *ctx, Graph *g, uint64_t *keys, uint64_t *keys_tmp, int64_t nkeys, int64_t n) {
    cudaStream_t s = ctx->stream;
    // sort
    int end_bit = 64;
    size_t tb = 0;
    BEEP_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys, keys_tmp, nkeys, 0, end_bit, s));
    BEEP_TRY(ctx->grow(ctx->scratch, tb + 1024));
    BEEP_CUDA_TRY(cub::DeviceRadixSort::SortKeys(ctx->scratch.ptr, tb, keys, keys_tmp, nkeys, 0, end_bit, s));
    // unique
    BEEP_TRY(ctx->grow(ctx->counter, 64));
    unsigned long long *d_num = ctx->counter.as<unsigned long long>();
    tb = 0;
    BEEP_CUDA_TRY(cub::DeviceSelect::Unique(nullptr, tb, keys_tmp, keys, d_num, nkeys, s));
    BEEP_TRY(ctx->grow(ctx->scratch, tb + 1024));
    BEEP_CUDA_TRY(cub::DeviceSelect::Unique(ctx->scratch.ptr, tb, keys_tmp, keys, d_num, nkeys, s));
    unsigned long long h_num = 0;
    BEEP_CUDA_TRY(cudaMemcpyAsync(&h_num, d_num, sizeof(h_num), cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    int64_t m = (int64_t)h_num;
    if (m > 0) {
        uint64_t last = 0;
        BEEP_CUDA_TRY(cudaMemcpyAsync(&last, keys + (m - 1), sizeof(last), cudaMemcpyDeviceToHost, s));
        BEEP_CUDA_TRY(cudaStreamSynchronize(s));
        if (last == ~0ull)
            --m; // self-loop sentinel
    }
    if (m >= (int64_t)0xffffffffll)
        return fail(BEEP_ERR_UNSUPPORTED, "graph has 2^32 or more directed edges");
    g->n = n;
    g->m = m;
    BEEP_TRY(ctx->grow(g->row_ptr, (size_t)(n + 1) * 4));
    BEEP_TRY(ctx->grow(g->col, (size_t)(m > 0 ? m : 1) * 4));
    uint32_t *deg = g->row_ptr.as<uint32_t>();
    BEEP_CUDA_TRY(cudaMemsetAsync(deg, 0, (size_t)(n + 1) * 4, s));
    if (m > 0) {
        k_keys_to_coo<<<grid_for(m, 256, ctx->num_sms), 256, 0, s>>>(keys, m, g->col.as<uint32_t>(), deg);
        ++ctx->launches;
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    tb = 0;
    BEEP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, deg, deg, n + 1, s));
    BEEP_TRY(ctx->grow(ctx->scratch, tb + 1024));
    BEEP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(ctx->scratch.ptr, tb, deg, deg, n + 1, s));
    return BEEP_OK;
}

beep_status finish_graph(Ctx *ctx, Graph *g) {
    cudaStream_t s = ctx->stream;
    BEEP_TRY(ctx->grow(ctx->counter, 64));
    unsigned long long *d = ctx->counter.as<unsigned long long>();
    BEEP_CUDA_TRY(cudaMemsetAsync(d, 0, 16, s));
    if (g->n > 0)
        k_degree_stats<<<grid_for(g->n, 256, ctx->num_sms), 256, 0, s>>>(g->row_ptr.as<uint32_t>(), g->n, d,
                                                                         reinterpret_cast<unsigned *>(d + 1));
    BEEP_CUDA_TRY(cudaGetLastError());
    unsigned long long h[2] = {0, 0};
    BEEP_CUDA_TRY(cudaMemcpyAsync(h, d, 16, cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    g->max_degree = (int64_t)(uint32_t)h[1];
    // cutoff = ceil(mean + 6 sd) over all n vertices (include/utils.cuh:241-260)
    if (g->n > 0) {
        const double n = (double)g->n;
        const double mean = (double)g->m / n;
        double var = (double)h[0] / n - mean * mean;
        if (var < 0)
            var = 0;
        g->cutoff = (uint32_t)std::ceil(mean + 6.0 * std::sqrt(var));
    } else {
        g->cutoff = 0;
    }
    g->views.clear();
    return BEEP_OK;
}

} // namespace

beep_status graph_build_from_device_csr(Ctx *ctx, Graph *g, int64_t n, int64_t m, const uint32_t *d_rp,
                                        const uint32_t *d_col) {
    cudaStream_t s = ctx->stream;
    if (n < 0 || m < 0 || n >= (int64_t)0xffffffffll || m >= (int64_t)0xffffffffll)
        return fail(BEEP_ERR_INVALID_ARG, "graph size out of range");
    PhaseTrace tr("graph", s);
    // Fast path: rows already strictly increasing with no self loop.
    BEEP_TRY(ctx->grow(ctx->counter, 64));
    unsigned *d_bad = reinterpret_cast<unsigned *>(ctx->counter.as<char>() + 32);
    unsigned *d_nchunks = reinterpret_cast<unsigned *>(ctx->counter.as<char>() + 36);
    BEEP_CUDA_TRY(cudaMemsetAsync(d_bad, 0, 8, s));
    if (n > 0) {
        BEEP_TRY(ctx->grow(ctx->scratch2, chunk_capacity(n, m) * sizeof(RowChunk)));
        RowChunk *chunks = ctx->scratch2.as<RowChunk>();
        const uint32_t cap = (uint32_t)std::min<size_t>(chunk_capacity(n, m), 0xffffffffu);
        k_check_csr<<<grid_for(n, 256, ctx->num_sms), 256, 0, s>>>(d_rp, d_col, n, m, d_bad, chunks, d_nchunks,
                                                                     cap);
        k_check_chunks<<<ctx->num_sms * 8, 256, 0, s>>>(d_rp, d_col, n, chunks, d_nchunks, cap, d_bad);
        ctx->launches += 2;
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    unsigned h_bad = 0;
    uint32_t h_m_end = 0;
    BEEP_CUDA_TRY(cudaMemcpyAsync(&h_bad, d_bad, 4, cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaMemcpyAsync(&h_m_end, d_rp + n, 4, cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    if ((int64_t)h_m_end != m)
        return fail(BEEP_ERR_INVALID_ARG, "row_ptr[n] != m");
    if (h_bad & 2u)
        return fail(BEEP_ERR_INVALID_ARG, "row_ptr is not non-decreasing within [0, m]");
    tr.mark("check");
    if (!h_bad) {
        g->n = n;
        g->m = m;
        BEEP_TRY(ctx->grow(g->row_ptr, (size_t)(n + 1) * 4));
        BEEP_TRY(ctx->grow(g->col, (size_t)(m > 0 ? m : 1) * 4));
        if (g->row_ptr.ptr != (const void *)d_rp)
            BEEP_CUDA_TRY(cudaMemcpyAsync(g->row_ptr.ptr, d_rp, (size_t)(n + 1) * 4, cudaMemcpyDeviceToDevice, s));
        if (m > 0 && g->col.ptr != (const void *)d_col)
            BEEP_CUDA_TRY(cudaMemcpyAsync(g->col.ptr, d_col, (size_t)m * 4, cudaMemcpyDeviceToDevice, s));
        tr.mark("copy");
        beep_status st = finish_graph(ctx, g);
        tr.mark("stats");
        return st;
    }
    // Slow path: sort + unique packed (src, dst) keys. Out-of-range ids fail.
    DevBuf keys, keys2;
    BEEP_TRY(keys.reserve((size_t)(m > 0 ? m : 1) * 8));
    BEEP_TRY(keys2.reserve((size_t)(m > 0 ? m : 1) * 8));
    if (n > 0) {
        k_csr_keys<<<grid_for(n * 32, 256, ctx->num_sms), 256, 0, s>>>(d_rp, d_col, n, keys.as<uint64_t>());
        ++ctx->launches;
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    BEEP_TRY(keys_to_graph(ctx, g, keys.as<uint64_t>(), keys2.as<uint64_t>(), m, n));
    // validate ids
    if (g->m > 0) {
        uint32_t maxc = 0;
        size_t tb = 0;
        unsigned *d_max = reinterpret_cast<unsigned *>(ctx->counter.as<char>() + 40);
        BEEP_CUDA_TRY(cub::DeviceReduce::Max(nullptr, tb, g->col.as<uint32_t>(), d_max, g->m, s));
        BEEP_TRY(ctx->grow(ctx->scratch, tb + 1024));
        BEEP_CUDA_TRY(cub::DeviceReduce::Max(ctx->scratch.ptr, tb, g->col.as<uint32_t>(), d_max, g->m, s));
        BEEP_CUDA_TRY(cudaMemcpyAsync(&maxc, d_max, 4, cudaMemcpyDeviceToHost, s));
        BEEP_CUDA_TRY(cudaStreamSynchronize(s));
        if ((int64_t)maxc >= n)
            return fail(BEEP_ERR_INVALID_ARG, "column index >= n");
    }
    return finish_graph(ctx, g);
}

beep_status graph_build_from_device_edges(Ctx *ctx, Graph *g, int64_t ne, const uint32_t *d_src,
                                          const uint32_t *d_dst) {
    cudaStream_t s = ctx->stream;
    if (ne < 0 || ne >= (int64_t)0xffffffffll)
        return fail(BEEP_ERR_INVALID_ARG, "edge count out of range");
    DevBuf keys, keys2;
    BEEP_TRY(keys.reserve((size_t)(ne > 0 ? ne : 1) * 8));
    BEEP_TRY(keys2.reserve((size_t)(ne > 0 ? ne : 1) * 8));
    BEEP_TRY(ctx->grow(ctx->counter, 64));
    unsigned *d_max = reinterpret_cast<unsigned *>(ctx->counter.as<char>() + 48);
    BEEP_CUDA_TRY(cudaMemsetAsync(d_max, 0, 4, s));
    if (ne > 0) {
        k_edge_keys<<<grid_for(ne, 256, ctx->num_sms), 256, 0, s>>>(d_src, d_dst, ne, keys.as<uint64_t>(), d_max);
        ++ctx->launches;
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    unsigned h_max = 0;
    BEEP_CUDA_TRY(cudaMemcpyAsync(&h_max, d_max, 4, cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    int64_t n = ne > 0 ? (int64_t)h_max + 1 : 0;
    BEEP_TRY(keys_to_graph(ctx, g, keys.as<uint64_t>(), keys2.as<uint64_t>(), ne, n));
    return finish_graph(ctx, g);
}

namespace {

beep_status build_view(Ctx *ctx, Graph *g, int32_t min_qdeg, int32_t asc, View *v) {
    cudaStream_t s = ctx->stream;
    const int64_t n = g->n, m = g->m;
    v->min_qdeg = min_qdeg;
    v->asc = asc;
    const uint32_t *rp = g->row_ptr.as<uint32_t>();
    const uint32_t *col = g->col.as<uint32_t>();
    const int64_t nn = n > 0 ? n : 1;
    const size_t cap = chunk_capacity(n, m);
    const size_t mm = m > 0 ? (size_t)m : 1;
    size_t need = Carve::need({(size_t)nn * 4, (size_t)nn, (size_t)nn * 4, (size_t)nn * 4, (size_t)nn * 4,
                               (size_t)nn * 4, (size_t)nn * 4, (size_t)nn * 4, mm * 8, mm * 8,
                               cap * sizeof(RowChunk), 16, (size_t)nn * 4, kPeelMaxRounds * 8});
    BEEP_TRY(ctx->grow(ctx->scratch2, need));
    Carve cv(ctx->scratch2.ptr);
    uint32_t *deg = cv.take<uint32_t>(nn);
    uint8_t *alive = cv.take<uint8_t>(nn);
    uint32_t *rank = cv.take<uint32_t>(nn);
    uint32_t *pkey = cv.take<uint32_t>(nn), *pid = cv.take<uint32_t>(nn);
    uint32_t *pkey2 = cv.take<uint32_t>(nn), *pid2 = cv.take<uint32_t>(nn);
    uint32_t *new_deg = cv.take<uint32_t>(nn);
    uint64_t *ekeys = cv.take<uint64_t>(mm), *ekeys2 = cv.take<uint64_t>(mm);
    RowChunk *chunks = cv.take<RowChunk>(cap);
    unsigned *d_nchunks = cv.take<unsigned>(4); // [0] chunk count, [2] peel rounds
    uint32_t *peel_list = cv.take<uint32_t>(nn);
    unsigned long long *peel_removed = cv.take<unsigned long long>(kPeelMaxRounds);
    const uint32_t ucap = (uint32_t)std::min<size_t>(cap, 0xffffffffu);
    BEEP_TRY(ctx->grow(ctx->counter, 64));
    unsigned long long *d_removed = ctx->counter.as<unsigned long long>();

    PhaseTrace tr("view", s);
    const int gv = grid_for(n, 256, ctx->num_sms);
    if (n > 0) {
        k_peel_init<<<gv, 256, 0, s>>>(rp, n, deg, alive);
        ++ctx->launches;
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    // Iterated peel, all rounds in one cooperative launch (no host round trip
    // per round).
    int *d_rounds = reinterpret_cast<int *>(d_nchunks + 2);
    BEEP_CUDA_TRY(cudaMemsetAsync(d_rounds, 0, 4, s));
    if (min_qdeg > 1 && n > 0) {
        BEEP_CUDA_TRY(cudaMemsetAsync(peel_removed, 0, kPeelMaxRounds * 8, s));
        int per_sm = 0;
        BEEP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_peel_fused, 256, 0));
        // two blocks per SM at most: enough threads for these elementwise
        // phases, and room left for kernels of other streams
        const int blocks = (int)std::max<int64_t>(
            1, std::min<int64_t>((int64_t)std::min(std::max(per_sm, 1), 2) * ctx->num_sms, (n + 255) / 256));
        uint32_t mq = (uint32_t)min_qdeg;
        int64_t nn_arg = n;
        void *args[] = {(void *)&rp, (void *)&col, (void *)&nn_arg, (void *)&mq, (void *)&deg, (void *)&alive,
                        (void *)&peel_list, (void *)&peel_removed, (void *)&d_rounds};
        BEEP_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)k_peel_fused, dim3(blocks), dim3(256), args, 0, s));
        ++ctx->launches;
    }
    tr.mark("peel");

    // Relabel by priority.
    const uint32_t maxdeg = (uint32_t)g->max_degree;
    int hb = 1;
    while (hb < 32 && ((uint64_t)1 << hb) <= (uint64_t)maxdeg)
        ++hb;
    unsigned long long *d_alive = d_removed + 1;
    BEEP_CUDA_TRY(cudaMemsetAsync(d_alive, 0, 8, s));
    if (n > 0) {
        k_prio_keys<<<gv, 256, 0, s>>>(deg, n, maxdeg, asc, pkey, pid, d_alive);
        ++ctx->launches;
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    size_t tb = 0;
    BEEP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, pkey, pkey2, pid, pid2, n, 0, hb, s));
    BEEP_TRY(ctx->grow(ctx->scratch, tb + 1024));
    BEEP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ctx->scratch.ptr, tb, pkey, pkey2, pid, pid2, n, 0, hb, s));
    // number of vertices that kept an edge
    ctx->h_pinned[1] = 0; // the copy below fills its low 4 bytes
    BEEP_CUDA_TRY(cudaMemcpyAsync(ctx->h_pinned, d_alive, 8, cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaMemcpyAsync(ctx->h_pinned + 1, d_rounds, 4, cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    const int64_t na = (int64_t)ctx->h_pinned[0];
    v->n = na;
    v->peel_rounds = std::max(1, (int)(uint32_t)ctx->h_pinned[1]);
    tr.mark("order");
    BEEP_TRY(ctx->grow(v->row_ptr, (size_t)(na + 1) * 4));
    BEEP_TRY(ctx->grow(v->orig, (size_t)(na > 0 ? na : 1) * 4));
    BEEP_TRY(ctx->grow(v->split, (size_t)(na > 0 ? na : 1) * 4));
    BEEP_CUDA_TRY(cudaMemsetAsync(rank, 0xff, (size_t)nn * 4, s));
    BEEP_CUDA_TRY(cudaMemsetAsync(new_deg, 0, (size_t)nn * 4, s));
    if (na > 0) {
        k_rank<<<grid_for(na, 256, ctx->num_sms), 256, 0, s>>>(pid2, na, v->orig.as<uint32_t>(), rank, deg,
                                                               new_deg);
        ++ctx->launches;
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    uint32_t *nrp = v->row_ptr.as<uint32_t>();
    tb = 0;
    BEEP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, new_deg, nrp, na + 1, s));
    BEEP_TRY(ctx->grow(ctx->scratch, tb + 1024));
    BEEP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(ctx->scratch.ptr, tb, new_deg, nrp, na + 1, s));
    // The view's entry count nrp[na] stays on the device: the buffers are
    // sized for all m input entries and the kernels read the count there.
    tr.mark("rank_scan");
    BEEP_TRY(ctx->grow(v->col, (size_t)(m > 0 ? m : 1) * 4));
    // rank bits: every rank is below na < 2^rb
    int rb = 1;
    while (rb < 32 && ((uint64_t)1 << rb) <= (uint64_t)na)
        ++rb;
    if (m > 0 && na > 0) {
        BEEP_CUDA_TRY(cudaMemsetAsync(d_nchunks, 0, 4, s));
        k_fill_keys<<<gv, 256, 0, s>>>(rp, col, rank, n, rb, ekeys, chunks, d_nchunks, ucap);
        k_fill_key_chunks<<<ctx->num_sms * 8, 256, 0, s>>>(col, rank, chunks, d_nchunks, ucap, rb, ekeys);
        ctx->launches += 2;
        BEEP_CUDA_TRY(cudaGetLastError());
    }
    tr.mark("fill");
    if (m > 0 && na > 0) {
        tb = 0;
        BEEP_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tb, ekeys, ekeys2, m, 0, 2 * rb, s));
        BEEP_TRY(ctx->grow(ctx->scratch, tb + 1024));
        BEEP_CUDA_TRY(cub::DeviceRadixSort::SortKeys(ctx->scratch.ptr, tb, ekeys, ekeys2, m, 0, 2 * rb, s));
        k_keys_low<<<grid_for(m, 256, ctx->num_sms), 256, 0, s>>>(ekeys2, nrp + na, rb, v->col.as<uint32_t>());
        ++ctx->launches;
        BEEP_CUDA_TRY(cudaGetLastError());
    }
    if (na > 0) {
        k_split<<<grid_for(na, 256, ctx->num_sms), 256, 0, s>>>(nrp, v->col.as<uint32_t>(), na,
                                                                v->split.as<uint32_t>());
        ++ctx->launches;
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    tr.mark("sort_split");
    return BEEP_OK;
}

} // namespace

beep_status get_view(Ctx *ctx, Graph *g, int32_t min_qdeg, int32_t asc, bool no_cache,
                     std::shared_ptr<View> *out, bool *built) {
    auto key = std::make_pair((int)min_qdeg, (int)asc);
    if (no_cache)
        g->views.erase(key);
    auto it = g->views.find(key);
    if (it != g->views.end()) {
        *out = it->second;
        if (built)
            *built = false;
        return BEEP_OK;
    }
    auto v = std::make_shared<View>();
    BEEP_TRY(build_view(ctx, g, min_qdeg, asc, v.get()));
    *out = v;
    g->views[key] = v;
    if (built)
        *built = true;
    return BEEP_OK;
}

} // namespace beep
