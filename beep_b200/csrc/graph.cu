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

// Row classes of the relabelled CSR (see the relabelled rows below).
constexpr int kRowClasses = 11;     // lengths 1, 2, 3-4, .., 129-256, 257-kHubTile, longer
constexpr uint32_t kHubTile = 4096; // entries of a hub tile (and of a block sort)
// vstat words: [0, kRowClasses) rows per class, then the hub tiles, the most
// tiles of one hub row and the peel rounds
constexpr int kVsTiles = kRowClasses, kVsMaxTiles = kRowClasses + 1, kVsRounds = kRowClasses + 2;
constexpr int kVsWords = 16;

__device__ __forceinline__ int row_class(uint32_t d) {
    if (d <= 1)
        return 0;
    if (d <= 256)
        return 32 - __clz((int)(d - 1)); // 2 -> 1, 3..4 -> 2, .., 129..256 -> 8
    return d <= kHubTile ? 9 : 10;
}

// Priority key (subgraph_matching.cuh:1299-1331, host_utils.cuh:230-246):
// ascending (degree, id) or descending degree with ties by ascending id.
// Vertices left with no edge get the largest key and are dropped.
// The key is the degree part alone; a stable radix sort of (key, id) pairs
// with ids in increasing order keeps ties by ascending id.
// vstat gets the kept vertices per row class and the hub tile counts.
__global__ void k_prio_keys(const uint32_t *__restrict__ deg, int64_t n, uint32_t maxdeg, int asc,
                            uint32_t *keys, uint32_t *ids, uint32_t *vstat) {
    __shared__ uint32_t hist[kRowClasses + 2];
    if (threadIdx.x < kRowClasses + 2)
        hist[threadIdx.x] = 0;
    __syncthreads();
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t d = deg[v];
        uint32_t k;
        if (d == 0) {
            k = maxdeg;
        } else {
            k = asc ? d - 1 : maxdeg - d;
            const int c = row_class(d);
            atomicAdd(&hist[c], 1u);
            if (c == kRowClasses - 1) {
                const uint32_t t = (d + kHubTile - 1) / kHubTile;
                atomicAdd(&hist[kVsTiles], t);
                atomicMax(&hist[kVsMaxTiles], t);
            }
        }
        keys[v] = k;
        ids[v] = (uint32_t)v;
    }
    __syncthreads();
    if (threadIdx.x < kRowClasses + 1 && hist[threadIdx.x])
        atomicAdd(&vstat[threadIdx.x], hist[threadIdx.x]);
    if (threadIdx.x == kVsMaxTiles && hist[threadIdx.x])
        atomicMax(&vstat[threadIdx.x], hist[threadIdx.x]);
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

// ---- relabelled rows --------------------------------------------------------
//
// New row j (input vertex v = orig[j]) holds rank[w] for every surviving
// neighbour w of v, in increasing order. Its length is v's degree after the
// peel, so the priority order makes the lengths monotone in j (rising for the
// ascending order, falling for the descending one) and every size class
// below is one contiguous range of rows. The rows are built in two steps:
// a gather that writes each row's entries, unordered, at its final place,
// then a sort of each row inside its own range, by size class: bitonic
// networks over 2..32 lanes of a warp (shuffles), over a warp's shared
// memory (up to 256 entries) or a block's (up to kHubTile), and for longer
// rows (hubs) sorted tiles of kHubTile entries merged in passes that all
// blocks of the GPU share.
// First row of class c and the rows it holds, from the class counts.
__device__ __forceinline__ uint32_t class_first(const uint32_t *cnt, int c, int asc) {
    uint32_t f = 0;
    for (int i = 0; i < kRowClasses; ++i)
        if (asc ? i < c : i > c)
            f += cnt[i];
    return f;
}

// Input row v's surviving entries, as new ids, at new row rank[v]'s place:
// rows of up to kSerialMax entries by one lane each, longer rows by chunks
// (k_view_fill_chunks) that reserve their part of the row with an atomic on
// the row's cursor.
__global__ void k_view_fill(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col,
                            const uint32_t *__restrict__ rank, int64_t n, const uint32_t *__restrict__ nrp,
                            uint32_t *vcol, RowChunk *chunks, unsigned *n_chunks, uint32_t cap) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n; base += warps * 32) {
        const int64_t v = base + lane;
        bool big = false;
        uint32_t b = 0, e = 0, rv = 0;
        if (v < n) {
            rv = rank[v];
            if (rv != 0xffffffffu) {
                b = rp[v];
                e = rp[v + 1];
                if (e - b > kSerialMax) {
                    big = true;
                } else {
                    uint32_t o = nrp[rv];
#pragma unroll 4
                    for (uint32_t k = b; k < e; ++k) {
                        const uint32_t r = rank[col[k]];
                        if (r != 0xffffffffu)
                            vcol[o++] = r;
                    }
                }
            }
        }
        push_chunks(big, rv, b, e, chunks, n_chunks, cap, lane);
    }
}

// A warp per chunk of kChunk = 32 x 32 entries: all loads first, then one
// atomic for the chunk's survivors, then the compacted stores.
__global__ void k_view_fill_chunks(const uint32_t *__restrict__ col, const uint32_t *__restrict__ rank,
                                   const RowChunk *__restrict__ chunks, const unsigned *__restrict__ n_chunks,
                                   uint32_t cap, const uint32_t *__restrict__ nrp, uint32_t *cur, uint32_t *vcol) {
    static_assert(kChunk == 32 * 32, "a lane holds kChunk / 32 entries");
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t nc = min(*n_chunks, cap);
    for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nc; c += warps) {
        const RowChunk ch = chunks[c];
        uint32_t r[32];
        uint32_t tot = 0;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const uint32_t k = ch.b + (uint32_t)(i * 32 + lane);
            r[i] = k < ch.e ? rank[col[k]] : 0xffffffffu;
        }
#pragma unroll
        for (int i = 0; i < 32; ++i)
            tot += (uint32_t)__popc(__ballot_sync(kFull, r[i] != 0xffffffffu));
        uint32_t o = 0;
        if (lane == 0 && tot)
            o = atomicAdd(&cur[ch.row], tot);
        o = nrp[ch.row] + __shfl_sync(kFull, o, 0);
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const unsigned bal = __ballot_sync(kFull, r[i] != 0xffffffffu);
            if (r[i] != 0xffffffffu)
                vcol[o + (uint32_t)__popc(bal & lt)] = r[i];
            o += (uint32_t)__popc(bal);
        }
    }
}

// Hub row h (new row h0 + h): its tile count, at htp[h + 1] (a scan turns
// them into each hub's first tile).
__global__ void k_hub_tiles(const uint32_t *__restrict__ nrp, uint32_t h0, uint32_t H, uint32_t *htp) {
    for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < H; h += gridDim.x * blockDim.x)
        htp[h + 1] = (nrp[h0 + h + 1] - nrp[h0 + h] + kHubTile - 1) / kHubTile;
}

// last h with htp[h] <= u (htp rising, htp[0] = 0 <= u)
__device__ __forceinline__ uint32_t hub_of(const uint32_t *__restrict__ htp, uint32_t H, uint32_t u) {
    uint32_t lo = 0, hi = H;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (htp[mid] <= u)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Bitonic sort, ascending, of s[0, S) (S a power of two) by `nt` threads
// numbered `t`; `sync` separates the stages.
template <typename Sync>
__device__ __forceinline__ void bitonic_shared(uint32_t *s, uint32_t S, uint32_t t, uint32_t nt, Sync sync) {
    for (uint32_t k = 2; k <= S; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t q = t; q < S / 2; q += nt) {
                const uint32_t i = 2 * q - (q & (j - 1)), l = i + j;
                const uint32_t a = s[i], b = s[l];
                if ((a > b) == ((i & k) == 0)) {
                    s[i] = b;
                    s[l] = a;
                }
            }
            sync();
        }
}

// One unit of the row sort: class c's rows [first, first + cnt) in units of
// (256 >> c) rows (c <= 5: a group of 2^c lanes per row), 8 rows (c = 6..8:
// a warp per row), one row (c = 9) or one hub tile (c = 10). Units are taken
// longest class first from a cursor, so the hubs' tiles start at once.
// Hub tiles go to out[]: the buffer that, after the merge passes, leaves the
// hub rows in vcol.
__global__ void __launch_bounds__(256) k_view_sort(const uint32_t *__restrict__ nrp, const uint32_t *__restrict__ vstat,
                                                   int asc, const uint32_t *__restrict__ htp, uint32_t *vcol,
                                                   uint32_t *out, unsigned *cursor) {
    __shared__ uint32_t buf[kHubTile];
    __shared__ uint32_t s_first[kRowClasses], s_cnt[kRowClasses], s_ustart[kRowClasses + 1];
    __shared__ uint32_t s_u;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        uint32_t cnt[kRowClasses];
        for (int c = 0; c < kRowClasses; ++c)
            cnt[c] = vstat[c];
        uint32_t acc = 0;
        for (int c = kRowClasses - 1; c >= 0; --c) {
            s_first[c] = class_first(cnt, c, asc);
            s_cnt[c] = cnt[c];
            s_ustart[c] = acc;
            uint32_t units = 0;
            if (c == 10)
                units = vstat[kVsTiles];
            else if (c == 9)
                units = cnt[c];
            else if (c >= 6)
                units = (cnt[c] + 7) / 8;
            else if (c >= 1)
                units = (cnt[c] + (256u >> c) - 1) / (256u >> c);
            acc += units;
        }
        s_ustart[kRowClasses] = acc; // total
    }
    __syncthreads();
    const uint32_t total = s_ustart[kRowClasses];
    for (;;) {
        if (threadIdx.x == 0)
            s_u = atomicAdd(cursor, 1u);
        __syncthreads();
        const uint32_t u = s_u;
        __syncthreads();
        if (u >= total)
            break;
        int c = kRowClasses - 1; // classes hold units in falling order
        while (c > 0 && u >= s_ustart[c - 1])
            --c;
        const uint32_t lu = u - s_ustart[c];
        const uint32_t first = s_first[c], cend = first + s_cnt[c];
        if (c >= 9) {
            uint32_t j, lo, len;
            uint32_t *dst = vcol;
            if (c == 10) {
                const uint32_t H = s_cnt[10];
                const uint32_t h = hub_of(htp, H, lu);
                j = first + h;
                lo = nrp[j] + (lu - htp[h]) * kHubTile;
                len = min(kHubTile, nrp[j + 1] - lo);
                dst = out;
            } else {
                j = first + lu;
                lo = nrp[j];
                len = nrp[j + 1] - lo;
            }
            uint32_t S = 512;
            while (S < len)
                S <<= 1;
            for (uint32_t i = threadIdx.x; i < S; i += blockDim.x)
                buf[i] = i < len ? vcol[lo + i] : 0xffffffffu;
            __syncthreads();
            bitonic_shared(buf, S, threadIdx.x, blockDim.x, [] { __syncthreads(); });
            for (uint32_t i = threadIdx.x; i < len; i += blockDim.x)
                dst[lo + i] = buf[i];
            __syncthreads();
        } else if (c >= 6) {
            const uint32_t j = first + lu * 8 + (uint32_t)warp;
            if (j < cend) {
                const uint32_t S = 1u << c, lo = nrp[j], len = nrp[j + 1] - lo;
                uint32_t *s = buf + warp * 256;
                for (uint32_t i = lane; i < S; i += 32)
                    s[i] = i < len ? vcol[lo + i] : 0xffffffffu;
                __syncwarp();
                bitonic_shared(s, S, lane, 32, [] { __syncwarp(); });
                for (uint32_t i = lane; i < len; i += 32)
                    vcol[lo + i] = s[i];
            }
        } else if (c >= 1) {
            // groups of P = 2^c lanes, a row each
            const uint32_t P = 1u << c, g = (uint32_t)lane >> c, i = (uint32_t)lane & (P - 1);
            const uint32_t j = first + lu * (256u >> c) + (uint32_t)warp * (32u >> c) + g;
            uint32_t lo = 0, len = 0;
            if (j < cend) {
                lo = nrp[j];
                len = nrp[j + 1] - lo;
            }
            uint32_t x = i < len ? vcol[lo + i] : 0xffffffffu;
            for (uint32_t k = 2; k <= P; k <<= 1)
                for (uint32_t jj = k >> 1; jj > 0; jj >>= 1) {
                    const uint32_t y = __shfl_xor_sync(kFull, x, (int)jj);
                    const bool keep_min = ((i & jj) == 0) == ((i & k) == 0);
                    x = keep_min ? min(x, y) : max(x, y);
                }
            if (i < len)
                vcol[lo + i] = x;
        }
    }
}

// Merge-path split: how many of A's entries are among the first d of the
// merge of A (na) and B (nb); entries are distinct.
__device__ __forceinline__ uint32_t merge_split(const uint32_t *A, uint32_t na, const uint32_t *B, uint32_t nb,
                                                uint32_t d) {
    uint32_t lo = d > nb ? d - nb : 0u, hi = min(d, na);
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (A[mid] < B[d - 1 - mid])
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Merge pass p over the hub rows: sorted runs of kHubTile << p entries are
// merged in pairs, src -> dst. Unit u is output window u - htp[h] (kHubTile
// entries) of hub h: its parts of the two runs are found by a merge-path
// search, staged in shared memory, and every thread merges 16 outputs. A run
// without a partner is copied.
__global__ void __launch_bounds__(256) k_view_merge(const uint32_t *__restrict__ nrp, uint32_t h0, uint32_t H,
                                                    const uint32_t *__restrict__ htp, int p,
                                                    const uint32_t *__restrict__ src, uint32_t *dst) {
    __shared__ uint32_t sm[kHubTile];
    __shared__ uint32_t s_split[2];
    static_assert(kHubTile == 256 * 16, "16 outputs a thread");
    const uint32_t TT = htp[H];
    for (uint32_t u = blockIdx.x; u < TT; u += gridDim.x) {
        const uint32_t h = hub_of(htp, H, u), w = u - htp[h];
        const uint32_t rb = nrp[h0 + h], L = nrp[h0 + h + 1] - rb;
        const uint64_t R = (uint64_t)kHubTile << p;
        const uint64_t ps = (uint64_t)(w >> (p + 1)) * 2 * R; // the pair's first entry
        const uint64_t left = (uint64_t)L - ps; // entries from the pair's first on (> 0)
        const uint32_t al = (uint32_t)(left < R ? left : R);
        const uint32_t bl = (uint32_t)(left - al < R ? left - al : R);
        const uint32_t d0 = (uint32_t)((uint64_t)w * kHubTile - ps), d1 = min(d0 + kHubTile, al + bl);
        const uint32_t *A = src + rb + ps, *B = A + al;
        if (threadIdx.x < 2)
            s_split[threadIdx.x] = merge_split(A, al, B, bl, threadIdx.x ? d1 : d0);
        __syncthreads();
        const uint32_t a0 = s_split[0], a1 = s_split[1], b0 = d0 - a0, b1 = d1 - a1;
        const uint32_t na = a1 - a0, nb = b1 - b0;
        for (uint32_t i = threadIdx.x; i < na; i += blockDim.x)
            sm[i] = A[a0 + i];
        for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x)
            sm[na + i] = B[b0 + i];
        __syncthreads();
        const uint32_t n = na + nb, dd = threadIdx.x * 16;
        if (dd < n) {
            const uint32_t de = min(dd + 16, n);
            uint32_t ai = merge_split(sm, na, sm + na, nb, dd), bi = dd - ai;
            uint32_t *o = dst + rb + ps + d0;
            for (uint32_t q = dd; q < de; ++q) {
                const bool take_a = bi >= nb || (ai < na && sm[ai] < sm[na + bi]);
                o[q] = take_a ? sm[ai++] : sm[na + bi++];
            }
        }
        __syncthreads();
    }
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
                               (size_t)nn * 4, (size_t)nn * 4, (size_t)nn * 4, mm * 4, cap * sizeof(RowChunk), 16,
                               (size_t)nn * 4, kPeelMaxRounds * 8, kVsWords * 4, ((size_t)nn + 1) * 4});
    BEEP_TRY(ctx->grow(ctx->scratch2, need));
    Carve cv(ctx->scratch2.ptr);
    uint32_t *deg = cv.take<uint32_t>(nn);
    uint8_t *alive = cv.take<uint8_t>(nn);
    uint32_t *rank = cv.take<uint32_t>(nn);
    uint32_t *pkey = cv.take<uint32_t>(nn), *pid = cv.take<uint32_t>(nn);
    uint32_t *pkey2 = cv.take<uint32_t>(nn), *pid2 = cv.take<uint32_t>(nn);
    uint32_t *new_deg = cv.take<uint32_t>(nn);
    uint32_t *hub_tmp = cv.take<uint32_t>(mm); // the hub rows' other merge buffer
    RowChunk *chunks = cv.take<RowChunk>(cap);
    unsigned *d_nchunks = cv.take<unsigned>(4); // [0] chunk count, [1] row sort cursor
    uint32_t *peel_list = cv.take<uint32_t>(nn);
    unsigned long long *peel_removed = cv.take<unsigned long long>(kPeelMaxRounds);
    uint32_t *vstat = cv.take<uint32_t>(kVsWords);
    uint32_t *htp = cv.take<uint32_t>((size_t)nn + 1); // first tile of every hub row
    const uint32_t ucap = (uint32_t)std::min<size_t>(cap, 0xffffffffu);

    PhaseTrace tr("view", s);
    const int gv = grid_for(n, 256, ctx->num_sms);
    if (n > 0) {
        k_peel_init<<<gv, 256, 0, s>>>(rp, n, deg, alive);
        ++ctx->launches;
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    // Iterated peel, all rounds in one cooperative launch (no host round trip
    // per round).
    BEEP_CUDA_TRY(cudaMemsetAsync(vstat, 0, kVsWords * 4, s));
    int *d_rounds = reinterpret_cast<int *>(vstat + kVsRounds);
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
    if (n > 0) {
        k_prio_keys<<<gv, 256, 0, s>>>(deg, n, maxdeg, asc, pkey, pid, vstat);
        ++ctx->launches;
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    size_t tb = 0;
    BEEP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, pkey, pkey2, pid, pid2, n, 0, hb, s));
    BEEP_TRY(ctx->grow(ctx->scratch, tb + 1024));
    BEEP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ctx->scratch.ptr, tb, pkey, pkey2, pid, pid2, n, 0, hb, s));
    // rows per class (their sum: the vertices that kept an edge), hub tiles,
    // peel rounds
    static_assert(kVsWords * 4 <= 64, "the pinned mirror holds 64 bytes");
    uint32_t *hv = reinterpret_cast<uint32_t *>(ctx->h_pinned);
    BEEP_CUDA_TRY(cudaMemcpyAsync(hv, vstat, kVsWords * 4, cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    uint32_t cls[kRowClasses];
    int64_t na = 0;
    for (int c = 0; c < kRowClasses; ++c) {
        cls[c] = hv[c];
        na += cls[c];
    }
    const uint32_t hub_tiles = hv[kVsTiles], hub_max_tiles = hv[kVsMaxTiles];
    v->n = na;
    v->peel_rounds = std::max(1, (int)hv[kVsRounds]);
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
    uint32_t *vcol = v->col.as<uint32_t>();
    if (m > 0 && na > 0) {
        // new_deg is free after the scan: the long rows' fill cursors
        BEEP_CUDA_TRY(cudaMemsetAsync(new_deg, 0, (size_t)na * 4, s));
        BEEP_CUDA_TRY(cudaMemsetAsync(d_nchunks, 0, 8, s));
        k_view_fill<<<gv, 256, 0, s>>>(rp, col, rank, n, nrp, vcol, chunks, d_nchunks, ucap);
        k_view_fill_chunks<<<ctx->num_sms * 8, 256, 0, s>>>(col, rank, chunks, d_nchunks, ucap, nrp, new_deg, vcol);
        ctx->launches += 2;
        BEEP_CUDA_TRY(cudaGetLastError());
    }
    tr.mark("fill");
    if (m > 0 && na > 0) {
        // hub rows: [h0, h0 + H) of the new order; their tiles go through
        // `passes` merges, so the tile sort writes them where the last
        // merge pass leaves them in vcol
        const uint32_t H = cls[kRowClasses - 1];
        const uint32_t h0 = asc ? (uint32_t)(na - H) : 0u;
        int passes = 0;
        while (((uint32_t)1 << passes) < hub_max_tiles)
            ++passes;
        uint32_t *bufs[2] = {vcol, hub_tmp};
        if (H > 0) {
            BEEP_CUDA_TRY(cudaMemsetAsync(htp, 0, 4, s));
            k_hub_tiles<<<grid_for(H, 256, ctx->num_sms), 256, 0, s>>>(nrp, h0, H, htp);
            ++ctx->launches;
            BEEP_CUDA_TRY(cudaGetLastError());
            tb = 0;
            BEEP_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, tb, htp + 1, htp + 1, H, s));
            BEEP_TRY(ctx->grow(ctx->scratch, tb + 1024));
            BEEP_CUDA_TRY(cub::DeviceScan::InclusiveSum(ctx->scratch.ptr, tb, htp + 1, htp + 1, H, s));
        }
        uint64_t units = hub_tiles + cls[9];
        for (int c = 1; c <= 8; ++c)
            units += c >= 6 ? (cls[c] + 7) / 8 : (cls[c] + (256u >> c) - 1) / (256u >> c);
        if (units > 0) {
            int per_sm = 0;
            BEEP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_view_sort, 256, 0));
            const int64_t blocks = std::min<int64_t>((int64_t)std::max(per_sm, 1) * ctx->num_sms, (int64_t)units);
            k_view_sort<<<(unsigned)blocks, 256, 0, s>>>(nrp, vstat, asc, htp, vcol, bufs[passes & 1],
                                                         d_nchunks + 1);
            ++ctx->launches;
            BEEP_CUDA_TRY(cudaGetLastError());
        }
        const unsigned mgrid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(hub_tiles, ctx->num_sms * 8ull));
        for (int p = 0; p < passes; ++p) {
            k_view_merge<<<mgrid, 256, 0, s>>>(nrp, h0, H, htp, p, bufs[(passes - p) & 1],
                                               bufs[(passes - p - 1) & 1]);
            ++ctx->launches;
            BEEP_CUDA_TRY(cudaGetLastError());
        }
    }
    tr.mark("sort");
    if (na > 0) {
        k_split<<<grid_for(na, 256, ctx->num_sms), 256, 0, s>>>(nrp, vcol, na, v->split.as<uint32_t>());
        ++ctx->launches;
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    tr.mark("split");
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
