// count.cu — the bitmap-intersection DFS kernels and their driver.
//
// Reference hot path: sgm_kernel_central_node_function
// (subgraph_matching/sgm_kernelsLD.cuh:7-273) with encode, count_tri,
// get_newIndex, backtrack and compute_intersection
// (subgraph_matching/include/device_utils.cuh:99-326, 426-456). Per root the
// reference builds the deg x deg bitmap of its oriented neighbour list in
// global memory and runs a 16-lane-partition DFS with a serial __ffs scan by
// lane 0 and a global-memory candidate stack.
//
// Here, per root r with domain list A (its neighbours, or only its later
// neighbours when every position must follow the root):
//   - row i of the bitmap holds the neighbours of A[i] inside A. Every edge
//     inside A is found once, from the lower-priority endpoint, by searching
//     that endpoint's higher-priority list against A;
//   - the DFS keeps no candidate stack: the candidate words of a level are
//     recomputed chunk by chunk (AND of the back-edge rows, minus used
//     vertices, minus bits below the symmetry bound) while the enumeration
//     state lives in registers, unrolled over the compile-time depth;
//   - the next candidate comes from __ballot_sync + __ffs across the warp;
//   - the last level is a popcount (as in the reference).
// Three tiers by domain size D:
//   small   D <= 64   warp per root, 64-bit rows in shared memory, one lane per
//                     level-1 vertex (thread-level DFS);
//   medium  D <= 1024 block per root, rows in shared memory, warps take
//                     level-1 vertices from a shared counter;
//   large   D > 1024  rows in a global arena; one launch builds the rows of a
//                     batch of roots, a second spreads the (root, level-1 vertex)
//                     tasks over every warp of the GPU.
#include <algorithm>
#include <cmath>
#include <mutex>

#include <cub/cub.cuh>

#include "internal.h"

namespace beep {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kSmallMaxD = 64;
constexpr int kMediumAMaxD = 256;
constexpr int kMediumMaxD = 1024;

struct ViewDev {
    const uint32_t *__restrict__ rp;
    const uint32_t *__restrict__ col;
    const uint32_t *__restrict__ split;
    const uint32_t *__restrict__ orig;
};

struct EnumDev {
    int32_t *out;            // k * K tuples
    unsigned long long *n;   // tuples reserved so far
    unsigned long long k;
};

// Plan fields the DFS reads, held in registers.
struct Lp {
    uint32_t back[kMaxQ];
    uint32_t sym[kMaxQ];
};

__device__ __forceinline__ Lp load_lp(const DevPlan &pl) {
    Lp lp;
#pragma unroll
    for (int i = 0; i < kMaxQ; ++i) {
        lp.back[i] = pl.back[i];
        lp.sym[i] = pl.sym[i];
    }
    return lp;
}

// Domain of root r: list A = col[beg, beg + D); level-1 index starts at j0.
__device__ __forceinline__ void root_domain(const ViewDev &v, const DevPlan &pl, uint32_t r, uint32_t &beg,
                                            uint32_t &D, uint32_t &j0) {
    const uint32_t b = v.rp[r], e = v.rp[r + 1], sp = v.split[r];
    if (pl.restricted) {
        beg = b + sp;
        D = e - b - sp;
        j0 = 0;
    } else {
        beg = b;
        D = e - b;
        // position 1 symmetric to the root: only neighbours after the root
        // (sgm_kernelsLD.cuh:60)
        j0 = pl.pos1_after_root ? sp : 0;
    }
}

// Higher-priority list of u and the part of A it can meet.
__device__ __forceinline__ void hd_range(const ViewDev &v, int asc, uint32_t u, uint32_t i, uint32_t D,
                                         uint32_t &hb, uint32_t &he, uint32_t &xb, uint32_t &xe) {
    const uint32_t ub = v.rp[u], ue = v.rp[u + 1], us = v.split[u];
    if (asc) {
        hb = ub + us;
        he = ue;
        xb = i + 1;
        xe = D;
    } else {
        hb = ub;
        he = ub + us;
        xb = 0;
        xe = i;
    }
}

__device__ __forceinline__ uint32_t lower_bound_g(const uint32_t *__restrict__ a, uint32_t lo, uint32_t hi,
                                                  uint32_t key) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Index of key in sorted a[lo, hi) or -1.
__device__ __forceinline__ int find_idx(const uint32_t *a, uint32_t lo, uint32_t hi, uint32_t key) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t x = a[mid];
        if (x == key)
            return (int)mid;
        if (x < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return -1;
}

// ---------------------------------------------------------------------------
// enumeration output
// ---------------------------------------------------------------------------
struct EnumCtx {
    EnumDev en;
    const uint32_t *A; // domain list (new ids)
    const uint32_t *orig;
    uint32_t root;
    int32_t K;
    int32_t order[kMaxQ];
};

__device__ __forceinline__ void emit_bits(const EnumCtx &ec, const uint32_t (&x)[kMaxQ], int P, uint64_t bits,
                                          uint32_t base) {
    if (!bits)
        return;
    if (*(volatile unsigned long long *)ec.en.n >= ec.en.k)
        return;
    const unsigned long long c = (unsigned long long)__popcll(bits);
    unsigned long long slot = atomicAdd(ec.en.n, c);
    while (bits && slot < ec.en.k) {
        const int b = __ffsll((long long)bits) - 1;
        bits &= bits - 1;
        int32_t *t = ec.en.out + slot * (unsigned long long)ec.K;
        t[ec.order[0]] = (int32_t)ec.orig[ec.root];
        for (int q = 1; q < P; ++q)
            t[ec.order[q]] = (int32_t)ec.orig[ec.A[x[q]]];
        t[ec.order[P]] = (int32_t)ec.orig[ec.A[base + b]];
        ++slot;
    }
}

// ---------------------------------------------------------------------------
// thread-level DFS on 64-bit rows (D <= 64)
// ---------------------------------------------------------------------------
template <int P, int DEND, bool ENUM>
__device__ __forceinline__ void dfs_thread(const Lp &lp, const uint64_t *rows, uint64_t all, uint32_t (&x)[kMaxQ],
                                           unsigned long long &cnt, const EnumCtx &ec) {
    uint64_t c = all;
    const uint32_t bk = lp.back[P], sy = lp.sym[P];
#pragma unroll
    for (int q = 1; q < P; ++q) {
        if (bk >> q & 1u)
            c &= rows[x[q]];
        c &= ~(1ull << x[q]);
        if (sy >> q & 1u)
            c &= ~((2ull << x[q]) - 1ull); // keep bits above x[q]
    }
    if constexpr (P == DEND - 1) {
        if constexpr (ENUM)
            emit_bits(ec, x, P, c, 0);
        cnt += (unsigned long long)__popcll(c);
    } else {
        while (c) {
            const int b = __ffsll((long long)c) - 1;
            c &= c - 1;
            x[P] = (uint32_t)b;
            dfs_thread<P + 1, DEND, ENUM>(lp, rows, all, x, cnt, ec);
        }
    }
}

// ---------------------------------------------------------------------------
// warp-level DFS on rows of W 32-bit words (lane k holds word k of a chunk)
// ---------------------------------------------------------------------------
template <int P, int DEND, bool ENUM>
__device__ __forceinline__ void dfs_warp(const Lp &lp, const uint32_t *bm, uint32_t W, uint32_t D,
                                         uint32_t (&x)[kMaxQ], unsigned long long &cnt, int lane, const EnumCtx &ec) {
    const uint32_t bk = lp.back[P], sy = lp.sym[P];
    uint32_t lo = 0;
#pragma unroll
    for (int q = 1; q < P; ++q)
        if (sy >> q & 1u)
            lo = max(lo, x[q] + 1);
    const uint32_t nch = (W + 31) >> 5;
    const uint32_t tail = D & 31;
    for (uint32_t ch = lo >> 10; ch < nch; ++ch) {
        const uint32_t k = (ch << 5) + lane;
        uint32_t w = 0;
        if (k < W) {
            w = (k + 1 < W || tail == 0) ? kFull : ((1u << tail) - 1u);
#pragma unroll
            for (int q = 1; q < P; ++q) {
                if (bk >> q & 1u)
                    w &= bm[(size_t)x[q] * W + k];
                if ((x[q] >> 5) == k)
                    w &= ~(1u << (x[q] & 31));
            }
            const uint32_t lw = lo >> 5;
            if (lw > k)
                w = 0;
            else if (lw == k)
                w &= ~((1u << (lo & 31)) - 1u);
        }
        if constexpr (P == DEND - 1) {
            if constexpr (ENUM)
                emit_bits(ec, x, P, (uint64_t)w, k << 5);
            cnt += (unsigned long long)__popc(w);
        } else {
            unsigned bal = __ballot_sync(kFull, w != 0);
            while (bal) {
                const int L = __ffs(bal) - 1;
                const uint32_t ww = __shfl_sync(kFull, w, L);
                const int b = __ffs(ww) - 1;
                if (lane == L)
                    w &= w - 1;
                x[P] = (((ch << 5) + (uint32_t)L) << 5) + (uint32_t)b;
                dfs_warp<P + 1, DEND, ENUM>(lp, bm, W, D, x, cnt, lane, ec);
                bal = __ballot_sync(kFull, w != 0);
            }
        }
    }
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ void make_ec(EnumCtx &ec, const EnumDev &en, const DevPlan &pl, const ViewDev &v) {
    ec.en = en;
    ec.orig = v.orig;
    ec.K = pl.K;
#pragma unroll
    for (int i = 0; i < kMaxQ; ++i)
        ec.order[i] = pl.order[i];
}

// ---------------------------------------------------------------------------
// Row building, flattened over the elements to search so that every thread of
// the group stays busy whatever the row lengths:
//   1. per row i: the part of A[i]'s higher-priority list that lies inside
//      [min, max] of the A entries it can meet (two binary searches);
//   2. exclusive prefix of those lengths;
//   3. each thread takes list elements t = tid, tid + nthr, ...: finds its row
//      by binary search on the prefix, loads the element (consecutive t read
//      consecutive addresses) and binary-searches it in A, setting both bits
//      of every edge found.
// Used by a warp (small tier), a block (medium tier) or a block on a chunk of
// rows (large tier).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t upper_bound_g(const uint32_t *__restrict__ a, uint32_t lo, uint32_t hi,
                                                  uint32_t key) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Exclusive prefix of buf[0, R) in place, total in buf[R]; one warp.
__device__ __forceinline__ void warp_excl_scan(uint32_t *buf, uint32_t R, int lane) {
    uint32_t carry = 0;
    for (uint32_t base = 0; base < R; base += 32) {
        const uint32_t idx = base + lane;
        const uint32_t x = idx < R ? buf[idx] : 0u;
        uint32_t inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, inc, o);
            if (lane >= o)
                inc += y;
        }
        if (idx < R)
            buf[idx] = carry + inc - x;
        carry += __shfl_sync(kFull, inc, 31);
    }
    if (lane == 0)
        buf[R] = carry;
}

template <bool BLOCK> __device__ __forceinline__ void group_sync() {
    if constexpr (BLOCK)
        __syncthreads();
    else
        __syncwarp();
}

template <bool BLOCK, typename SetFn>
__device__ __forceinline__ void build_rows_flat(const ViewDev &v, int asc, const uint32_t *A, uint32_t D,
                                                uint32_t i0, uint32_t i1, uint32_t *s_hb, uint32_t *s_pre,
                                                uint32_t tid, uint32_t nthr, SetFn set) {
    const uint32_t R = i1 - i0;
    for (uint32_t r = tid; r < R; r += nthr) {
        const uint32_t i = i0 + r;
        uint32_t hb, he, xb, xe, c = 0;
        hd_range(v, asc, A[i], i, D, hb, he, xb, xe);
        if (xb < xe && hb < he) {
            const uint32_t lo = lower_bound_g(v.col, hb, he, A[xb]);
            const uint32_t hi = upper_bound_g(v.col, lo, he, A[xe - 1]);
            hb = lo;
            c = hi - lo;
        }
        s_hb[r] = hb;
        s_pre[r] = c;
    }
    group_sync<BLOCK>();
    if (tid < 32)
        warp_excl_scan(s_pre, R, (int)tid);
    group_sync<BLOCK>();
    const uint32_t T = s_pre[R];
    for (uint32_t t = tid; t < T; t += nthr) {
        // row r: last with s_pre[r] <= t
        uint32_t lo = 0, hi = R;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s_pre[mid] <= t)
                lo = mid;
            else
                hi = mid;
        }
        const uint32_t i = i0 + lo;
        const uint32_t w = v.col[s_hb[lo] + (t - s_pre[lo])];
        const uint32_t xb = asc ? i + 1 : 0, xe = asc ? D : i;
        const int k = find_idx(A, xb, xe, w);
        if (k >= 0)
            set(i, (uint32_t)k);
    }
}

// ---------------------------------------------------------------------------
// small tier: warp per root
// ---------------------------------------------------------------------------
constexpr int kSmallWarps = 8;

template <int DEND, bool ENUM>
__global__ void __launch_bounds__(kSmallWarps * 32) k_small(ViewDev v, DevPlan pl, const uint32_t *__restrict__ roots,
                                                           uint32_t nroots, int rev, unsigned long long *counter,
                                                           EnumDev en) {
    __shared__ uint64_t s_rows[kSmallWarps][kSmallMaxD];
    __shared__ uint32_t s_A[kSmallWarps][kSmallMaxD];
    __shared__ uint32_t s_hb[kSmallWarps][kSmallMaxD];
    __shared__ uint32_t s_pre[kSmallWarps][kSmallMaxD + 1];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const Lp lp = load_lp(pl);
    uint64_t *rows = s_rows[wib];
    uint32_t *A = s_A[wib];
    EnumCtx ec;
    if constexpr (ENUM)
        make_ec(ec, en, pl, v);
    unsigned long long cnt = 0;
    for (uint32_t ri = blockIdx.x * kSmallWarps + wib; ri < nroots; ri += gridDim.x * kSmallWarps) {
        const uint32_t r = roots[rev ? nroots - 1 - ri : ri];
        uint32_t beg, D, j0;
        root_domain(v, pl, r, beg, D, j0);
        for (uint32_t i = lane; i < D; i += 32) {
            A[i] = v.col[beg + i];
            rows[i] = 0;
        }
        __syncwarp();
        build_rows_flat<false>(v, pl.asc, A, D, 0, D, s_hb[wib], s_pre[wib], (uint32_t)lane, 32u,
                               [&](uint32_t i, uint32_t k) {
                                   atomicOr((unsigned long long *)&rows[i], 1ull << k);
                                   atomicOr((unsigned long long *)&rows[k], 1ull << i);
                               });
        __syncwarp();
        const uint64_t all = (D >= 64) ? ~0ull : ((1ull << D) - 1ull);
        if constexpr (ENUM) {
            ec.A = A;
            ec.root = r;
        }
        for (uint32_t j = j0 + lane; j < D; j += 32) {
            uint32_t x[kMaxQ];
            x[1] = j;
            dfs_thread<2, DEND, ENUM>(lp, rows, all, x, cnt, ec);
        }
        __syncwarp();
    }
    cnt = warp_sum(cnt);
    if (lane == 0 && cnt)
        atomicAdd(counter, cnt);
}

// ---------------------------------------------------------------------------
// medium tier: block per root, bitmap in shared memory
// ---------------------------------------------------------------------------
template <int DEND, bool ENUM>
__global__ void __launch_bounds__(1024) k_medium(ViewDev v, DevPlan pl, const uint32_t *__restrict__ roots,
                                                uint32_t nroots, int rev, unsigned *cursor,
                                                unsigned long long *counter, EnumDev en, uint32_t maxD) {
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t s_ri, s_j;
    const int lane = threadIdx.x & 31;
    const Lp lp = load_lp(pl);
    const uint32_t pad = (maxD + 4) & ~3u;
    uint32_t *A = sm;
    uint32_t *s_hb = sm + pad;
    uint32_t *s_pre = sm + 2 * pad;
    uint32_t *rows = sm + 3 * pad;
    EnumCtx ec;
    if constexpr (ENUM)
        make_ec(ec, en, pl, v);
    unsigned long long cnt = 0;
    for (;;) {
        if (threadIdx.x == 0)
            s_ri = atomicAdd(cursor, 1u);
        __syncthreads();
        const uint32_t ri = s_ri;
        if (ri >= nroots)
            break;
        const uint32_t r = roots[rev ? nroots - 1 - ri : ri];
        uint32_t beg, D, j0;
        root_domain(v, pl, r, beg, D, j0);
        const uint32_t W = (D + 31) >> 5;
        for (uint32_t i = threadIdx.x; i < D; i += blockDim.x)
            A[i] = v.col[beg + i];
        for (uint32_t i = threadIdx.x; i < D * W; i += blockDim.x)
            rows[i] = 0;
        if (threadIdx.x == 0)
            s_j = j0;
        __syncthreads();
        build_rows_flat<true>(v, pl.asc, A, D, 0, D, s_hb, s_pre, threadIdx.x, blockDim.x,
                              [&](uint32_t i, uint32_t k) {
                                  atomicOr(&rows[(size_t)i * W + (k >> 5)], 1u << (k & 31));
                                  atomicOr(&rows[(size_t)k * W + (i >> 5)], 1u << (i & 31));
                              });
        __syncthreads();
        if constexpr (ENUM) {
            ec.A = A;
            ec.root = r;
        }
        for (;;) {
            uint32_t j = 0;
            if (lane == 0)
                j = atomicAdd(&s_j, 1u);
            j = __shfl_sync(kFull, j, 0);
            if (j >= D)
                break;
            uint32_t x[kMaxQ];
            x[1] = j;
            dfs_warp<2, DEND, ENUM>(lp, rows, W, D, x, cnt, lane, ec);
        }
        __syncthreads();
    }
    cnt = warp_sum(cnt);
    if (lane == 0 && cnt)
        atomicAdd(counter, cnt);
}

// ---------------------------------------------------------------------------
// large tier: rows of a batch of roots in a global arena
// ---------------------------------------------------------------------------
struct Batch {
    const uint32_t *root;    // [nb]
    const uint64_t *off;     // [nb] word offset of the root's rows in the arena
    const uint32_t *cstart;  // [nb+1] prefix of row chunks
    const uint32_t *tstart;  // [nb+1] prefix of DFS tasks (level-1 vertices)
    uint32_t nb;
};

constexpr uint32_t kRowsPerChunk = 256;
constexpr uint32_t kLargeSmemA = 48 * 1024; // domain entries staged in shared memory

__device__ __forceinline__ uint32_t find_batch(const uint32_t *__restrict__ start, uint32_t nb, uint32_t t) {
    // last b with start[b] <= t
    uint32_t lo = 0, hi = nb;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (start[mid] <= t)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(512) k_large_rows(ViewDev v, DevPlan pl, Batch bt, uint32_t *arena,
                                                    unsigned *cursor) {
    extern __shared__ __align__(16) uint32_t sA[];
    __shared__ uint32_t s_c;
    __shared__ uint32_t s_hb[kRowsPerChunk], s_pre[kRowsPerChunk + 1];
    const uint32_t total = bt.cstart[bt.nb];
    for (;;) {
        if (threadIdx.x == 0)
            s_c = atomicAdd(cursor, 1u);
        __syncthreads();
        const uint32_t c = s_c;
        if (c >= total)
            break;
        const uint32_t b = find_batch(bt.cstart, bt.nb, c);
        const uint32_t r = bt.root[b];
        uint32_t beg, D, j0;
        root_domain(v, pl, r, beg, D, j0);
        const uint32_t W = (D + 31) >> 5;
        uint32_t *rows = arena + bt.off[b];
        const uint32_t i0 = (c - bt.cstart[b]) * kRowsPerChunk;
        const uint32_t i1 = min(D, i0 + kRowsPerChunk);
        const uint32_t *A = v.col + beg;
        if (D <= kLargeSmemA) {
            for (uint32_t i = threadIdx.x; i < D; i += blockDim.x)
                sA[i] = A[i];
            __syncthreads();
            A = sA;
        }
        build_rows_flat<true>(v, pl.asc, A, D, i0, i1, s_hb, s_pre, threadIdx.x, blockDim.x,
                              [&](uint32_t i, uint32_t k) {
                                  atomicOr(&rows[(size_t)i * W + (k >> 5)], 1u << (k & 31));
                                  atomicOr(&rows[(size_t)k * W + (i >> 5)], 1u << (i & 31));
                              });
        __syncthreads();
    }
}

template <int DEND, bool ENUM>
__global__ void __launch_bounds__(256) k_large_dfs(ViewDev v, DevPlan pl, Batch bt, const uint32_t *arena,
                                                   unsigned *cursor, unsigned long long *counter, EnumDev en) {
    const int lane = threadIdx.x & 31;
    const Lp lp = load_lp(pl);
    const uint32_t total = bt.tstart[bt.nb];
    EnumCtx ec;
    if constexpr (ENUM)
        make_ec(ec, en, pl, v);
    unsigned long long cnt = 0;
    for (;;) {
        uint32_t t = 0;
        if (lane == 0)
            t = atomicAdd(cursor, 1u);
        t = __shfl_sync(kFull, t, 0);
        if (t >= total)
            break;
        const uint32_t b = find_batch(bt.tstart, bt.nb, t);
        const uint32_t r = bt.root[b];
        uint32_t beg, D, j0;
        root_domain(v, pl, r, beg, D, j0);
        const uint32_t W = (D + 31) >> 5;
        if constexpr (ENUM) {
            ec.A = v.col + beg;
            ec.root = r;
        }
        uint32_t x[kMaxQ];
        x[1] = j0 + (t - bt.tstart[b]);
        dfs_warp<2, DEND, ENUM>(lp, arena + bt.off[b], W, D, x, cnt, lane, ec);
    }
    cnt = warp_sum(cnt);
    if (lane == 0 && cnt)
        atomicAdd(counter, cnt);
}

// ---------------------------------------------------------------------------
// root classification
// ---------------------------------------------------------------------------
// tier: 0 none, 1 small, 2 medium (D <= 256), 3 medium (D <= 1024), 4 large. Also accumulates the adjacency
// bytes the kernels must read for the roofline.
__global__ void k_classify(ViewDev v, DevPlan pl, int64_t n, uint32_t min_deg, uint32_t cap_deg, uint8_t *tier,
                           uint32_t *dom, unsigned *tier_max) {
    uint32_t mx[4] = {0, 0, 0, 0};
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t deg = v.rp[r + 1] - v.rp[r];
        uint32_t beg, D, j0;
        root_domain(v, pl, (uint32_t)r, beg, D, j0);
        uint8_t t = 0;
        // roots: degree in [max_qdeg, cap) (subgraph_matching.cuh:1086-1098);
        // enough domain vertices for the other dend-1 positions and at least
        // one level-1 vertex.
        if (deg >= min_deg && deg < cap_deg && D + 1 >= (uint32_t)pl.dend && j0 < D)
            t = D <= kSmallMaxD ? 1 : (D <= kMediumAMaxD ? 2 : (D <= kMediumMaxD ? 3 : 4));
        tier[r] = t;
        dom[r] = D;
        if (t)
            mx[t - 1] = max(mx[t - 1], D);
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const uint32_t m = __reduce_max_sync(kFull, mx[t]);
        if ((threadIdx.x & 31) == 0 && m)
            atomicMax(&tier_max[t], m);
    }
}

// (D, j0) of each listed root.
__global__ void k_gather_dom(ViewDev v, DevPlan pl, const uint32_t *__restrict__ list, uint32_t nl, uint32_t *D_out,
                             uint32_t *j0_out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += gridDim.x * blockDim.x) {
        uint32_t beg, D, j0;
        root_domain(v, pl, list[i], beg, D, j0);
        D_out[i] = D;
        j0_out[i] = j0;
    }
}

// Adjacency bytes of the searched roots: row pointers and split of the root
// (12 B), its domain list (4 B each) and, per domain vertex, its row pointers
// and split (12 B) plus its higher-priority list (4 B each).
__global__ void k_alg_bytes(ViewDev v, DevPlan pl, const uint8_t *__restrict__ tier, int64_t n,
                            unsigned long long *bytes) {
    unsigned long long acc[3] = {0, 0, 0};
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
        const int t = tier[r];
        if (!t)
            continue;
        uint32_t beg, D, j0;
        root_domain(v, pl, (uint32_t)r, beg, D, j0);
        unsigned long long a = (lane == 0) ? 12ull + 4ull * D : 0ull;
        for (uint32_t i = lane; i < D; i += 32) {
            uint32_t hb, he, xb, xe;
            hd_range(v, pl.asc, v.col[beg + i], i, D, hb, he, xb, xe);
            a += 12ull + 4ull * (he - hb);
        }
        acc[t == 1 ? 0 : (t == 4 ? 2 : 1)] += a;
    }
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        const unsigned long long x = warp_sum(acc[t]);
        if (lane == 0 && x)
            atomicAdd(&bytes[t], x);
    }
}

struct TierSel {
    const uint8_t *tier;
    uint8_t want;
    __host__ __device__ bool operator()(const uint32_t &i) const { return tier[i] == want; }
};

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
template <bool ENUM>
beep_status launch_small(int dend, int grid, cudaStream_t s, const ViewDev &v, const DevPlan &pl, const uint32_t *roots,
                         uint32_t n, int rev, unsigned long long *counter, const EnumDev &en) {
    switch (dend) {
#define BEEP_CASE(D)                                                                                               \
    case D:                                                                                                        \
        k_small<D, ENUM><<<grid, kSmallWarps * 32, 0, s>>>(v, pl, roots, n, rev, counter, en);                      \
        break;
        BEEP_CASE(3)
        BEEP_CASE(4)
        BEEP_CASE(5)
        BEEP_CASE(6)
        BEEP_CASE(7)
        BEEP_CASE(8)
        BEEP_CASE(9)
        BEEP_CASE(10)
#undef BEEP_CASE
    default:
        return fail(BEEP_ERR_UNSUPPORTED, "depth out of range");
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    return BEEP_OK;
}

template <int D, bool ENUM> beep_status set_medium_attr(size_t smem) {
    BEEP_CUDA_TRY(cudaFuncSetAttribute(k_medium<D, ENUM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return BEEP_OK;
}

template <bool ENUM>
beep_status launch_medium(int dend, int grid, int block, size_t smem, cudaStream_t s, const ViewDev &v,
                          const DevPlan &pl, const uint32_t *roots, uint32_t n, int rev, unsigned *cursor,
                          unsigned long long *counter, const EnumDev &en, uint32_t maxD) {
    switch (dend) {
#define BEEP_CASE(D)                                                                                               \
    case D:                                                                                                        \
        BEEP_TRY((set_medium_attr<D, ENUM>(smem)));                                                                \
        k_medium<D, ENUM><<<grid, block, smem, s>>>(v, pl, roots, n, rev, cursor, counter, en, maxD);                \
        break;
        BEEP_CASE(3)
        BEEP_CASE(4)
        BEEP_CASE(5)
        BEEP_CASE(6)
        BEEP_CASE(7)
        BEEP_CASE(8)
        BEEP_CASE(9)
        BEEP_CASE(10)
#undef BEEP_CASE
    default:
        return fail(BEEP_ERR_UNSUPPORTED, "depth out of range");
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    return BEEP_OK;
}

template <bool ENUM>
beep_status launch_large_dfs(int dend, int grid, cudaStream_t s, const ViewDev &v, const DevPlan &pl, const Batch &bt,
                             const uint32_t *arena, unsigned *cursor, unsigned long long *counter,
                             const EnumDev &en) {
    switch (dend) {
#define BEEP_CASE(D)                                                                                               \
    case D:                                                                                                        \
        k_large_dfs<D, ENUM><<<grid, 256, 0, s>>>(v, pl, bt, arena, cursor, counter, en);                           \
        break;
        BEEP_CASE(3)
        BEEP_CASE(4)
        BEEP_CASE(5)
        BEEP_CASE(6)
        BEEP_CASE(7)
        BEEP_CASE(8)
        BEEP_CASE(9)
        BEEP_CASE(10)
#undef BEEP_CASE
    default:
        return fail(BEEP_ERR_UNSUPPORTED, "depth out of range");
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    return BEEP_OK;
}

struct Timer {
    struct Rec {
        cudaEvent_t a, b;
        double *out;
    };
    bool on = false;
    cudaStream_t s = nullptr;
    std::vector<Rec> recs;
    int start() {
        if (!on)
            return -1;
        Rec r{nullptr, nullptr, nullptr};
        cudaEventCreate(&r.a);
        cudaEventCreate(&r.b);
        cudaEventRecord(r.a, s);
        recs.push_back(r);
        return (int)recs.size() - 1;
    }
    void stop(int id, double *out) {
        if (id < 0)
            return;
        cudaEventRecord(recs[id].b, s);
        recs[id].out = out;
    }
    void collect() {
        for (auto &r : recs) {
            float ms = 0;
            if (r.out) {
                cudaEventSynchronize(r.b);
                cudaEventElapsedTime(&ms, r.a, r.b);
                *r.out += ms;
            }
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        recs.clear();
    }
    ~Timer() { collect(); }
};

} // namespace

beep_status run_count(Ctx *ctx, Graph *g, const QueryPlan &plan, uint32_t options, const EnumRequest *enreq,
                      beep_stats *stats) {
    cudaStream_t s = ctx->stream;
    beep_stats st;
    std::memset(&st, 0, sizeof(st));
    const DevPlan &pl = plan.dev;
    Timer tm;
    tm.on = (options & BEEP_OPT_TIMING) != 0;
    tm.s = s;
    st.cutoff = g->cutoff;
    st.ascending = pl.asc;

    const bool enumerate = enreq && enreq->k > 0 && enreq->d_out;
    EnumDev en{nullptr, nullptr, 0};

    BEEP_TRY(ctx->counter.reserve(512));
    // u64 [8] count, [9] tuples reserved, [10..12] adjacency bytes by tier; u32 cursors at u64 [16..]
    unsigned long long *d_cnt = ctx->counter.as<unsigned long long>() + 8;
    unsigned *d_cursor = reinterpret_cast<unsigned *>(ctx->counter.as<unsigned long long>() + 16);
    BEEP_CUDA_TRY(cudaMemsetAsync(d_cnt, 0, 8 * 8, s));
    if (enumerate) {
        en.out = enreq->d_out;
        en.n = d_cnt + 1;
        en.k = enreq->k;
    }

    if (g->n == 0 || pl.dend < 3) {
        // sgc with K - LUNMAT < 3: the reference's main path never reaches a
        // counting level (check_terminate/backtrack need l >= 3).
        if (stats)
            *stats = st;
        return BEEP_OK;
    }

    // peel + priority relabelling (cached per (min_qdeg, order))
    int tprep = tm.start();
    View *v = nullptr;
    bool built = false;
    BEEP_TRY(get_view(ctx, g, plan.info.min_qdeg, pl.asc, (options & BEEP_OPT_NO_VIEW_CACHE) != 0, &v, &built,
                      nullptr));
    tm.stop(tprep, &st.prep_ms);
    st.peel_rounds = v->peel_rounds;
    if (built)
        st.kernel_launches += 8 + 2 * v->peel_rounds;
    if (v->n == 0) {
        tm.collect();
        if (stats)
            *stats = st;
        return BEEP_OK;
    }
    ViewDev vd{v->row_ptr.as<uint32_t>(), v->col.as<uint32_t>(), v->split.as<uint32_t>(), v->orig.as<uint32_t>()};
    const int64_t n = v->n;

    // classify roots into tiers
    size_t need = (size_t)n * 1 + 256 + (size_t)n * 4 * 8 + 4096;
    BEEP_TRY(ctx->scratch2.reserve(need));
    char *base = ctx->scratch2.as<char>();
    uint8_t *tier = reinterpret_cast<uint8_t *>(base);
    uint32_t *dom = reinterpret_cast<uint32_t *>(base + (((size_t)n + 255) & ~(size_t)255));
    uint32_t *lists[4]; // small, medium (<= 256), medium (<= 1024), large
    for (int t = 0; t < 4; ++t)
        lists[t] = dom + (size_t)n * (t + 1);
    uint32_t *d_nsel = dom + (size_t)n * 5;       // [0..3] counts, [4..7] max domain per tier
    uint32_t *d_gD = dom + (size_t)n * 5 + 64;     // large-tier gather
    uint32_t *d_gj = d_gD + (size_t)n;
    BEEP_CUDA_TRY(cudaMemsetAsync(d_nsel, 0, 64, s));
    uint64_t cap_deg = 0xffffffffull;
    if (options & BEEP_OPT_REFERENCE_ROOT_CAP)
        cap_deg = std::min<uint64_t>(0xffffffffull, (uint64_t)g->cutoff * 100ull);
    int tcount = tm.start();
    const int gv = std::max(1, (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 32));
    k_classify<<<gv, 256, 0, s>>>(vd, pl, n, (uint32_t)plan.info.max_qdeg, (uint32_t)cap_deg, tier, dom,
                                  d_nsel + 4);
    BEEP_CUDA_TRY(cudaGetLastError());
    st.kernel_launches += 1;
    uint32_t nsel[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = 0; t < 4; ++t) {
        size_t tb = 0;
        cub::CountingInputIterator<uint32_t> it(0);
        TierSel sel{tier, (uint8_t)(t + 1)};
        BEEP_CUDA_TRY(cub::DeviceSelect::If(nullptr, tb, it, lists[t], d_nsel + t, n, sel, s));
        BEEP_TRY(ctx->scratch.reserve(tb + 1024));
        BEEP_CUDA_TRY(cub::DeviceSelect::If(ctx->scratch.ptr, tb, it, lists[t], d_nsel + t, n, sel, s));
        st.kernel_launches += 1;
    }
    BEEP_CUDA_TRY(cudaMemcpyAsync(nsel, d_nsel, sizeof(nsel), cudaMemcpyDeviceToHost, s));
    const uint32_t max_medA = nsel[5], max_medB = nsel[6];
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    st.roots_small = nsel[0];
    st.roots_medium = (int64_t)nsel[1] + nsel[2];
    st.roots_large = nsel[3];
    st.roots = (int64_t)nsel[0] + nsel[1] + nsel[2] + nsel[3];
    // heaviest roots first: in ascending order they have the largest ids
    const int rev = pl.asc ? 1 : 0;
    BEEP_CUDA_TRY(cudaMemsetAsync(d_cursor, 0, 16, s));

    // large tier: batches of roots whose bitmaps fit the arena
    if (nsel[3] > 0) {
        std::vector<uint32_t> lr(nsel[3]), lD(nsel[3]), lj(nsel[3]);
        k_gather_dom<<<std::max(1u, std::min(nsel[3] / 256 + 1, 1024u)), 256, 0, s>>>(vd, pl, lists[3], nsel[3], d_gD,
                                                                                      d_gj);
        BEEP_CUDA_TRY(cudaGetLastError());
        BEEP_CUDA_TRY(cudaMemcpyAsync(lr.data(), lists[3], 4ull * nsel[3], cudaMemcpyDeviceToHost, s));
        BEEP_CUDA_TRY(cudaMemcpyAsync(lD.data(), d_gD, 4ull * nsel[3], cudaMemcpyDeviceToHost, s));
        BEEP_CUDA_TRY(cudaMemcpyAsync(lj.data(), d_gj, 4ull * nsel[3], cudaMemcpyDeviceToHost, s));
        BEEP_CUDA_TRY(cudaStreamSynchronize(s));
        st.kernel_launches += 1;
        struct R {
            uint32_t r, D, j0;
        };
        std::vector<R> rs(nsel[3]);
        for (uint32_t i = 0; i < nsel[3]; ++i)
            rs[i] = R{lr[i], lD[i], lj[i]};
        std::sort(rs.begin(), rs.end(), [](const R &a, const R &b) { return a.D > b.D; });
        size_t free_b = 0, total_b = 0;
        BEEP_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        size_t arena_cap = std::max<size_t>((size_t)256 << 20, std::min<size_t>((size_t)48 << 30, free_b / 2 +
                                                                                       ctx->arena.bytes));
        size_t i0 = 0;
        while (i0 < rs.size()) {
            size_t words = 0, i1 = i0;
            std::vector<uint32_t> broot, cstart{0}, tstart{0};
            std::vector<uint64_t> boff;
            while (i1 < rs.size()) {
                const uint64_t W = (rs[i1].D + 31) / 32;
                const uint64_t w = (uint64_t)rs[i1].D * W;
                if (i1 > i0 && (words + w) * 4 > arena_cap)
                    break;
                broot.push_back(rs[i1].r);
                boff.push_back(words);
                words += (w + 31) & ~(uint64_t)31; // 128-byte aligned rows
                cstart.push_back(cstart.back() + (rs[i1].D + kRowsPerChunk - 1) / kRowsPerChunk);
                tstart.push_back(tstart.back() + (rs[i1].D - rs[i1].j0));
                ++i1;
            }
            if (words * 4 > arena_cap)
                return fail(BEEP_ERR_OUT_OF_MEMORY, "a root's neighbourhood bitmap (" + std::to_string(words * 4) +
                                                        " bytes) exceeds the bitmap arena");
            BEEP_TRY(ctx->arena.reserve(words * 4));
            // batch descriptors
            const uint32_t nb = (uint32_t)broot.size();
            size_t dbytes = nb * 4 + nb * 8 + (nb + 1) * 8 + 1024;
            BEEP_TRY(ctx->scratch.reserve(dbytes));
            char *db = ctx->scratch.as<char>();
            uint64_t *d_off = reinterpret_cast<uint64_t *>(db);
            uint32_t *d_root = reinterpret_cast<uint32_t *>(db + nb * 8);
            uint32_t *d_cs = d_root + nb;
            uint32_t *d_ts = d_cs + nb + 1;
            BEEP_CUDA_TRY(cudaMemcpyAsync(d_off, boff.data(), nb * 8, cudaMemcpyHostToDevice, s));
            BEEP_CUDA_TRY(cudaMemcpyAsync(d_root, broot.data(), nb * 4, cudaMemcpyHostToDevice, s));
            BEEP_CUDA_TRY(cudaMemcpyAsync(d_cs, cstart.data(), (nb + 1) * 4, cudaMemcpyHostToDevice, s));
            BEEP_CUDA_TRY(cudaMemcpyAsync(d_ts, tstart.data(), (nb + 1) * 4, cudaMemcpyHostToDevice, s));
            BEEP_CUDA_TRY(cudaMemsetAsync(ctx->arena.ptr, 0, words * 4, s));
            BEEP_CUDA_TRY(cudaMemsetAsync(d_cursor, 0, 16, s));
            st.bitmap_bytes += words * 4;
            Batch bt{d_root, d_off, d_cs, d_ts, nb};
            uint32_t maxD = rs[i0].D;
            size_t smemA = std::min<size_t>(maxD, kLargeSmemA) * 4;
            BEEP_CUDA_TRY(cudaFuncSetAttribute(k_large_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemA));
            int te = tm.start();
            k_large_rows<<<ctx->num_sms, 512, smemA, s>>>(vd, pl, bt, ctx->arena.as<uint32_t>(), d_cursor);
            BEEP_CUDA_TRY(cudaGetLastError());
            tm.stop(te, &st.large_encode_ms);
            int td = tm.start();
            if (enumerate)
                BEEP_TRY(launch_large_dfs<true>(pl.dend, ctx->num_sms * 8, s, vd, pl, bt, ctx->arena.as<uint32_t>(),
                                                d_cursor + 1, d_cnt, en));
            else
                BEEP_TRY(launch_large_dfs<false>(pl.dend, ctx->num_sms * 8, s, vd, pl, bt, ctx->arena.as<uint32_t>(),
                                                 d_cursor + 1, d_cnt, en));
            tm.stop(td, &st.large_dfs_ms);
            st.large_encode_launches++;
            st.large_dfs_launches++;
            st.kernel_launches += 2;
            BEEP_CUDA_TRY(cudaStreamSynchronize(s)); // arena reuse by the next batch
            i0 = i1;
        }
        BEEP_CUDA_TRY(cudaMemsetAsync(d_cursor, 0, 16, s));
    }
    // medium tiers: block per root, bitmap in shared memory
    for (int sub = 0; sub < 2; ++sub) {
        const uint32_t nm = nsel[1 + sub];
        if (nm == 0)
            continue;
        const uint32_t maxD = sub == 0 ? max_medA : max_medB;
        const uint32_t W = (maxD + 31) / 32;
        const size_t pad = (maxD + 4) & ~3u;
        const size_t smem = (3 * pad + (size_t)maxD * W) * 4;
        const int block = sub == 0 ? 256 : 1024;
        const int per_sm = std::max(1, (int)std::min<size_t>(2048 / block, (200 * 1024) / (smem + 1024)));
        const int grid = ctx->num_sms * per_sm;
        int tmid = tm.start();
        if (enumerate)
            BEEP_TRY(launch_medium<true>(pl.dend, grid, block, smem, s, vd, pl, lists[1 + sub], nm, rev,
                                         d_cursor + 2 + sub, d_cnt, en, maxD));
        else
            BEEP_TRY(launch_medium<false>(pl.dend, grid, block, smem, s, vd, pl, lists[1 + sub], nm, rev,
                                          d_cursor + 2 + sub, d_cnt, en, maxD));
        tm.stop(tmid, &st.medium_ms);
        st.medium_launches++;
        st.kernel_launches += 1;
    }
    // small tier
    if (nsel[0] > 0) {
        int grid = (int)std::min<int64_t>(((int64_t)nsel[0] + kSmallWarps - 1) / kSmallWarps,
                                          (int64_t)ctx->num_sms * 8);
        int tsm = tm.start();
        if (enumerate)
            BEEP_TRY(launch_small<true>(pl.dend, grid, s, vd, pl, lists[0], nsel[0], rev, d_cnt, en));
        else
            BEEP_TRY(launch_small<false>(pl.dend, grid, s, vd, pl, lists[0], nsel[0], rev, d_cnt, en));
        tm.stop(tsm, &st.small_ms);
        st.small_launches++;
        st.kernel_launches += 1;
    }
    tm.stop(tcount, &st.count_ms);
    if (options & BEEP_OPT_ALG_BYTES) {
        k_alg_bytes<<<gv, 256, 0, s>>>(vd, pl, tier, n, d_cnt + 2);
        BEEP_CUDA_TRY(cudaGetLastError());
        st.kernel_launches += 1;
    }
    unsigned long long h[5] = {0, 0, 0, 0, 0};
    BEEP_CUDA_TRY(cudaMemcpyAsync(h, d_cnt, sizeof(h), cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    tm.collect();
    st.count = h[0];
    st.small_bytes = h[2];
    st.medium_bytes = h[3];
    st.large_bytes = h[4];
    st.adjacency_bytes = h[2] + h[3] + h[4];
    if (stats)
        *stats = st;
    return BEEP_OK;
}

} // namespace beep

// ===========================================================================
// Allocation-free counting (beep_count_noalloc)
//
// Some callers cannot let a library allocate device memory: a process whose
// device memory is handed out by its own pool or caching allocator (a
// cudaMalloc from a library can fail there, or fragment the pool), or a
// latency-critical loop where the device-wide synchronisation of
// cudaMalloc/cudaFree is not acceptable. For them this path counts with no
// allocation at all. Its only scratch is the file-scope array below, of
// BEEP_NOALLOC_SCRATCH_BYTES: a control block (count, root cursor, largest
// domain) and, for roots whose bitmap does not fit in shared memory, one
// bitmap slice per block. Every GPU that loads the library holds the array
// until the process exits. All calls on a device share it and it keeps the
// last call's contents, so each call clears the control block first; calls
// that overlap on the GPU (other streams or host threads) race on it.
// ===========================================================================
namespace beep {
namespace {

constexpr size_t kNoAllocCtrlBytes = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[BEEP_NOALLOC_SCRATCH_BYTES];

struct NoAllocCtrl {
    unsigned long long count;
    unsigned int cursor;
    unsigned int max_domain;
};

// Root domain straight from a sorted, simple CSR in vertex-id order.
__device__ __forceinline__ void csr_root_domain(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col,
                                                const DevPlan &pl, uint32_t r, uint32_t &beg, uint32_t &D,
                                                uint32_t &j0, uint32_t &deg) {
    const uint32_t b = rp[r], e = rp[r + 1];
    const uint32_t sp = lower_bound_g(col, b, e, r) - b;
    deg = e - b;
    if (pl.restricted) {
        beg = b + sp;
        D = e - b - sp;
        j0 = 0;
    } else {
        beg = b;
        D = e - b;
        j0 = pl.pos1_after_root ? sp : 0;
    }
}

__device__ __forceinline__ bool csr_is_root(const DevPlan &pl, uint32_t deg, uint32_t D, uint32_t j0,
                                            uint32_t min_deg) {
    return deg >= min_deg && D + 1 >= (uint32_t)pl.dend && j0 < D;
}

__global__ void k_noalloc_maxdom(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, int64_t n,
                                 DevPlan pl, uint32_t min_deg, NoAllocCtrl *ctrl) {
    uint32_t mx = 0;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        uint32_t beg, D, j0, deg;
        csr_root_domain(rp, col, pl, (uint32_t)v, beg, D, j0, deg);
        if (csr_is_root(pl, deg, D, j0, min_deg))
            mx = max(mx, D);
    }
    mx = __reduce_max_sync(kFull, mx);
    if ((threadIdx.x & 31) == 0 && mx)
        atomicMax(&ctrl->max_domain, mx);
}

// Rows [i0, i1) of the domain A (size D) of a root, ids ascending: the
// higher-priority list of u is its neighbours above u.
__device__ __forceinline__ void csr_build_rows(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col,
                                               const uint32_t *A, uint32_t D, uint32_t i0, uint32_t i1,
                                               uint32_t *rows, uint32_t W, uint32_t *s_hb, uint32_t *s_pre) {
    const uint32_t R = i1 - i0, tid = threadIdx.x, nthr = blockDim.x;
    for (uint32_t r = tid; r < R; r += nthr) {
        const uint32_t i = i0 + r, u = A[i];
        uint32_t hb = 0, c = 0;
        if (i + 1 < D) {
            const uint32_t b = rp[u], e = rp[u + 1];
            const uint32_t lo = lower_bound_g(col, b, e, A[i + 1]);
            const uint32_t hi = upper_bound_g(col, lo, e, A[D - 1]);
            hb = lo;
            c = hi - lo;
        }
        s_hb[r] = hb;
        s_pre[r] = c;
    }
    __syncthreads();
    if (tid < 32)
        warp_excl_scan(s_pre, R, (int)tid);
    __syncthreads();
    const uint32_t T = s_pre[R];
    for (uint32_t t = tid; t < T; t += nthr) {
        uint32_t lo = 0, hi = R;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s_pre[mid] <= t)
                lo = mid;
            else
                hi = mid;
        }
        const uint32_t i = i0 + lo;
        const uint32_t w = col[s_hb[lo] + (t - s_pre[lo])];
        const int k = find_idx(A, i + 1, D, w);
        if (k >= 0) {
            atomicOr(&rows[(size_t)i * W + ((uint32_t)k >> 5)], 1u << (k & 31));
            atomicOr(&rows[(size_t)k * W + (i >> 5)], 1u << (i & 31));
        }
    }
    __syncthreads();
}

// Block per root over every vertex (the medium-tier kernel reading the
// caller's CSR); rows in shared memory up to smem_maxD, else in this block's
// slice of the scratch array.
template <int DEND>
__global__ void __launch_bounds__(512) k_noalloc_count(const uint32_t *__restrict__ rp,
                                                       const uint32_t *__restrict__ col, int64_t n, DevPlan pl,
                                                       uint32_t min_deg, unsigned char *scratch,
                                                       uint64_t slice_words, uint32_t smem_maxD) {
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t s_v, s_j;
    NoAllocCtrl *ctrl = reinterpret_cast<NoAllocCtrl *>(scratch);
    uint32_t *slice = reinterpret_cast<uint32_t *>(scratch + kNoAllocCtrlBytes) + (uint64_t)blockIdx.x * slice_words;
    const uint32_t pad = (smem_maxD + 4) & ~3u;
    uint32_t *sA = sm, *s_hb = sm + pad, *s_pre = sm + 2 * pad, *srows = sm + 3 * pad;
    const int lane = threadIdx.x & 31;
    const Lp lp = load_lp(pl);
    EnumCtx ec{};
    unsigned long long cnt = 0;
    for (;;) {
        if (threadIdx.x == 0)
            s_v = atomicAdd(&ctrl->cursor, 1u);
        __syncthreads();
        const uint32_t v = s_v;
        if ((int64_t)v >= n)
            break;
        uint32_t beg, D, j0, deg;
        csr_root_domain(rp, col, pl, v, beg, D, j0, deg);
        if (csr_is_root(pl, deg, D, j0, min_deg)) {
            const uint32_t W = (D + 31) >> 5;
            const bool in_smem = D <= smem_maxD;
            uint32_t *rows = in_smem ? srows : slice;
            const uint32_t *A = col + beg;
            if (in_smem) {
                for (uint32_t i = threadIdx.x; i < D; i += blockDim.x)
                    sA[i] = A[i];
                A = sA;
            }
            for (uint64_t i = threadIdx.x; i < (uint64_t)D * W; i += blockDim.x)
                rows[i] = 0;
            if (threadIdx.x == 0)
                s_j = j0;
            __syncthreads();
            for (uint32_t i0 = 0; i0 < D; i0 += smem_maxD)
                csr_build_rows(rp, col, A, D, i0, min(D, i0 + smem_maxD), rows, W, s_hb, s_pre);
            for (;;) {
                uint32_t j = 0;
                if (lane == 0)
                    j = atomicAdd(&s_j, 1u);
                j = __shfl_sync(kFull, j, 0);
                if (j >= D)
                    break;
                uint32_t x[kMaxQ];
                x[1] = j;
                dfs_warp<2, DEND, false>(lp, rows, W, D, x, cnt, lane, ec);
            }
        }
        __syncthreads();
    }
    cnt = warp_sum(cnt);
    if (lane == 0 && cnt)
        atomicAdd(&ctrl->count, cnt);
}

std::mutex g_noalloc_mu;
void *g_noalloc_ptr[128] = {nullptr};

} // namespace
} // namespace beep

extern "C" beep_status beep_count_noalloc(int device, void *cuda_stream, int64_t n, int64_t m,
                                          const int32_t *d_row_ptr, const int32_t *d_col_ind, const beep_query *q,
                                          beep_mode mode, uint64_t *out_count) {
    using namespace beep;
    if (!q || !out_count || !d_row_ptr || (m > 0 && !d_col_ind) || n < 0 || m < 0 || n >= (int64_t)0xffffffffll ||
        m >= (int64_t)0xffffffffll)
        return fail(BEEP_ERR_INVALID_ARG, "beep_count_noalloc: bad arguments");
    if (device < 0 || device >= 128)
        return fail(BEEP_ERR_INVALID_ARG, "beep_count_noalloc: device id out of range");
    if (mode != BEEP_MODE_SGM && mode != BEEP_MODE_SGC)
        return fail(BEEP_ERR_INVALID_ARG, "unknown mode");
    BEEP_CUDA_TRY(cudaSetDevice(device));
    // Set-up, once per device with the device current: the device address of
    // the scratch array (its host-side name is not a device address).
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[device]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return fail(BEEP_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            g_noalloc_ptr[device] = p;
        }
        scratch = g_noalloc_ptr[device];
    }
    QueryPlan plan;
    BEEP_TRY(compile_plan(q->impl.qn, q->impl.row_ptr, q->impl.col, mode, &plan));
    if (plan.dev.dend < 3) {
        *out_count = 0;
        return BEEP_OK;
    }
    if (mode == BEEP_MODE_SGC && plan.info.unmat)
        return fail(BEEP_ERR_UNSUPPORTED, "sgc with an unmaterialised last level depends on the reference's priority "
                                          "order, which needs the peeled and relabelled graph: use beep_count");
    DevPlan pl = plan.dev;
    pl.asc = 1; // vertex ids ascending are the priority order here
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    const uint32_t *rp = reinterpret_cast<const uint32_t *>(d_row_ptr);
    const uint32_t *col = reinterpret_cast<const uint32_t *>(d_col_ind);
    NoAllocCtrl *ctrl = reinterpret_cast<NoAllocCtrl *>(scratch);
    int num_sms = 148;
    BEEP_CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    BEEP_CUDA_TRY(cudaMemsetAsync(scratch, 0, kNoAllocCtrlBytes, s));
    const uint32_t min_deg = (uint32_t)plan.info.max_qdeg;
    if (n > 0) {
        const int g0 = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms * 16));
        k_noalloc_maxdom<<<g0, 256, 0, s>>>(rp, col, n, pl, min_deg, ctrl);
        BEEP_CUDA_TRY(cudaGetLastError());
    }
    uint32_t maxD = 0;
    BEEP_CUDA_TRY(cudaMemcpyAsync(&maxD, &ctrl->max_domain, sizeof(maxD), cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    if (maxD == 0) {
        *out_count = 0;
        return BEEP_OK;
    }
    const uint32_t smem_maxD = (uint32_t)kMediumMaxD;
    const uint64_t arena_words = (BEEP_NOALLOC_SCRATCH_BYTES - kNoAllocCtrlBytes) / 4;
    uint64_t slice_words = 0;
    int grid = num_sms;
    if (maxD > smem_maxD) {
        slice_words = ((uint64_t)maxD * ((maxD + 31) / 32) + 63) & ~(uint64_t)63;
        if (slice_words > arena_words)
            return fail(BEEP_ERR_UNSUPPORTED,
                        "beep_count_noalloc: the largest search domain has " + std::to_string(maxD) +
                            " vertices; its bitmap needs " + std::to_string(slice_words * 4) +
                            " bytes, more than the " + std::to_string(BEEP_NOALLOC_SCRATCH_BYTES) +
                            "-byte scratch of the allocation-free path (domains up to 23170 vertices); use beep_count");
        grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)num_sms, arena_words / slice_words));
    }
    const size_t pad = (smem_maxD + 4) & ~3u;
    const size_t smem = (3 * pad + (size_t)smem_maxD * ((smem_maxD + 31) / 32)) * 4;
    unsigned char *scr = static_cast<unsigned char *>(scratch);
    switch (pl.dend) {
#define BEEP_CASE(DD)                                                                                              \
    case DD:                                                                                                       \
        BEEP_CUDA_TRY(cudaFuncSetAttribute(k_noalloc_count<DD>, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                           (int)smem));                                                            \
        k_noalloc_count<DD><<<grid, 512, smem, s>>>(rp, col, n, pl, min_deg, scr, slice_words, smem_maxD);          \
        break;
        BEEP_CASE(3)
        BEEP_CASE(4)
        BEEP_CASE(5)
        BEEP_CASE(6)
        BEEP_CASE(7)
        BEEP_CASE(8)
        BEEP_CASE(9)
        BEEP_CASE(10)
#undef BEEP_CASE
    default:
        return fail(BEEP_ERR_UNSUPPORTED, "depth out of range");
    }
    BEEP_CUDA_TRY(cudaGetLastError());
    unsigned long long c = 0;
    BEEP_CUDA_TRY(cudaMemcpyAsync(&c, &ctrl->count, sizeof(c), cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    *out_count = c;
    return BEEP_OK;
}
