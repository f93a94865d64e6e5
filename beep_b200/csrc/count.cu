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
//   - the last level is a popcount (as in the reference); free suffixes and
//     the 4-wheel are counted in closed form.
// Tiers by domain size D (limits are runtime parameters, defaults shown):
//   small   D <= 64   a group of 8 or 32 lanes per root, 64-bit rows in shared
//                     memory, a lane per level-1 vertex or (level-1, level-2)
//                     pair (thread-level DFS);
//   medium  D <= 1024 block per root, rows in shared memory, a thread (D <= 256)
//                     or a warp per level-1 vertex;
//   large   D > 1024  rows in a global arena; one launch builds the rows of a
//                     batch of roots (and a second the non-zero-word lists of
//                     wide rows), a third spreads the (root, level-1 vertex)
//                     tasks over every warp of the GPU.
// Queries without a central vertex take a fifth, list-walking tier.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "internal.h"

namespace beep {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kSmallMaxD = 64;
constexpr int kMediumAMaxD = 256;
constexpr int kMediumMaxD = 1024;
// 64-bit words per row of the thread-walker medium sub-tier (kMediumAMaxD bits)
constexpr uint32_t kThreadNW = kMediumAMaxD / 64;

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
    int free_from;
    uint32_t free_back;
};

__device__ __forceinline__ Lp load_lp(const DevPlan &pl) {
    Lp lp;
#pragma unroll
    for (int i = 0; i < kMaxQ; ++i) {
        lp.back[i] = pl.back[i];
        lp.sym[i] = pl.sym[i];
    }
    lp.free_from = pl.free_from;
    lp.free_back = pl.free_back;
    return lp;
}

// ---------------------------------------------------------------------------
// count overflow. A pair's count is a u64 (the reference's counter,
// subgraph_matching.cuh:1277, wraps silently). Here counts of kCountLimit =
// 2^64 - 2^52 or more are reported as overflow instead:
//   - closed-form terms (C(A, L), wheel pair terms) are added saturating: a
//     lane counter that would reach the limit is set to it;
//   - leaf popcounts (at most 64 each) are added unchecked: between two
//     flushes a lane adds fewer than 2^51 that way (2^45 additions take a
//     lane more than nine hours), so a saturated counter stays below 2^64;
//   - flushes sum lanes saturating and check the global add for a carry.
// A pair's counter is six words: the walks' count and its overflow flag,
// then the neighbourhood statistics' positive and negative sums with theirs.
// ---------------------------------------------------------------------------
constexpr unsigned long long kCountLimit = BEEP_COUNT_LIMIT;
static_assert(BEEP_COUNT_LIMIT == 0ull - (1ull << 52), "count limit");

__device__ __forceinline__ unsigned long long sat_add(unsigned long long a, unsigned long long b) {
    const unsigned long long s = a + b;
    return (s < a || s >= kCountLimit) ? kCountLimit : s;
}

__device__ __forceinline__ unsigned long long binom2(unsigned long long x) { return x * (x - (x ? 1 : 0)) / 2; }

// 128-bit product saturated to the count limit.
__device__ __forceinline__ unsigned long long sat_mul(unsigned long long a, unsigned long long b) {
    const unsigned __int128 p = (unsigned __int128)a * b;
    return p >= (unsigned __int128)kCountLimit ? kCountLimit : (unsigned long long)p;
}

// cnt + C(A, L) for L <= 4, the binomial exact through a 128-bit product
// (A < 2^32), saturating at kCountLimit.
__device__ __forceinline__ unsigned long long add_binom(unsigned long long cnt, uint32_t A, int L) {
    if (A < (uint32_t)L)
        return cnt;
    unsigned __int128 num = 1;
    for (int i = 0; i < L; ++i)
        num *= (unsigned __int128)(A - (uint32_t)i);
    const uint32_t fact = L <= 1 ? 1u : (L == 2 ? 2u : (L == 3 ? 6u : 24u));
    const unsigned __int128 s = num / fact + (unsigned __int128)cnt;
    return s >= (unsigned __int128)kCountLimit ? kCountLimit : (unsigned long long)s;
}

// Adds a flushed (saturated) sum to a pair's counter; sets its overflow flag
// (the word after the count) when the sum or the new total reaches the limit.
__device__ __forceinline__ void flush_count(unsigned long long *pc, unsigned long long v) {
    if (v >= kCountLimit) {
        atomicOr(pc + 1, 1ull);
        return;
    }
    if (!v)
        return;
    const unsigned long long old = atomicAdd(pc, v);
    if (old + v < old || old + v >= kCountLimit)
        atomicOr(pc + 1, 1ull);
}

// Positions P..DEND-1 form a free suffix when they share one back-edge set B
// (none of it inside the suffix) and each must follow the one before it: the
// completions of an assignment x[1..P-1] are then the L-subsets (L = DEND - P)
// of position P's candidate set -- provided no later position has a tighter
// bound from an assigned position than position P has (checked here), so the
// count is C(A, L) with A = |candidates of P|. With B empty, A is the unused
// domain vertices at or above P's bound and needs no bitmap.
template <int P, int DEND>
__device__ __forceinline__ bool suffix_applies(const Lp &lp, const uint32_t (&x)[kMaxQ], uint32_t lo) {
    constexpr int L = DEND - P;
    if constexpr (L > 4) {
        return false;
    } else {
        if (P < lp.free_from)
            return false;
#pragma unroll
        for (int p = P + 1; p < DEND; ++p)
#pragma unroll
            for (int q = 1; q < P; ++q)
                if ((lp.sym[p] >> q & 1u) && x[q] + 1 > lo)
                    return false;
        return true;
    }
}

template <int P>
__device__ __forceinline__ uint32_t level_bound(const Lp &lp, const uint32_t (&x)[kMaxQ]) {
    uint32_t lo = 0;
#pragma unroll
    for (int q = 1; q < P; ++q)
        if (lp.sym[P] >> q & 1u)
            lo = max(lo, x[q] + 1);
    return lo;
}

template <int P>
__device__ __forceinline__ uint32_t free_count_rootonly(uint32_t D, const uint32_t (&x)[kMaxQ], uint32_t lo) {
    uint32_t A = D > lo ? D - lo : 0u;
#pragma unroll
    for (int q = 1; q < P; ++q)
        A -= (x[q] >= lo) ? 1u : 0u;
    return A;
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

// Whether sorted a[lo, hi) holds key.
__device__ __forceinline__ bool contains_g(const uint32_t *__restrict__ a, uint32_t lo, uint32_t hi, uint32_t key) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t x = a[mid];
        if (x == key)
            return true;
        if (x < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return false;
}

// Index of key in sorted a[lo, hi) or -1 (a holds fewer than 2^31 entries).
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

// An enumerating walk stops once k tuple slots are reserved (the pair's exact
// count comes from a counting pair of the same call).
__device__ __forceinline__ bool enum_full(const EnumCtx &ec) {
    return ec.en.out != nullptr && *(const volatile unsigned long long *)ec.en.n >= ec.en.k;
}

__device__ __forceinline__ void emit_bits(const EnumCtx &ec, const uint32_t (&x)[kMaxQ], int P, uint64_t bits,
                                          uint32_t base) {
    // a pair that enumerates nothing may share an enumerating launch
    if (!bits || ec.en.out == nullptr)
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
// rows + (i - rlo) * NW is the row of domain vertex i, NW 64-bit words (only
// rows i >= rlo exist; the plan reads no other). One thread walks the whole
// subtree below its level-1 vertex; the candidate words of a level stay in
// registers.
// Word k of position P's candidate set: the domain bits at or above lo, AND
// the rows of P's back edges, minus the vertices already used.
template <int P, int NW>
__device__ __forceinline__ uint64_t cand_word(const Lp &lp, const uint64_t *rows, uint32_t rlo, uint32_t D,
                                              uint32_t lo, const uint32_t (&x)[kMaxQ], uint32_t k) {
    const uint32_t base = k * 64;
    uint64_t w = base + 64 <= D ? ~0ull : (base < D ? ((1ull << (D - base)) - 1ull) : 0ull);
    if (lo > base)
        w = lo >= base + 64 ? 0ull : (w & ~((1ull << (lo - base)) - 1ull));
    const uint32_t bk = lp.back[P];
#pragma unroll
    for (int q = 1; q < P; ++q) {
        if (bk >> q & 1u)
            w &= rows[(size_t)(x[q] - rlo) * NW + k];
        if ((x[q] >> 6) == k)
            w &= ~(1ull << (x[q] & 63));
    }
    return w;
}

// Position of the j-th set bit (0-based) of w, which has more than j set bits.
__device__ __forceinline__ uint32_t select64(uint64_t w, uint32_t j) {
    uint32_t pos = 0;
#pragma unroll
    for (int sh = 32; sh >= 1; sh >>= 1) {
        const uint32_t c = (uint32_t)__popcll(w & ((1ull << sh) - 1ull));
        if (j >= c) {
            j -= c;
            w >>= sh;
            pos += (uint32_t)sh;
        }
    }
    return pos;
}

template <int P, int DEND, bool ENUM, int NW>
__device__ __forceinline__ void dfs_thread(const Lp &lp, const uint64_t *rows, uint32_t rlo, uint32_t D,
                                           uint32_t (&x)[kMaxQ], unsigned long long &cnt, const EnumCtx &ec) {
    if constexpr (P >= DEND) {
        return; // never called: the callers stop at the last position
    } else {
        const uint32_t lo = level_bound<P>(lp, x);
        bool closed = false; // count this level's candidates as C(A, DEND - P)
        if constexpr (!ENUM && DEND - P <= 4) {
            if (suffix_applies<P, DEND>(lp, x, lo)) {
                if (lp.free_back == 0) {
                    cnt = add_binom(cnt, free_count_rootonly<P>(D, x, lo), DEND - P);
                    return;
                }
                closed = DEND - P >= 2; // one level: the leaf popcount below is the same
            }
        }
        if constexpr (NW == 1) {
            // one word: the candidate set stays in a register
            uint64_t c = cand_word<P, 1>(lp, rows, rlo, D, lo, x, 0);
            if (closed) {
                cnt = add_binom(cnt, (uint32_t)__popcll(c), DEND - P);
                return;
            }
            if constexpr (P == DEND - 1) {
                if constexpr (ENUM)
                    emit_bits(ec, x, P, c, 0);
                cnt += (unsigned long long)__popcll(c);
            } else {
                while (c) {
                    if constexpr (ENUM) {
                        if (enum_full(ec))
                            return;
                    }
                    const int b = __ffsll((long long)c) - 1;
                    c &= c - 1;
                    x[P] = (uint32_t)b;
                    dfs_thread<P + 1, DEND, ENUM, 1>(lp, rows, rlo, D, x, cnt, ec);
                }
            }
            return;
        }
        const uint32_t k0 = lo >> 6, nw = min((uint32_t)NW, (D + 63) >> 6);
        if (closed || P == DEND - 1) {
            uint32_t A = 0;
            for (uint32_t k = k0; k < nw; ++k) {
                const uint64_t w = cand_word<P, NW>(lp, rows, rlo, D, lo, x, k);
                if constexpr (ENUM)
                    emit_bits(ec, x, P, w, k * 64);
                A += (uint32_t)__popcll(w);
            }
            cnt = closed ? add_binom(cnt, A, DEND - P) : cnt + (unsigned long long)A;
            return;
        }
        if constexpr (P < DEND - 1 && NW > 1) {
            // one call site per level; only the current word and its index live
            // across the call (the next word is recomputed from the rows)
            uint32_t k = k0;
            if (k >= nw)
                return;
            uint64_t w = cand_word<P, NW>(lp, rows, rlo, D, lo, x, k);
            for (;;) {
                if constexpr (ENUM) {
                    if (enum_full(ec))
                        return;
                }
                while (!w) {
                    if (++k >= nw)
                        return;
                    w = cand_word<P, NW>(lp, rows, rlo, D, lo, x, k);
                }
                const int b = __ffsll((long long)w) - 1;
                w &= w - 1;
                x[P] = k * 64 + (uint32_t)b;
                dfs_thread<P + 1, DEND, ENUM, NW>(lp, rows, rlo, D, x, cnt, ec);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// warp-level DFS on rows of W 32-bit words (lane k holds word k of a chunk)
// ---------------------------------------------------------------------------
// bm + (i - rlo) * W is the row of domain vertex i (rows i >= rlo only).
// A group of G lanes (G = 32: a warp; gmask its lanes, glane the lane within
// it) walks the words of a level G at a time; every lane of the group calls
// this together.
//
// LIST (large tier, G = 32): rows of cap > 0 carry, beside the bitmap, the
// number of their non-zero words (nzc[i - rlo]) and, when that is at most
// cap, the indices of those words in ascending order (nzl + (i - rlo) * cap).
// A level then visits only the non-zero words of its sparsest back-edge row,
// 32 a step: in a hub's neighbourhood a row has a few dozen bits among
// hundreds of thousands, and the full scan costs ceil(D / 1024) warp steps
// per level however few candidates there are.
struct RowLists {
    const uint32_t *nzc = nullptr; // non-zero words per row
    const uint32_t *nzl = nullptr; // their indices, cap per row
    uint32_t cap = 0;              // 0: no lists
};

// ---------------------------------------------------------------------------
// work donation of the large tier. The reference hands a DFS subtree to an
// idle block through a ticket queue once the global roots run out
// (include/queue.cuh:17-56, device_utils.cuh:328-424, sgm_kernelsLD.cuh:
// 89-106, 135-271), with unbounded spins and a recipient that reads the
// donor's bitmap while the donor may overwrite it. Here the large tier's rows
// sit in the arena for the whole launch, so a donated task is just indices:
// (batch entry, x1, level P, x[2 .. P-1], an iteration range of level P).
//   - Warps first take the static (root, x1) tasks from the cursor. A warp
//     that finds it empty claims the next queue slot (head) and waits for it.
//   - A running warp at a level 2 <= P <= max_level that is not closed-form
//     checks at every iteration whether slots are claimed but not reserved
//     (head > tail); if so and at least min_iters iterations remain, it
//     reserves a slot (tail), writes the upper half of its remaining range
//     there, publishes it (ready flag after a fence) and keeps the lower half.
//   - Termination: pending counts reserved donated tasks not yet finished and
//     static_done the finished static tasks. A waiting warp leaves when every
//     static task is done and nothing is pending: no task runs, so none can
//     be donated any more.
//   - Waits are bounded: a waiting warp that sees no progress (a reservation,
//     a finished task or a donor's heartbeat) for timeout_ns sets the error
//     word and returns, so a kernel never spins without end; the host reports
//     BEEP_ERR_TIMEOUT.
// ---------------------------------------------------------------------------
struct DonTask {
    uint32_t b;          // batch entry (root) of the task
    uint32_t x1;         // level-1 vertex (domain index)
    uint32_t level;      // level whose iteration range the task covers
    uint32_t it_lo, it_hi;
    uint32_t x[kMaxQ - 2]; // x[2 .. level - 1]
    uint32_t pad[3];
};
static_assert(sizeof(DonTask) == 64, "donated task record");

enum DonCtl : uint32_t {
    kDonHead = 0,       // slots claimed by waiting warps
    kDonTail = 1,       // slots reserved by donors
    kDonPending = 2,    // donated tasks reserved and not finished
    kDonHeartbeat = 3,  // bumped by running warps that see waiters but cannot donate
    kDonError = 4,      // 1: a wait ran out
    kDonCount = 5,      // donations made
    kDonStaticDone = 6, // static tasks finished
    kDonDone = 7,       // donated tasks finished
    kDonWords = 8
};

struct Don {
    DonTask *tasks = nullptr;
    unsigned *ready = nullptr; // cap flags
    unsigned *ctl = nullptr;   // kDonWords
    uint32_t cap = 0;          // 0: no donation
    uint32_t max_level = 0;    // donate at levels 2 .. max_level
    uint32_t min_iters = 2;    // ... when at least this many iterations remain
    unsigned long long timeout_ns = 1000000000ull;
};

__device__ __forceinline__ unsigned ld_volatile(const unsigned *p) { return *(const volatile unsigned *)p; }

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Earliest and latest exit of a launch's warps: exit_t[0] holds the largest
// complemented time (so one zero fill starts both words), exit_t[1] the
// largest time. Called by one lane of each warp (or block) as it leaves.
__device__ __forceinline__ void record_exit(unsigned long long *exit_t) {
    if (exit_t) {
        const unsigned long long t = global_ns();
        atomicMax(exit_t, ~t);
        atomicMax(exit_t + 1, t);
    }
}

// What a donating warp knows about its task: where to donate, and the task's
// batch entry and level-1 vertex (copied into every task it donates); and
// when lane 0 last bumped the heartbeat.
struct DonCtx {
    const Don *dn = nullptr;
    uint32_t b = 0, x1 = 0;
    unsigned long long last_beat = 0;
};

// Lane 0 of a warp that sees waiting warps but cannot donate shows progress,
// at most every 100 microseconds.
__device__ __forceinline__ void heartbeat(DonCtx &dc) {
    const unsigned long long t = global_ns();
    if (t - dc.last_beat > 100000ull) {
        dc.last_beat = t;
        atomicAdd(&dc.dn->ctl[kDonHeartbeat], 1u);
    }
}

// Lane 0 reserves a slot and writes the task [lo, hi) of level P; false when
// the queue is full (the donor keeps the work).
template <int P>
__device__ __forceinline__ bool donate(const DonCtx &dc, const uint32_t (&x)[kMaxQ], uint32_t lo, uint32_t hi,
                                       int lane) {
    const Don &dn = *dc.dn;
    uint32_t s = 0;
    if (lane == 0) {
        atomicAdd(&dn.ctl[kDonPending], 1u);
        s = atomicAdd(&dn.ctl[kDonTail], 1u);
        if (s < dn.cap) {
            DonTask *t = dn.tasks + s;
            t->b = dc.b;
            t->x1 = dc.x1;
            t->level = (uint32_t)P;
            t->it_lo = lo;
            t->it_hi = hi;
#pragma unroll
            for (int q = 2; q < P; ++q)
                t->x[q - 2] = x[q];
            __threadfence();
            atomicExch(&dn.ready[s], 1u);
            atomicAdd(&dn.ctl[kDonCount], 1u);
        } else {
            atomicSub(&dn.ctl[kDonPending], 1u);
        }
    }
    s = __shfl_sync(kFull, s, 0);
    return s < dn.cap;
}

template <int P, int DEND, bool ENUM, int G = 32, bool LIST = false, bool DON = false>
__device__ __forceinline__ void dfs_warp(const Lp &lp, const uint32_t *bm, uint32_t rlo, uint32_t W, uint32_t D,
                                         uint32_t (&x)[kMaxQ], unsigned long long &cnt, int glane, const EnumCtx &ec,
                                         unsigned gmask = kFull, const RowLists &rl = RowLists(),
                                         DonCtx *dc = nullptr, uint32_t r_lo = 0,
                                         uint32_t r_hi = 0xffffffffu) {
    static_assert(!DON || G == 32, "donation is by whole warps");
    constexpr int LG = G == 32 ? 5 : (G == 16 ? 4 : (G == 8 ? 3 : (G == 4 ? 2 : (G == 2 ? 1 : 0))));
    static_assert((1 << LG) == G, "group size must be a power of two up to 32");
    static_assert(!LIST || G == 32, "row lists are read by whole warps");
    const uint32_t bk = lp.back[P];
    const uint32_t lo = level_bound<P>(lp, x);
    bool closed = false; // group-uniform: count this level's candidates as C(A, DEND - P)
    if constexpr (!ENUM && DEND - P <= 4) {
        if (suffix_applies<P, DEND>(lp, x, lo)) {
            if (lp.free_back == 0) {
                if (glane == 0)
                    cnt = add_binom(cnt, free_count_rootonly<P>(D, x, lo), DEND - P);
                return;
            }
            closed = DEND - P >= 2; // one level: the leaf popcount below is the same
        }
    }
    const int gbase = (threadIdx.x & 31) & ~(G - 1);
    uint32_t acc = 0;
    const uint32_t nch = (W + G - 1) >> LG;
    const uint32_t tail = D & 31;
    // Steps it0 .. it1 - 1 of G words each: consecutive words from the bound
    // on, or (listed) the non-zero words of the sparsest back-edge row.
    uint32_t it0 = lo >> (5 + LG), it1 = nch, nl = 0;
    bool listed = false;
    const uint32_t *bl = nullptr;
    if constexpr (LIST) {
        if (rl.cap) {
            uint32_t best = 0xffffffffu;
#pragma unroll
            for (int q = 1; q < P; ++q)
                if (bk >> q & 1u) {
                    const uint32_t c = rl.nzc[x[q] - rlo];
                    if (c < best) {
                        best = c;
                        bl = rl.nzl + (size_t)(x[q] - rlo) * rl.cap;
                    }
                }
            if (best <= rl.cap) {
                listed = true;
                nl = best;
                it0 = 0;
                it1 = (best + G - 1) >> LG;
            }
        }
    }
    // a donated task covers part of this level's iterations
    it0 = max(it0, r_lo);
    it1 = min(it1, r_hi);
    for (uint32_t it = it0; it < it1; ++it) {
        if constexpr (ENUM && P < DEND - 1) {
            unsigned full = glane == 0 ? (unsigned)enum_full(ec) : 0u;
            full = __shfl_sync(gmask, full, 0, G);
            if (full)
                return;
        }
        if constexpr (DON && P < DEND - 1) {
            // below the donation levels: only show progress to waiting warps
            // (a long subtree must not look like a hang)
            if (P > (int)dc->dn->max_level && glane == 0) {
                const unsigned long long t = global_ns();
                if (t - dc->last_beat > 200000ull) {
                    dc->last_beat = t;
                    const unsigned *ctl = dc->dn->ctl;
                    if (ld_volatile(&ctl[kDonHead]) > ld_volatile(&ctl[kDonTail]))
                        atomicAdd(&dc->dn->ctl[kDonHeartbeat], 1u);
                }
            }
            // hand the upper half of the remaining iterations to a waiting warp
            if (!closed && P <= (int)dc->dn->max_level) {
                unsigned want = 0;
                if (glane == 0) {
                    const unsigned *ctl = dc->dn->ctl;
                    want = ld_volatile(&ctl[kDonHead]) > ld_volatile(&ctl[kDonTail]) && !ld_volatile(&ctl[kDonError]);
                }
                want = __shfl_sync(kFull, want, 0);
                if (want) {
                    const uint32_t mid = it + 1 + (it1 - it - 1) / 2;
                    if (it1 - it >= dc->dn->min_iters && donate<P>(*dc, x, mid, it1, glane))
                        it1 = mid;
                    else if (glane == 0)
                        heartbeat(*dc);
                }
            }
        }
        // this lane's word (none when k >= W)
        uint32_t k;
        if (LIST && listed) {
            const uint32_t e = (it << LG) + (uint32_t)glane;
            k = e < nl ? bl[e] : 0xffffffffu;
        } else {
            k = (it << LG) + (uint32_t)glane;
        }
        uint32_t w = 0;
        if (k < W) {
            w = (k + 1 < W || tail == 0) ? kFull : ((1u << tail) - 1u);
#pragma unroll
            for (int q = 1; q < P; ++q) {
                if (bk >> q & 1u)
                    w &= bm[(size_t)(x[q] - rlo) * W + k];
                if ((x[q] >> 5) == k)
                    w &= ~(1u << (x[q] & 31));
            }
            const uint32_t lw = lo >> 5;
            if (lw > k)
                w = 0;
            else if (lw == k)
                w &= ~((1u << (lo & 31)) - 1u);
        }
        if (closed) {
            acc += (uint32_t)__popc(w);
            continue;
        }
        if constexpr (P == DEND - 1) {
            if constexpr (ENUM)
                emit_bits(ec, x, P, (uint64_t)w, k << 5);
            cnt += (unsigned long long)__popc(w);
        } else {
            unsigned bal = __ballot_sync(gmask, w != 0) >> gbase;
            if constexpr (G < 32)
                bal &= (1u << G) - 1u;
            while (bal) {
                const int L = __ffs(bal) - 1;
                const uint32_t ww = __shfl_sync(gmask, w, L, G);
                const int b = __ffs(ww) - 1;
                if (glane == L)
                    w &= w - 1;
                uint32_t kk = (it << LG) + (uint32_t)L;
                if (LIST && listed)
                    kk = __shfl_sync(gmask, k, L, G);
                x[P] = (kk << 5) + (uint32_t)b;
                dfs_warp<P + 1, DEND, ENUM, G, LIST, DON>(lp, bm, rlo, W, D, x, cnt, glane, ec, gmask, rl, dc);
                bal = __ballot_sync(gmask, w != 0) >> gbase;
                if constexpr (G < 32)
                    bal &= (1u << G) - 1u;
            }
        }
    }
    if (closed) {
        uint32_t A = acc;
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1)
            A += __shfl_xor_sync(gmask, A, o, G);
        if (glane == 0)
            cnt = add_binom(cnt, A, DEND - P);
    }
}

// Sum over the warp, saturating at kCountLimit (every lane gets it).
__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = sat_add(v, __shfl_xor_sync(kFull, v, o));
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
// Used by a warp group (small tier: a binary search over at most 64 entries;
// a per-group hash measured slower, 0.80 -> 1.10 ms on C2, its set-up costing
// more than the searches it saves on such small domains) or a block on a
// chunk of rows (large tier, whose domains are too large for a shared-memory
// hash); the medium tier looks list entries up in a hash of the domain
// (build_rows_hashed).
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

// Exclusive prefix of buf[0, R) in place, total in buf[R], by a group of G
// lanes (G = 32: a warp) whose mask is gmask; glane is the lane within it.
template <int G>
__device__ __forceinline__ void group_excl_scan(uint32_t *buf, uint32_t R, int glane, unsigned gmask) {
    uint32_t carry = 0;
    for (uint32_t base = 0; base < R; base += G) {
        const uint32_t idx = base + glane;
        const uint32_t x = idx < R ? buf[idx] : 0u;
        uint32_t inc = x;
#pragma unroll
        for (int o = 1; o < G; o <<= 1) {
            const uint32_t y = __shfl_up_sync(gmask, inc, o, G);
            if (glane >= o)
                inc += y;
        }
        if (idx < R)
            buf[idx] = carry + inc - x;
        carry += __shfl_sync(gmask, inc, G - 1, G);
    }
    if (glane == 0)
        buf[R] = carry;
}

__device__ __forceinline__ void warp_excl_scan(uint32_t *buf, uint32_t R, int lane) {
    group_excl_scan<32>(buf, R, lane, kFull);
}

// G = 0: the whole block; else a group of G lanes of one warp.
template <int G> __device__ __forceinline__ void group_sync(unsigned gmask) {
    if constexpr (G == 0)
        __syncthreads();
    else
        __syncwarp(gmask);
}

// Lists longer than this are first cut to [min, max] of the A entries they
// can meet (two binary searches); shorter ones are searched whole, which
// costs fewer dependent loads.
constexpr uint32_t kTrimMin = 16;

// floor(log2(x)) + 1 for x >= 1 (the steps of a binary search over x entries)
__device__ __forceinline__ uint32_t search_steps(uint32_t x) { return 32u - (uint32_t)__clz(x | 1u); }

// Only edges with an endpoint at index >= rlo are found (the rows below rlo
// are not stored): in ascending order row i searches A[max(i + 1, rlo), D),
// in descending order rows below rlo search nothing.
//
// Each row picks the cheaper direction: its list slice (c entries) searched
// in A (shared memory, c * log D steps), or the nA entries of A it can meet
// searched in the list slice (global memory, nA * log c steps) when the
// slice is much longer than that part of A -- the usual case for domain
// vertices of high degree. s_len[r] holds the slice length, with the top bit
// set for the second direction.
template <int G, typename SetFn>
__device__ __forceinline__ void build_rows_flat(const ViewDev &v, int asc, const uint32_t *A, uint32_t D,
                                                uint32_t rlo, uint32_t i0, uint32_t i1, uint32_t *s_hb,
                                                uint32_t *s_pre, uint32_t *s_len, uint32_t tid, uint32_t nthr,
                                                unsigned gmask, SetFn set) {
    constexpr uint32_t kByA = 0x80000000u;
    const uint32_t R = i1 - i0;
    const uint32_t logD = search_steps(D);
    for (uint32_t r = tid; r < R; r += nthr) {
        const uint32_t i = i0 + r;
        uint32_t hb, he, xb, xe, c = 0, work = 0, len = 0;
        hd_range(v, asc, A[i], i, D, hb, he, xb, xe);
        if (asc)
            xb = max(xb, rlo);
        else if (i < rlo)
            xe = 0;
        if (xb < xe && hb < he) {
            if (he - hb > kTrimMin) {
                const uint32_t lo = lower_bound_g(v.col, hb, he, A[xb]);
                const uint32_t hi = upper_bound_g(v.col, lo, he, A[xe - 1]);
                hb = lo;
                c = hi - lo;
            } else {
                c = he - hb;
            }
            const uint32_t nA = xe - xb;
            len = c;
            work = c;
            if (c > 0 && c < kByA && (uint64_t)nA * search_steps(c) * 2 < (uint64_t)c * logD) {
                len = c | kByA;
                work = nA;
            }
        }
        s_hb[r] = hb;
        s_len[r] = len;
        s_pre[r] = work;
    }
    group_sync<G>(gmask);
    if constexpr (G == 0) {
        if (tid < 32)
            warp_excl_scan(s_pre, R, (int)tid);
    } else {
        group_excl_scan<G>(s_pre, R, (int)tid, gmask);
    }
    group_sync<G>(gmask);
    const uint32_t T = s_pre[R];
    // kU items per thread per step: their rows are searched and their list
    // entries loaded before any is searched in A, so a thread keeps kU
    // independent chains in flight
    constexpr int kU = 4;
    for (uint32_t t = tid; t < T; t += nthr * kU) {
        uint32_t rr[kU], wv[kU];
#pragma unroll
        for (int j = 0; j < kU; ++j) {
            const uint32_t tj = t + nthr * j;
            rr[j] = 0xffffffffu;
            wv[j] = 0;
            if (tj < T) {
                // row: last with s_pre[r] <= tj
                uint32_t lo = 0, hi = R;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (s_pre[mid] <= tj)
                        lo = mid;
                    else
                        hi = mid;
                }
                rr[j] = lo;
                if (!(s_len[lo] & kByA))
                    wv[j] = v.col[s_hb[lo] + (tj - s_pre[lo])];
            }
        }
#pragma unroll
        for (int j = 0; j < kU; ++j) {
            const uint32_t lo = rr[j];
            if (lo == 0xffffffffu)
                continue;
            const uint32_t i = i0 + lo;
            const uint32_t len = s_len[lo];
            const uint32_t xb = asc ? max(i + 1, rlo) : 0, xe = asc ? D : i;
            if (len & kByA) {
                const uint32_t k = xb + (t + nthr * j - s_pre[lo]);
                const uint32_t hb = s_hb[lo];
                if (contains_g(v.col, hb, hb + (len & ~kByA), A[k]))
                    set(i, k);
            } else {
                const int k = find_idx(A, xb, xe, wv[j]);
                if (k >= 0)
                    set(i, (uint32_t)k);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Row building for a block over a domain of at most kMediumMaxD vertices,
// through a shared-memory hash of the domain (vertex id -> domain index):
//   1. per row i: A[i]'s higher-priority list, untrimmed (its two row
//      pointers and split, one global round trip per row);
//   2. exclusive prefix of the per-row work;
//   3. warp w takes the contiguous work range [w * chunk, (w + 1) * chunk),
//      32 items a step (consecutive lanes read consecutive list entries);
//      each lane's row advances monotonically instead of being searched per
//      item, its row's offsets held in registers. A list entry is looked up
//      in the hash; the A entries of a row whose list is far longer than that
//      part of A (nA * log2(c) * 4 < c) are instead searched in the list.
// The hash has 2^k >= 8D slots of vertex ids (all ones: empty) with the
// domain index beside each; multiplicative hashing, linear probing. Most
// lookups miss (a list entry outside the domain), so a filter of 8 bits per
// slot, indexed by three more bits of the same hash, answers most of them
// with one shared load; at load factor <= 1/8 a lookup that passes it probes
// about one slot. (On C2, 2D slots and no filter: k_medium 1.73 ms; 8D: 1.48;
// 8D with the filter and the row offsets in registers: 1.44.)
// ---------------------------------------------------------------------------
constexpr uint32_t kHashEmpty = 0xffffffffu;

__host__ __device__ __forceinline__ uint32_t hash_slots(uint32_t maxD) {
    uint32_t s = 64;
    while (s < 8 * maxD)
        s <<= 1;
    return s;
}

__device__ __forceinline__ uint32_t hash_of(uint32_t w, uint32_t hshift) { return (w * 0x9E3779B1u) >> hshift; }

// Fills the hash of A[0, D) and its filter (nslots / 4 words after the
// indices) (block-wide; the caller syncs before and after).
__device__ __forceinline__ void hash_build(const uint32_t *A, uint32_t D, uint32_t *hkeys, uint16_t *hidx,
                                           uint32_t nslots, uint32_t hshift) {
    uint32_t *filt = hkeys + nslots + nslots / 2;
    for (uint32_t i = threadIdx.x; i < nslots; i += blockDim.x)
        hkeys[i] = kHashEmpty;
    for (uint32_t i = threadIdx.x; i < nslots / 4; i += blockDim.x)
        filt[i] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < D; i += blockDim.x) {
        const uint32_t w = A[i];
        const uint32_t fi = (w * 0x9E3779B1u) >> (hshift - 3);
        atomicOr(&filt[fi >> 5], 1u << (fi & 31));
        uint32_t s = hash_of(w, hshift);
        while (atomicCAS(&hkeys[s], kHashEmpty, w) != kHashEmpty)
            s = (s + 1) & (nslots - 1);
        hidx[s] = (uint16_t)i;
    }
}

// Domain index of w, or -1 (at once when w's filter bit is clear).
__device__ __forceinline__ int hash_find(const uint32_t *hkeys, const uint16_t *hidx, uint32_t nslots,
                                         uint32_t hshift, uint32_t w) {
    const uint32_t h = w * 0x9E3779B1u, fi = h >> (hshift - 3);
    if (!((hkeys[nslots + nslots / 2 + (fi >> 5)] >> (fi & 31)) & 1u))
        return -1;
    uint32_t s = h >> hshift;
    for (;;) {
        const uint32_t key = hkeys[s];
        if (key == w)
            return (int)hidx[s];
        if (key == kHashEmpty)
            return -1;
        s = (s + 1) & (nslots - 1);
    }
}

template <typename SetFn>
__device__ __forceinline__ void build_rows_hashed(const ViewDev &v, int asc, const uint32_t *A, uint32_t D,
                                                  uint32_t rlo, uint32_t *s_hb, uint32_t *s_pre, uint32_t *s_len,
                                                  const uint32_t *hkeys, const uint16_t *hidx, uint32_t nslots,
                                                  uint32_t hshift, SetFn set) {
    constexpr uint32_t kByA = 0x80000000u;
    const uint32_t R = D, tid = threadIdx.x, nthr = blockDim.x;
    for (uint32_t r = tid; r < R; r += nthr) {
        uint32_t hb, he, xb, xe, work = 0, len = 0;
        hd_range(v, asc, A[r], r, D, hb, he, xb, xe);
        if (asc)
            xb = max(xb, rlo);
        else if (r < rlo)
            xe = 0;
        if (xb < xe && hb < he) {
            const uint32_t c = he - hb, nA = xe - xb;
            len = c;
            work = c;
            if (c < kByA && (uint64_t)nA * search_steps(c) * 4 < (uint64_t)c) {
                len = c | kByA;
                work = nA;
            }
        }
        s_hb[r] = hb;
        s_len[r] = len;
        s_pre[r] = work;
    }
    __syncthreads();
    if (tid < 32)
        warp_excl_scan(s_pre, R, (int)tid);
    __syncthreads();
    const uint32_t T = s_pre[R];
    const uint32_t nw = nthr >> 5, lane = tid & 31;
    const uint32_t chunk = ((T + nw - 1) / nw + 31) & ~31u;
    const uint32_t t_begin = (tid >> 5) * chunk, t_end = min(T, t_begin + chunk);
    uint32_t r = 0;
    if (t_begin + lane < t_end) { // the row of this lane's first item: last r with s_pre[r] <= t
        uint32_t lo = 0, hi = R;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s_pre[mid] <= t_begin + lane)
                lo = mid;
            else
                hi = mid;
        }
        r = lo;
    }
    // kU items per lane per step: their list entries are loaded before any is
    // looked up, so a lane keeps kU global loads in flight
    constexpr int kU = 4;
    // the lane's current row in registers: its end in the item space, the
    // list offset of its items and its length word
    uint32_t r_end = 0, r_base = 0, r_len = 0;
    if (t_begin + lane < t_end) {
        r_end = s_pre[r + 1];
        r_base = s_hb[r] - s_pre[r];
        r_len = s_len[r];
    }
    for (uint32_t t = t_begin + lane; t < t_end; t += 32 * kU) {
        uint32_t rr[kU], wv[kU], lr[kU];
#pragma unroll
        for (int j = 0; j < kU; ++j) {
            const uint32_t tj = t + 32u * j;
            rr[j] = 0xffffffffu;
            wv[j] = 0;
            if (tj < t_end) {
                if (r_end <= tj) {
                    do
                        ++r;
                    while (s_pre[r + 1] <= tj);
                    r_end = s_pre[r + 1];
                    r_base = s_hb[r] - s_pre[r];
                    r_len = s_len[r];
                }
                rr[j] = r;
                lr[j] = r_len;
                if (!(r_len & kByA))
                    wv[j] = v.col[r_base + tj];
            }
        }
#pragma unroll
        for (int j = 0; j < kU; ++j) {
            const uint32_t rj = rr[j];
            if (rj == 0xffffffffu)
                continue;
            const uint32_t len = lr[j];
            const uint32_t xb = asc ? max(rj + 1, rlo) : 0, xe = asc ? D : rj;
            if (len & kByA) {
                const uint32_t k = xb + (t + 32u * j - s_pre[rj]);
                const uint32_t hb = s_hb[rj];
                if (contains_g(v.col, hb, hb + (len & ~kByA), A[k]))
                    set(rj, k);
            } else {
                const int k = hash_find(hkeys, hidx, nslots, hshift, wv[j]);
                if (k >= (int)xb && k < (int)xe)
                    set(rj, (uint32_t)k);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// work items. A pair is one (graph view, compiled query); an item is one root
// of one pair, packed as (pair << 32) | root. One launch per tier serves the
// items of every pair of a call (the plain count is a call with one pair).
// ---------------------------------------------------------------------------
// Slots after the per-pair counters: adjacency bytes read per tier (3), the
// algorithmic bytes of the searched roots per tier (3), 2 spare.
constexpr uint32_t kAux = 8;
// words of a pair's counter: (count, flag), (statistics plus, flag), (minus, flag)
constexpr uint32_t kPairWords = 6;

struct PairDev {
    ViewDev v;
    const uint32_t *g_rp, *g_col; // the graph's deduplicated input CSR (input ids)
    DevPlan pl;
    unsigned long long *count; // this pair's match count
    EnumDev en;                // enumeration output (out == nullptr: none)
    uint32_t min_deg;          // roots: degree >= max_qdeg ...
    uint32_t cap_deg;          // ... and < cap_deg (reference root cap, else 2^32-1)
    uint32_t shard_mod;        // > 1: only roots whose input id % shard_mod == shard_rem
    uint32_t shard_rem;
};

__device__ __forceinline__ uint32_t item_pair(uint64_t it) { return (uint32_t)(it >> 32); }
__device__ __forceinline__ uint32_t item_root(uint64_t it) { return (uint32_t)it; }

// The fields of a pair a kernel keeps in registers while it works on the
// pair's items (items are grouped by pair, so it reloads rarely).
struct PairRegs {
    ViewDev v;
    Lp lp;
    int restricted, pos1, asc, rows_needed;
    unsigned long long *count;
};

__device__ __forceinline__ void load_pair(const PairDev *__restrict__ pairs, uint32_t p, PairRegs &pr) {
    const PairDev &pd = pairs[p];
    pr.v = pd.v;
    pr.lp = load_lp(pd.pl);
    pr.restricted = pd.pl.restricted;
    pr.pos1 = pd.pl.pos1_after_root;
    pr.asc = pd.pl.asc;
    pr.rows_needed = pd.pl.rows_needed;
    pr.count = pd.count;
}

__device__ __forceinline__ void pair_domain(const PairRegs &pr, uint32_t r, uint32_t &beg, uint32_t &D,
                                            uint32_t &j0) {
    const uint32_t b = pr.v.rp[r], e = pr.v.rp[r + 1], sp = pr.v.split[r];
    if (pr.restricted) {
        beg = b + sp;
        D = e - b - sp;
        j0 = 0;
    } else {
        beg = b;
        D = e - b;
        // position 1 symmetric to the root: only neighbours after the root
        // (sgm_kernelsLD.cuh:60)
        j0 = pr.pos1 ? sp : 0;
    }
}

// First stored row of a root's bitmap: the plan reads the rows of level-1
// candidates only (j0), none (D) or all (0).
__device__ __forceinline__ uint32_t pair_rlo(const PairRegs &pr, uint32_t D, uint32_t j0) {
    return pr.rows_needed == 2 ? 0u : (pr.rows_needed == 1 ? j0 : D);
}

// ---------------------------------------------------------------------------
// small tier: a group of G lanes per root (G = 8 for domains of at most
// kTinyMaxD vertices, four roots per warp; G = 32 up to kSmallMaxD), 64-bit
// rows, one lane per level-1 vertex. Up to depth 4 the kernel is held to 51
// registers (five blocks per SM, no spills), a few percent faster on C2.
// ---------------------------------------------------------------------------
constexpr int kSmallWarps = 8;
constexpr int kTinyMaxD = 16;

template <int G> __device__ __forceinline__ unsigned long long group_sum(unsigned long long v, unsigned gmask) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1)
        v = sat_add(v, __shfl_xor_sync(gmask, v, o, G));
    return v;
}

// ---------------------------------------------------------------------------
// the 4-wheel in closed form on shared-memory rows (small and medium tiers)
// ---------------------------------------------------------------------------
// The same count as wheel4_task (large tier) for one x1 = a: U = OR of the
// rows of a's neighbours above a, then C(|row(a) & row(x3) above a|, 2) for
// every x3 of U above a. Rows of the whole domain (rlo = 0).
// One thread, rows of NW 64-bit words: row(a) and U stay in registers.
template <int NW>
__device__ __forceinline__ unsigned long long wheel4_thread(const uint64_t *rows, uint32_t a) {
    uint64_t ra[NW], U[NW];
    const uint32_t aw = a >> 6;
    const uint64_t above = ~((2ull << (a & 63)) - 1ull); // bits of word aw above a
#pragma unroll
    for (int k = 0; k < NW; ++k) {
        const uint64_t w = rows[(size_t)a * NW + k];
        ra[k] = (uint32_t)k > aw ? w : ((uint32_t)k == aw ? (w & above) : 0ull);
        U[k] = 0;
    }
#pragma unroll
    for (int k = 0; k < NW; ++k) {
        uint64_t w = ra[k];
        while (w) {
            const uint32_t b = (uint32_t)k * 64 + (uint32_t)(__ffsll((long long)w) - 1);
            w &= w - 1;
#pragma unroll
            for (int kk = 0; kk < NW; ++kk)
                U[kk] |= rows[(size_t)b * NW + kk];
        }
    }
    unsigned long long cnt = 0;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
        uint64_t u = (uint32_t)k > aw ? U[k] : ((uint32_t)k == aw ? (U[k] & above) : 0ull);
        while (u) {
            const uint32_t c = (uint32_t)k * 64 + (uint32_t)(__ffsll((long long)u) - 1);
            u &= u - 1;
            uint32_t n = 0;
#pragma unroll
            for (int kk = 0; kk < NW; ++kk)
                n += (uint32_t)__popcll(ra[kk] & rows[(size_t)c * NW + kk]);
            cnt = sat_add(cnt, (unsigned long long)n * (n - (n ? 1u : 0u)) / 2);
        }
    }
    return cnt;
}

// One warp, rows of W <= 32 32-bit words (lane k holds word k); the count is
// returned on lane 0.
__device__ __forceinline__ unsigned long long wheel4_warp(const uint32_t *rows, uint32_t W, uint32_t a, int lane) {
    const uint32_t k = (uint32_t)lane;
    const uint32_t aw = a >> 5;
    const uint32_t above = ~((2u << (a & 31)) - 1u);
    auto hi = [&](uint32_t w) { return k > aw ? w : (k == aw ? (w & above) : 0u); };
    const uint32_t ra = k < W ? hi(rows[(size_t)a * W + k]) : 0u;
    uint32_t U = 0, w = ra;
    unsigned bal = __ballot_sync(kFull, w != 0);
    while (bal) {
        const int L = __ffs(bal) - 1;
        const uint32_t ww = __shfl_sync(kFull, w, L);
        const uint32_t b = ((uint32_t)L << 5) + (uint32_t)(__ffs(ww) - 1);
        if (lane == L)
            w &= w - 1;
        if (k < W)
            U |= rows[(size_t)b * W + k];
        bal = __ballot_sync(kFull, w != 0);
    }
    uint32_t u = k < W ? hi(U) : 0u;
    unsigned long long cnt = 0;
    bal = __ballot_sync(kFull, u != 0);
    while (bal) {
        const int L = __ffs(bal) - 1;
        const uint32_t uu = __shfl_sync(kFull, u, L);
        const uint32_t c = ((uint32_t)L << 5) + (uint32_t)(__ffs(uu) - 1);
        if (lane == L)
            u &= u - 1;
        uint32_t n = k < W ? (uint32_t)__popc(ra & rows[(size_t)c * W + k]) : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            n += __shfl_xor_sync(kFull, n, o);
        if (lane == 0)
            cnt = sat_add(cnt, (unsigned long long)n * (n - (n ? 1u : 0u)) / 2);
        bal = __ballot_sync(kFull, u != 0);
    }
    return cnt;
}

template <int DEND, bool ENUM, int G, int MAXD>
__global__ void __launch_bounds__(kSmallWarps * 32, DEND <= 4 ? 5 : 1) k_small(const PairDev *__restrict__ pairs,
                                                           const uint64_t *__restrict__ items, uint32_t nitems,
                                                           unsigned long long *exit_t) {
    constexpr int NG = kSmallWarps * 32 / G; // groups per block
    __shared__ uint64_t s_rows[NG][MAXD];
    __shared__ uint32_t s_A[NG][MAXD];
    __shared__ uint32_t s_hb[NG][MAXD];
    __shared__ uint32_t s_len[NG][MAXD];
    __shared__ uint32_t s_pre[NG][MAXD + 1];
    const int gid = threadIdx.x / G, glane = threadIdx.x % G;
    const int lane = threadIdx.x & 31;
    const unsigned gmask = G == 32 ? kFull : (((1u << G) - 1u) << (lane & ~(G - 1)));
    uint64_t *rows = s_rows[gid];
    uint32_t *A = s_A[gid];
    PairRegs pr;
    uint32_t cur = 0xffffffffu;
    EnumCtx ec;
    unsigned long long cnt = 0;
    bool wheel = false; // the 4-wheel's closed form (counts)
    for (uint32_t ri = blockIdx.x * NG + gid; ri < nitems; ri += gridDim.x * NG) {
        const uint64_t it = items[ri];
        const uint32_t p = item_pair(it), r = item_root(it);
        if (p != cur) { // group-uniform
            cnt = group_sum<G>(cnt, gmask);
            if (glane == 0)
                flush_count(pr.count, cnt);
            cnt = 0;
            cur = p;
            load_pair(pairs, p, pr);
            if constexpr (ENUM)
                make_ec(ec, pairs[p].en, pairs[p].pl, pr.v);
            wheel = DEND == 5 && !ENUM && pairs[p].pl.wheel4;
        }
        if constexpr (ENUM) { // k tuples reserved: skip the root before its rows are built
            unsigned full = glane == 0 ? (unsigned)enum_full(ec) : 0u;
            full = __shfl_sync(gmask, full, 0, G);
            if (full)
                continue;
        }
        uint32_t beg, D, j0;
        pair_domain(pr, r, beg, D, j0);
        const uint32_t rlo = pair_rlo(pr, D, j0);
        for (uint32_t i = glane; i < D; i += G) {
            A[i] = pr.v.col[beg + i];
            rows[i] = 0;
        }
        __syncwarp(gmask);
        if (rlo < D)
            build_rows_flat<G>(pr.v, pr.asc, A, D, rlo, 0, D, s_hb[gid], s_pre[gid], s_len[gid], (uint32_t)glane,
                               (uint32_t)G, gmask, [&](uint32_t i, uint32_t k) {
                                   if (i >= rlo)
                                       atomicOr((unsigned long long *)&rows[i - rlo], 1ull << k);
                                   if (k >= rlo)
                                       atomicOr((unsigned long long *)&rows[k - rlo], 1ull << i);
                               });
        __syncwarp(gmask);
        if constexpr (ENUM) {
            ec.A = A;
            ec.root = r;
        }
        if (wheel) { // group-uniform; rows of the whole domain
            for (uint32_t j = j0 + glane; j < D; j += G)
                cnt = sat_add(cnt, wheel4_thread<1>(rows, j));
        } else if (DEND == 3 || pr.lp.free_from <= 2) { // group-uniform
            for (uint32_t j = j0 + glane; j < D; j += G) {
                uint32_t x[kMaxQ];
                x[1] = j;
                dfs_thread<2, DEND, ENUM, 1>(pr.lp, rows, rlo, D, x, cnt, ec);
            }
        } else {
            // one lane per (level-1, level-2) pair (see k_medium)
            const uint32_t n1 = D - j0;
            uint32_t *s_cnt = s_pre[gid];
            for (uint32_t i = glane; i < n1; i += G) {
                uint32_t x[kMaxQ];
                x[1] = j0 + i;
                const uint32_t lo2 = level_bound<2>(pr.lp, x);
                s_cnt[i] = (uint32_t)__popcll(cand_word<2, 1>(pr.lp, rows, rlo, D, lo2, x, 0));
            }
            __syncwarp(gmask);
            group_excl_scan<G>(s_cnt, n1, glane, gmask);
            __syncwarp(gmask);
            const uint32_t T = s_cnt[n1];
            for (uint32_t t = glane; t < T; t += G) {
                uint32_t a = 0, b = n1;
                while (b - a > 1) {
                    const uint32_t mid = (a + b) >> 1;
                    if (s_cnt[mid] <= t)
                        a = mid;
                    else
                        b = mid;
                }
                uint32_t x[kMaxQ];
                x[1] = j0 + a;
                const uint32_t lo2 = level_bound<2>(pr.lp, x);
                x[2] = select64(cand_word<2, 1>(pr.lp, rows, rlo, D, lo2, x, 0), t - s_cnt[a]);
                dfs_thread<3, DEND, ENUM, 1>(pr.lp, rows, rlo, D, x, cnt, ec);
            }
        }
        __syncwarp(gmask);
    }
    cnt = group_sum<G>(cnt, gmask);
    if (glane == 0)
        flush_count(pr.count, cnt);
    if (lane == 0)
        record_exit(exit_t);
}

// ---------------------------------------------------------------------------
// neighbourhood statistics in the medium tier (counts only). A five-vertex
// query whose plan has a statistics form (NbForm) is counted at a root from
// the root's rows of the whole domain, already in shared memory: d_u (popcount
// of row u), E and, per edge (u, w), the common neighbours row(u) & row(w) --
// the terms nbhd_task sums in the large tier, over the tasks u >= j0, into
// plus / minus. The walk would instead enumerate every (x1, x2, x3) prefix.
// Block-wide (block-uniform call); s_deg: D words, s_misc: 2 words.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void nbhd_term(int form, unsigned long long du, unsigned long long dw, uint32_t c_all,
                                          uint32_t c_above, unsigned long long rest, unsigned long long &plus,
                                          unsigned long long &minus, unsigned long long &tri) {
    switch (form) {
    case kNbTriIso: // triangles (u < w < x) once, times the isolated vertex's choices
        plus = sat_add(plus, sat_mul(c_above, rest));
        break;
    case kNbPath4: // paths x - u - w - y, minus the closed ones (x = y): 3T
        plus = sat_add(plus, (du - 1) * (dw - 1));
        minus = sat_add(minus, c_all);
        break;
    case kNbPaw: // triangles (u, w, x) with x after w: each once
        tri += c_above;
        break;
    case kNbDiamond: // C(common neighbours, 2) of the edge (u, w)
        plus = sat_add(plus, binom2(c_all));
        break;
    default:
        break;
    }
}

// Degrees of rows[0, D) into s_deg and their sum into s_misc[0]; a warp per
// row (rw words of 32 bits, at most 32), or a thread per row (rw > 32 words
// never occur here: the thread sub-tier's rows are 8 words).
__device__ __forceinline__ void nbhd_degrees(const uint32_t *rows, uint32_t rw, uint32_t D, uint32_t *s_deg,
                                             uint32_t *s_misc) {
    const int lane = threadIdx.x & 31;
    uint32_t part = 0;
    for (uint32_t u = threadIdx.x >> 5; u < D; u += blockDim.x >> 5) {
        uint32_t d = (uint32_t)lane < rw ? (uint32_t)__popc(rows[(size_t)u * rw + lane]) : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            d += __shfl_xor_sync(kFull, d, o);
        if (lane == 0) {
            s_deg[u] = d;
            part += d;
        }
    }
    if (lane == 0 && part)
        atomicAdd(&s_misc[0], part);
}

// Thread sub-tier: rows of NW 64-bit words, a thread per task u.
template <int NW>
__device__ __forceinline__ void nbhd_medium_thread(int form, const uint64_t *r64, uint32_t D, uint32_t j0,
                                                   uint32_t *s_deg, uint32_t *s_misc, unsigned long long &plus,
                                                   unsigned long long &minus) {
    if (threadIdx.x == 0) {
        s_misc[0] = 0;
        s_misc[1] = j0;
    }
    __syncthreads();
    nbhd_degrees(reinterpret_cast<const uint32_t *>(r64), 2 * NW, D, s_deg, s_misc);
    __syncthreads();
    const unsigned long long E = s_misc[0] / 2, rest = D >= 3 ? D - 3 : 0;
    if (form == kNbTwoEdges && threadIdx.x == 0)
        plus = sat_add(plus, binom2(E)); // C(E, 2): E < 2^15 here
    for (;;) {
        const uint32_t u = atomicAdd(&s_misc[1], 1u);
        if (u >= D)
            break;
        const unsigned long long du = s_deg[u];
        if (form == kNbWedgeIso) {
            plus = sat_add(plus, binom2(du) * rest);
            continue;
        }
        if (form == kNbTwoEdges) {
            minus = sat_add(minus, binom2(du));
            continue;
        }
        uint64_t ru[NW];
#pragma unroll
        for (int i = 0; i < NW; ++i)
            ru[i] = r64[(size_t)u * NW + i];
        const bool all_w = form == kNbPaw; // else the edges (u, w) with w after u
        const uint32_t ui = u >> 6;
        unsigned long long tri = 0;
#pragma unroll
        for (int i = 0; i < NW; ++i) {
            uint64_t bits = ru[i];
            if (!all_w)
                bits = (uint32_t)i < ui ? 0ull : ((uint32_t)i == ui ? (bits & ~((2ull << (u & 63)) - 1ull)) : bits);
            while (bits) {
                const uint32_t w = (uint32_t)i * 64 + (uint32_t)(__ffsll((long long)bits) - 1);
                bits &= bits - 1;
                const uint64_t *rw = r64 + (size_t)w * NW;
                const uint32_t wi = w >> 6;
                const uint64_t wm = ~((2ull << (w & 63)) - 1ull); // bits of word wi above w
                uint32_t c_all = 0, c_above = 0;
#pragma unroll
                for (int k = 0; k < NW; ++k) {
                    const uint64_t x = ru[k] & rw[k];
                    c_all += (uint32_t)__popcll(x);
                    c_above += (uint32_t)__popcll((uint32_t)k < wi ? 0ull : ((uint32_t)k == wi ? (x & wm) : x));
                }
                nbhd_term(form, du, s_deg[w], c_all, c_above, rest, plus, minus, tri);
            }
        }
        if (form == kNbPaw && du >= 2)
            plus = sat_add(plus, sat_mul(tri, du - 2));
    }
}

// Warp sub-tier: rows of W <= 32 words, a warp per task u (lane k holds word
// k of row u; each edge's common neighbours are one warp sum).
__device__ __forceinline__ void nbhd_medium_warp(int form, const uint32_t *rows, uint32_t W, uint32_t D,
                                                 uint32_t j0, uint32_t *s_deg, uint32_t *s_misc,
                                                 unsigned long long &plus, unsigned long long &minus) {
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        s_misc[0] = 0;
        s_misc[1] = j0;
    }
    __syncthreads();
    nbhd_degrees(rows, W, D, s_deg, s_misc);
    __syncthreads();
    const unsigned long long E = s_misc[0] / 2, rest = D >= 3 ? D - 3 : 0;
    if (form == kNbTwoEdges && threadIdx.x == 0)
        plus = sat_add(plus, binom2(E)); // C(E, 2): E < 2^19 here
    for (;;) {
        uint32_t u = 0;
        if (lane == 0)
            u = atomicAdd(&s_misc[1], 1u);
        u = __shfl_sync(kFull, u, 0);
        if (u >= D)
            break;
        const unsigned long long du = s_deg[u];
        if (form == kNbWedgeIso || form == kNbTwoEdges) {
            if (lane == 0) {
                if (form == kNbWedgeIso)
                    plus = sat_add(plus, binom2(du) * rest);
                else
                    minus = sat_add(minus, binom2(du));
            }
            continue;
        }
        const uint32_t ru = (uint32_t)lane < W ? rows[(size_t)u * W + lane] : 0u;
        const uint32_t uw = u >> 5;
        uint32_t bits = ru;
        if (form != kNbPaw)
            bits = (uint32_t)lane < uw ? 0u : ((uint32_t)lane == uw ? (bits & ~((2u << (u & 31)) - 1u)) : bits);
        unsigned long long tri = 0;
        unsigned bal = __ballot_sync(kFull, bits != 0);
        while (bal) {
            const int L = __ffs(bal) - 1;
            const uint32_t wb = __shfl_sync(kFull, bits, L);
            const uint32_t w = (uint32_t)L * 32 + (uint32_t)(__ffs(wb) - 1);
            if (lane == L)
                bits &= bits - 1;
            bal = __ballot_sync(kFull, bits != 0);
            const uint32_t x = (uint32_t)lane < W ? (ru & rows[(size_t)w * W + lane]) : 0u;
            const uint32_t wi = w >> 5;
            uint32_t c_all = (uint32_t)__popc(x);
            uint32_t c_above = (uint32_t)__popc((uint32_t)lane < wi ? 0u
                                                                     : ((uint32_t)lane == wi ? (x & ~((2u << (w & 31)) - 1u)) : x));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                c_all += __shfl_xor_sync(kFull, c_all, o);
                c_above += __shfl_xor_sync(kFull, c_above, o);
            }
            if (lane == 0)
                nbhd_term(form, du, s_deg[w], c_all, c_above, rest, plus, minus, tri);
        }
        if (form == kNbPaw && lane == 0 && du >= 2)
            plus = sat_add(plus, sat_mul(tri, du - 2));
    }
}

// ---------------------------------------------------------------------------
// medium tier: block per root, bitmap in shared memory
// ---------------------------------------------------------------------------
// G lanes per level-1 vertex (32: domains of up to 1024 vertices, rows of up
// to 32 words walked a warp at a time), or G = 0: one thread per level-1
// vertex over rows of 4 x 64 bits (domains of up to 256 vertices), the whole
// subtree in registers. The thread walker is latency-bound: up to depth 5 it
// is held to 64 registers (four 256-thread blocks per SM), which measured ~10%
// faster on C2 than 77 registers at three blocks; deeper walks keep 128
// registers to avoid spills.
template <int DEND, bool ENUM, int G>
__global__ void __launch_bounds__(G == 0 ? 256 : 1024, G == 0 ? (DEND <= 5 ? 4 : 2) : 1) k_medium(const PairDev *__restrict__ pairs,
                                                const uint64_t *__restrict__ items, uint32_t nitems,
                                                unsigned *cursor, uint32_t maxD, unsigned long long *exit_t) {
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t s_ri, s_j, s_full;
    const int lane = threadIdx.x & 31;
    const uint32_t pad = (maxD + 4) & ~3u;
    const uint32_t nslots = hash_slots(maxD), hshift = 32u - (uint32_t)__ffs((int)nslots) + 1u;
    uint32_t *A = sm;
    uint32_t *s_hb = sm + pad;
    uint32_t *s_pre = sm + 2 * pad;
    uint32_t *s_len = sm + 3 * pad;
    uint32_t *hkeys = sm + 4 * pad;                                 // domain hash: vertex ids ...
    uint16_t *hidx = reinterpret_cast<uint16_t *>(hkeys + nslots); // ... their domain indices, the filter
    uint32_t *rows = hkeys + nslots + nslots / 2 + nslots / 4;
    PairRegs pr;
    uint32_t cur = 0xffffffffu;
    EnumCtx ec;
    unsigned long long cnt = 0;
    bool wheel = false; // the 4-wheel's closed form (counts)
    int nbform = kNbNone; // a neighbourhood-statistics form (counts)
    unsigned long long nb_plus = 0, nb_minus = 0;
    for (;;) {
        if (threadIdx.x == 0)
            s_ri = atomicAdd(cursor, 1u);
        __syncthreads();
        const uint32_t ri = s_ri;
        if (ri >= nitems)
            break;
        const uint64_t it = items[ri];
        const uint32_t p = item_pair(it), r = item_root(it);
        if (p != cur) { // block-uniform
            cnt = warp_sum(cnt);
            nb_plus = warp_sum(nb_plus);
            nb_minus = warp_sum(nb_minus);
            if (lane == 0) {
                flush_count(pr.count, cnt);
                flush_count(pr.count + 2, nb_plus);
                flush_count(pr.count + 4, nb_minus);
            }
            cnt = nb_plus = nb_minus = 0;
            cur = p;
            load_pair(pairs, p, pr);
            if constexpr (ENUM)
                make_ec(ec, pairs[p].en, pairs[p].pl, pr.v);
            wheel = DEND == 5 && !ENUM && pairs[p].pl.wheel4;
            nbform = (DEND == 5 && !ENUM) ? (int)pairs[p].pl.nbhd : (int)kNbNone;
        }
        if constexpr (ENUM) { // k tuples reserved: skip the root before its rows are built
            if (threadIdx.x == 0)
                s_full = enum_full(ec) ? 1u : 0u;
            __syncthreads();
            const bool full = s_full != 0;
            __syncthreads(); // every thread has read s_full before thread 0 writes it again
            if (full)
                continue;
        }
        uint32_t beg, D, j0;
        pair_domain(pr, r, beg, D, j0);
        const uint32_t rlo = pair_rlo(pr, D, j0);
        const uint32_t W = (D + 31) >> 5;
        const uint32_t row_words = G == 0 ? 2 * kThreadNW : W; // 32-bit words per row
        for (uint32_t i = threadIdx.x; i < D; i += blockDim.x)
            A[i] = pr.v.col[beg + i];
        for (uint32_t i = threadIdx.x; i < (D - rlo) * row_words; i += blockDim.x)
            rows[i] = 0;
        if (threadIdx.x == 0)
            s_j = j0;
        __syncthreads();
        if (rlo < D) { // block-uniform
            hash_build(A, D, hkeys, hidx, nslots, hshift);
            __syncthreads();
            if constexpr (G == 0) {
                unsigned long long *r64 = reinterpret_cast<unsigned long long *>(rows);
                build_rows_hashed(pr.v, pr.asc, A, D, rlo, s_hb, s_pre, s_len, hkeys, hidx, nslots, hshift,
                                  [&](uint32_t i, uint32_t k) {
                                      if (i >= rlo)
                                          atomicOr(&r64[(size_t)(i - rlo) * kThreadNW + (k >> 6)], 1ull << (k & 63));
                                      if (k >= rlo)
                                          atomicOr(&r64[(size_t)(k - rlo) * kThreadNW + (i >> 6)], 1ull << (i & 63));
                                  });
            } else {
                build_rows_hashed(pr.v, pr.asc, A, D, rlo, s_hb, s_pre, s_len, hkeys, hidx, nslots, hshift,
                                  [&](uint32_t i, uint32_t k) {
                                      if (i >= rlo)
                                          atomicOr(&rows[(size_t)(i - rlo) * W + (k >> 5)], 1u << (k & 31));
                                      if (k >= rlo)
                                          atomicOr(&rows[(size_t)(k - rlo) * W + (i >> 5)], 1u << (i & 31));
                                  });
            }
        }
        __syncthreads();
        if constexpr (ENUM) {
            ec.A = A;
            ec.root = r;
        }
        bool stats_done = false; // counted by the neighbourhood statistics
        if constexpr (DEND == 5 && !ENUM) {
            if (nbform) { // block-uniform; rows of the whole domain
                if constexpr (G == 0)
                    nbhd_medium_thread<kThreadNW>(nbform, reinterpret_cast<const uint64_t *>(rows), D, j0, s_hb,
                                                  s_len, nb_plus, nb_minus);
                else
                    nbhd_medium_warp(nbform, rows, W, D, j0, s_hb, s_len, nb_plus, nb_minus);
                stats_done = true;
            }
        }
        if (stats_done) {
        } else if constexpr (G == 0) {
            const uint64_t *r64 = reinterpret_cast<const uint64_t *>(rows);
            if (wheel) { // block-uniform; rows of the whole domain
                for (;;) {
                    const uint32_t j = atomicAdd(&s_j, 1u);
                    if (j >= D)
                        break;
                    cnt = sat_add(cnt, wheel4_thread<kThreadNW>(r64, j));
                }
            } else if (DEND == 3 || pr.lp.free_from <= 2) { // block-uniform
                // level 2 is the last or is counted in closed form: O(1) per level-1 vertex
                for (;;) {
                    const uint32_t j = atomicAdd(&s_j, 1u);
                    if (j >= D)
                        break;
                    uint32_t x[kMaxQ];
                    x[1] = j;
                    dfs_thread<2, DEND, ENUM, kThreadNW>(pr.lp, r64, rlo, D, x, cnt, ec);
                }
            } else {
                // one thread per (level-1, level-2) pair, so that threads get
                // even shares whatever the level-1 vertices' candidate counts
                const uint32_t n1 = D - j0, nw = (D + 63) >> 6;
                uint32_t *s_cnt = s_pre; // free again once the rows are built
                for (uint32_t i = threadIdx.x; i < n1; i += blockDim.x) {
                    uint32_t x[kMaxQ];
                    x[1] = j0 + i;
                    const uint32_t lo2 = level_bound<2>(pr.lp, x);
                    uint32_t c = 0;
                    for (uint32_t k = lo2 >> 6; k < nw; ++k)
                        c += (uint32_t)__popcll(cand_word<2, kThreadNW>(pr.lp, r64, rlo, D, lo2, x, k));
                    s_cnt[i] = c;
                }
                __syncthreads();
                if (threadIdx.x < 32)
                    warp_excl_scan(s_cnt, n1, (int)threadIdx.x);
                __syncthreads();
                const uint32_t T = s_cnt[n1];
                for (uint32_t t = threadIdx.x; t < T; t += blockDim.x) {
                    uint32_t a = 0, b = n1; // last i with s_cnt[i] <= t
                    while (b - a > 1) {
                        const uint32_t mid = (a + b) >> 1;
                        if (s_cnt[mid] <= t)
                            a = mid;
                        else
                            b = mid;
                    }
                    uint32_t x[kMaxQ];
                    x[1] = j0 + a;
                    const uint32_t lo2 = level_bound<2>(pr.lp, x);
                    uint32_t j = t - s_cnt[a];
                    uint32_t k = lo2 >> 6;
                    uint64_t w = cand_word<2, kThreadNW>(pr.lp, r64, rlo, D, lo2, x, k);
                    for (uint32_t pc = (uint32_t)__popcll(w); j >= pc; pc = (uint32_t)__popcll(w)) {
                        j -= pc;
                        w = cand_word<2, kThreadNW>(pr.lp, r64, rlo, D, lo2, x, ++k);
                    }
                    x[2] = k * 64 + select64(w, j);
                    dfs_thread<3, DEND, ENUM, kThreadNW>(pr.lp, r64, rlo, D, x, cnt, ec);
                }
            }
        } else {
            const int glane = lane & (G - 1);
            const unsigned gmask = G == 32 ? kFull : (((1u << G) - 1u) << (lane & ~(G - 1)));
            for (;;) {
                uint32_t j = 0;
                if (glane == 0)
                    j = atomicAdd(&s_j, 1u);
                j = __shfl_sync(gmask, j, 0, G);
                if (j >= D)
                    break;
                if constexpr (G == 32) {
                    if (wheel) { // block-uniform; rows of the whole domain
                        cnt = sat_add(cnt, wheel4_warp(rows, W, j, glane));
                        continue;
                    }
                }
                uint32_t x[kMaxQ];
                x[1] = j;
                dfs_warp<2, DEND, ENUM, G>(pr.lp, rows, rlo, W, D, x, cnt, glane, ec, gmask);
            }
        }
        __syncthreads();
    }
    cnt = warp_sum(cnt);
    nb_plus = warp_sum(nb_plus);
    nb_minus = warp_sum(nb_minus);
    if (lane == 0) {
        flush_count(pr.count, cnt);
        flush_count(pr.count + 2, nb_plus);
        flush_count(pr.count + 4, nb_minus);
    }
    if (threadIdx.x == 0)
        record_exit(exit_t);
}

// ---------------------------------------------------------------------------
// large tier: rows of a batch of roots in a global arena
// ---------------------------------------------------------------------------
struct Batch {
    const uint64_t *item;    // [nb] (pair, root)
    const uint64_t *off;     // [nb] word offset of the root's rows in the arena
    const uint32_t *cstart;  // [nb+1] prefix of row chunks
    const uint32_t *tstart;  // [nb+1] prefix of DFS tasks (level-1 vertices)
    uint32_t nb;
};

constexpr uint32_t kRowsPerChunk = 256;
constexpr int kLargeDfsBlocksPerSm = 8; // k_large_wheel grid: 256-thread blocks per SM
constexpr uint32_t kDonCap = 1u << 18;   // donated tasks per walk launch (16 MiB of records)
constexpr uint32_t kCursorBlock = 256;   // work cursors allocated at a time
constexpr uint32_t kWheelGroupMin = 16;  // 4-wheel pair phase by 8-lane groups from this x1 list length
constexpr uint32_t kMaxDonLaunches = 64; // walk launches of a call with a donation queue
// Depth slot of a root in the tier lists: its plan's depth, except the large
// tier's 4-wheel roots, which take slot 2 (no plan has depth 2) and run on
// k_large_wheel.
constexpr uint32_t kWheelSlot = 2;
constexpr int kDepthsConst = 11; // dend 0..10
// Slots kDepthsConst.. hold the same depths for enumerating pairs, which run
// in launches of their own (the walk that writes tuples, with no closed
// forms), so that counting pairs of the same call keep theirs.
constexpr uint32_t kNbhdSlot = 1; // the large tier's roots of neighbourhood-statistics plans
__host__ __device__ __forceinline__ uint32_t depth_slot(const DevPlan &pl, uint32_t tier, bool enumerating) {
    return (enumerating ? (uint32_t)kDepthsConst : 0u) +
           ((tier == 4 && pl.wheel4) ? kWheelSlot : ((tier == 4 && pl.nbhd) ? kNbhdSlot : (uint32_t)pl.dend));
}
constexpr uint32_t kLargeSmemA = 48 * 1024; // domain entries staged in shared memory

// Rows of at least kListMinW words also get non-zero-word lists of
// W / 8 entries (rounded down to 32): 1 + W / 8 more words a row, under 13%.
constexpr uint32_t kListMinW = 256;
__host__ __device__ __forceinline__ uint32_t list_cap(uint32_t W) { return W >= kListMinW ? (W / 8) & ~31u : 0u; }

// Arena words of one large root: rows [rlo, D) of W = ceil(D / 32) words,
// then (list_cap(W) > 0) each row's non-zero word count and its list,
// rounded up to 32 words.
// Roots of a neighbourhood-statistics plan keep, after their rows and lists,
// the degree of every domain vertex in the neighbourhood graph (D words,
// rounded up to even) and its edge count (one u64).
__host__ __device__ __forceinline__ uint64_t nb_deg_offset(uint32_t D, uint32_t rlo) {
    const uint32_t W = (D + 31) / 32, cap = list_cap(W);
    return ((uint64_t)(D - rlo) * (W + (cap ? cap + 1 : 0)) + 1) & ~(uint64_t)1;
}
__host__ __device__ __forceinline__ uint64_t nb_edges_offset(uint32_t D, uint32_t rlo) {
    return nb_deg_offset(D, rlo) + ((uint64_t)(D + 1) & ~(uint64_t)1);
}
__host__ __device__ __forceinline__ uint64_t large_root_words(uint32_t D, uint32_t rlo, bool nb = false) {
    return ((nb ? nb_edges_offset(D, rlo) + 2 : nb_deg_offset(D, rlo)) + 31) & ~(uint64_t)31;
}

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

__global__ void __launch_bounds__(512) k_large_rows(const PairDev *__restrict__ pairs, Batch bt, uint32_t *arena,
                                                    unsigned *cursor) {
    extern __shared__ __align__(16) uint32_t sA[];
    __shared__ uint32_t s_c;
    __shared__ uint32_t s_hb[kRowsPerChunk], s_len[kRowsPerChunk], s_pre[kRowsPerChunk + 1];
    const uint32_t total = bt.cstart[bt.nb];
    for (;;) {
        if (threadIdx.x == 0)
            s_c = atomicAdd(cursor, 1u);
        __syncthreads();
        const uint32_t c = s_c;
        if (c >= total)
            break;
        const uint32_t b = find_batch(bt.cstart, bt.nb, c);
        const uint64_t it = bt.item[b];
        PairRegs pr;
        load_pair(pairs, item_pair(it), pr);
        uint32_t beg, D, j0;
        pair_domain(pr, item_root(it), beg, D, j0);
        const uint32_t rlo = pair_rlo(pr, D, j0);
        const uint32_t W = (D + 31) >> 5;
        uint32_t *rows = arena + bt.off[b];
        const uint32_t i0 = (c - bt.cstart[b]) * kRowsPerChunk;
        const uint32_t i1 = min(D, i0 + kRowsPerChunk);
        const uint32_t *A = pr.v.col + beg;
        if (D <= kLargeSmemA) {
            for (uint32_t i = threadIdx.x; i < D; i += blockDim.x)
                sA[i] = A[i];
            __syncthreads();
            A = sA;
        }
        if (rlo < D) // block-uniform
            build_rows_flat<0>(pr.v, pr.asc, A, D, rlo, i0, i1, s_hb, s_pre, s_len, threadIdx.x, blockDim.x, kFull,
                               [&](uint32_t i, uint32_t k) {
                                   if (i >= rlo)
                                       atomicOr(&rows[(size_t)(i - rlo) * W + (k >> 5)], 1u << (k & 31));
                                   if (k >= rlo)
                                       atomicOr(&rows[(size_t)(k - rlo) * W + (i >> 5)], 1u << (i & 31));
                               });
        __syncthreads();
    }
}

// Non-zero-word counts and lists of the rows k_large_rows built (roots with
// list_cap(W) > 0 only): a warp per row, 32 words a step. Blocks take the
// 256-row chunks of the batch in turn.
__global__ void __launch_bounds__(256) k_large_lists(const PairDev *__restrict__ pairs, Batch bt, uint32_t *arena) {
    const uint32_t total = bt.cstart[bt.nb];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
        const uint32_t b = find_batch(bt.cstart, bt.nb, c);
        const uint64_t it = bt.item[b];
        PairRegs pr;
        load_pair(pairs, item_pair(it), pr);
        uint32_t beg, D, j0;
        pair_domain(pr, item_root(it), beg, D, j0);
        const uint32_t W = (D + 31) >> 5, cap = list_cap(W);
        if (cap == 0)
            continue;
        const uint32_t rlo = pair_rlo(pr, D, j0);
        const uint32_t *rows = arena + bt.off[b];
        uint32_t *nzc = arena + bt.off[b] + (size_t)(D - rlo) * W;
        uint32_t *nzl = nzc + (D - rlo);
        const uint32_t i0 = max(rlo, (c - bt.cstart[b]) * kRowsPerChunk);
        const uint32_t i1 = min(D, (c - bt.cstart[b] + 1) * kRowsPerChunk);
        for (uint32_t i = i0 + warp; i < i1; i += nwarps) {
            const uint32_t *row = rows + (size_t)(i - rlo) * W;
            uint32_t *lst = nzl + (size_t)(i - rlo) * cap;
            uint32_t n = 0;
#pragma unroll 4
            for (uint32_t k0 = 0; k0 < W; k0 += 32) {
                const uint32_t k = k0 + (uint32_t)lane;
                const uint32_t w = k < W ? row[k] : 0u;
                const unsigned bal = __ballot_sync(kFull, w != 0);
                const uint32_t pos = n + (uint32_t)__popc(bal & ((1u << lane) - 1u));
                if (w != 0 && pos < cap)
                    lst[pos] = k;
                n += (uint32_t)__popc(bal);
            }
            if (lane == 0)
                nzc[i - rlo] = n;
        }
    }
}

// ---------------------------------------------------------------------------
// the 4-wheel in closed form per (x1, x3) pair (large tier, counts only)
// ---------------------------------------------------------------------------
// Plan (the reference's chain for the 4-wheel): x2 in row(x1), x2 > x1;
// x3 in row(x2), x3 > x1; x4 in row(x1) & row(x3), x4 > x1, x4 > x2. For a
// fixed (x1, x3), x2 and x4 are two elements of S = row(x1) & row(x3) above
// x1 with x2 < x4: C(|S|, 2) completions. A task (root, x1) therefore
// collects the x3 > x1 that share a neighbour above x1 with x1 -- the OR U of
// the rows of those neighbours, with the list of U's non-zero words -- and
// counts S once per x3, instead of walking every (x2, x3) path: on R-MAT hub
// neighbourhoods the paths outnumber the distinct pairs about 30 to 1.
//
// Scratch per warp (U zero on entry and left zero on exit): U and its word
// list tl (W words each), and la (W words) for x1's non-zero words when its
// row has no list. Rows are those of the whole domain (rlo = 0).
__device__ __forceinline__ void wheel4_task(const uint32_t *__restrict__ bm, const RowLists &rl, uint32_t W,
                                            uint32_t a, uint32_t *U, uint32_t *U2, uint32_t *tl, uint32_t *la,
                                            int lane, unsigned long long &cnt) {
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t *ra = bm + (size_t)a * W;
    const uint32_t aw = a >> 5;
    const uint32_t above = ~((2u << (a & 31)) - 1u); // bits of word aw above a
    // non-zero words of row(a) at or above aw: its list, or a scan into la
    const uint32_t *al = la;
    uint32_t na = 0;
    if (rl.cap && rl.nzc[a] <= rl.cap) {
        al = rl.nzl + (size_t)a * rl.cap;
        na = rl.nzc[a];
    } else {
        for (uint32_t k0 = aw & ~31u; k0 < W; k0 += 32) {
            const uint32_t k = k0 + (uint32_t)lane;
            const uint32_t w = (k < W && k >= aw) ? ra[k] : 0u;
            const unsigned bal = __ballot_sync(kFull, w != 0);
            if (w)
                la[na + (uint32_t)__popc(bal & lt)] = k;
            na += (uint32_t)__popc(bal);
        }
        __syncwarp();
    }
    // U = OR over b in row(a), b > a, of row(b)'s bits above a; tl lists U's
    // non-zero words. U2 keeps the bits OR-ed in at least twice: an x3 reached
    // from one b only has c = |row(a) & row(x3) above a| = 1 and C(1, 2) = 0,
    // so only U2's x3 need the pair phase (c counts exactly the b whose row
    // holds x3).
    uint32_t nt = 0;
    auto or_word = [&](const uint32_t *rb, uint32_t k) {
        uint32_t v = 0;
        if (k < W && k >= aw) {
            v = rb[k];
            if (k == aw)
                v &= above;
        }
        bool fresh = false;
        if (v) {
            const uint32_t old = U[k];
            fresh = old == 0;
            U[k] = old | v;
            if (old & v)
                U2[k] |= old & v;
        }
        const unsigned fb = __ballot_sync(kFull, fresh);
        if (fresh)
            tl[nt + (uint32_t)__popc(fb & lt)] = k;
        nt += (uint32_t)__popc(fb);
    };
    for (uint32_t i = 0; i < na; ++i) {
        const uint32_t e = al[i];
        if (e < aw)
            continue;
        uint32_t wa = ra[e];
        if (e == aw)
            wa &= above;
        while (wa) {
            const uint32_t b = (e << 5) + (uint32_t)(__ffs(wa) - 1);
            wa &= wa - 1;
            const uint32_t *rb = bm + (size_t)b * W;
            const uint32_t nb = rl.cap ? rl.nzc[b] : 0xffffffffu;
            if (nb <= rl.cap) {
                const uint32_t *bl = rl.nzl + (size_t)b * rl.cap;
                for (uint32_t j0 = 0; j0 < nb; j0 += 32)
                    or_word(rb, j0 + (uint32_t)lane < nb ? bl[j0 + lane] : 0xffffffffu);
            } else {
                for (uint32_t k0 = aw & ~31u; k0 < W; k0 += 32)
                    or_word(rb, k0 + (uint32_t)lane);
            }
            __syncwarp(); // U's words visible to every lane before the next row
        }
    }
    // every x3 of U: |S| over the shorter of the two word lists. With a long
    // list for x1 (na >= kWheelGroupMin words), groups of 8 lanes take four
    // x3 at a time and read 8 consecutive list entries and their words at
    // once; otherwise each lane walks its own x3's short list (R-MAT hubs of
    // ~10^4: 337 -> 230 ms for the large tier's 4-wheel; sparse Chung-Lu
    // neighbourhoods: no gain from groups).
    if (na >= kWheelGroupMin) {
        const uint32_t grp = (uint32_t)lane >> 3, gl = (uint32_t)lane & 7u;
        for (uint32_t t0 = 0; t0 < nt; t0 += 32) {
            uint32_t u = 0, k = 0;
            if (t0 + (uint32_t)lane < nt) {
                k = tl[t0 + lane];
                u = U2[k];
                U[k] = 0;
                U2[k] = 0;
            }
            for (;;) {
                uint32_t c = 0xffffffffu;
#pragma unroll
                for (uint32_t g = 0; g < 4; ++g) {
                    const unsigned bal = __ballot_sync(kFull, u != 0);
                    if (!bal)
                        break;
                    const int L = __ffs(bal) - 1;
                    const uint32_t uL = __shfl_sync(kFull, u, L), kL = __shfl_sync(kFull, k, L);
                    if (lane == L)
                        u &= u - 1;
                    if (grp == g)
                        c = (kL << 5) + (uint32_t)(__ffs(uL) - 1);
                }
                if (!__ballot_sync(kFull, c != 0xffffffffu))
                    break;
                uint32_t s = 0;
                if (c != 0xffffffffu) {
                    const uint32_t *rc = bm + (size_t)c * W;
                    const uint32_t ncw = rl.cap ? rl.nzc[c] : 0xffffffffu;
                    const bool use_c = ncw <= rl.cap && ncw < na;
                    const uint32_t *lst = use_c ? rl.nzl + (size_t)c * rl.cap : al;
                    const uint32_t n = use_c ? ncw : na;
                    for (uint32_t i = gl; i < n; i += 8) {
                        const uint32_t e = lst[i];
                        if (e < aw)
                            continue;
                        const uint32_t w = ra[e] & rc[e];
                        s += (uint32_t)__popc(e == aw ? (w & above) : w);
                    }
                }
                s += __shfl_xor_sync(kFull, s, 1);
                s += __shfl_xor_sync(kFull, s, 2);
                s += __shfl_xor_sync(kFull, s, 4);
                if (gl == 0 && c != 0xffffffffu)
                    cnt = sat_add(cnt, (unsigned long long)s * (s - (s ? 1u : 0u)) / 2);
            }
        }
        __syncwarp(); // U back to zero before the warp's next task
        return;
    }
    for (uint32_t t0 = 0; t0 < nt; t0 += 32) {
        uint32_t u = 0, k = 0;
        if (t0 + (uint32_t)lane < nt) {
            k = tl[t0 + lane];
            u = U2[k];
            U[k] = 0;
            U2[k] = 0;
        }
        while (u) {
            const uint32_t c = (k << 5) + (uint32_t)(__ffs(u) - 1);
            u &= u - 1;
            const uint32_t *rc = bm + (size_t)c * W;
            const uint32_t ncw = rl.cap ? rl.nzc[c] : 0xffffffffu;
            const bool use_c = ncw <= rl.cap && ncw < na;
            const uint32_t *lst = use_c ? rl.nzl + (size_t)c * rl.cap : al;
            const uint32_t n = use_c ? ncw : na;
            uint32_t s = 0;
            for (uint32_t i = 0; i < n; ++i) {
                const uint32_t e = lst[i];
                if (e < aw)
                    continue;
                const uint32_t w = ra[e] & rc[e];
                s += (uint32_t)__popc(e == aw ? (w & above) : w);
            }
            cnt = sat_add(cnt, (unsigned long long)s * (s - (s ? 1u : 0u)) / 2);
        }
    }
    __syncwarp(); // U back to zero before the warp's next task
}

// A donated task of level P resumes the walk at that level over its
// iteration range (the task's x[2 .. P-1] restored first).
template <int P, int DEND, bool ENUM>
__device__ __forceinline__ void run_donated(const Lp &lp, const uint32_t *rows, uint32_t rlo, uint32_t W, uint32_t D,
                                            uint32_t (&x)[kMaxQ], unsigned long long &cnt, int lane,
                                            const EnumCtx &ec, const RowLists &rl, DonCtx &dc, const DonTask &t) {
    if constexpr (P < DEND - 1) {
        if (t.level == (uint32_t)P) {
#pragma unroll
            for (int q = 2; q < P; ++q)
                x[q] = t.x[q - 2];
            dfs_warp<P, DEND, ENUM, 32, true, true>(lp, rows, rlo, W, D, x, cnt, lane, ec, kFull, rl, &dc, t.it_lo,
                                                     t.it_hi);
            return;
        }
        run_donated<P + 1, DEND, ENUM>(lp, rows, rlo, W, D, x, cnt, lane, ec, rl, dc, t);
    }
}

// The large tier's walks: every warp takes (root, x1) tasks from the cursor,
// then waits for donated ones (see the donation comment above) until none
// can come. exit_t (may be null): the earliest and latest warp exit times.
template <int DEND, bool ENUM>
__global__ void __launch_bounds__(256, (!ENUM && DEND <= 5) ? 3 : 1) k_large_dfs(const PairDev *__restrict__ pairs, Batch bt,
                                                                      const uint32_t *arena, unsigned *cursor,
                                                                      const __grid_constant__ Don dn,
                                                                      unsigned long long *exit_t) {
    const int lane = threadIdx.x & 31;
    const uint32_t base0 = bt.tstart[0]; // the items' tasks are tstart[0] .. tstart[nb] - 1
    const uint32_t total = bt.tstart[bt.nb] - base0;
    PairRegs pr;
    uint32_t cur = 0xffffffffu;
    EnumCtx ec;
    unsigned long long cnt = 0;
    DonCtx dc;
    dc.dn = &dn;
    // pair registers, domain and rows of batch entry b
    uint32_t D = 0, W = 0, rlo = 0, j0 = 0;
    const uint32_t *rows = nullptr;
    RowLists rl;
    auto setup = [&](uint32_t b) {
        const uint64_t it = bt.item[b];
        const uint32_t p = item_pair(it), r = item_root(it);
        if (p != cur) {
            cnt = warp_sum(cnt);
            if (lane == 0)
                flush_count(pr.count, cnt);
            cnt = 0;
            cur = p;
            load_pair(pairs, p, pr);
            if constexpr (ENUM)
                make_ec(ec, pairs[p].en, pairs[p].pl, pr.v);
        }
        uint32_t beg;
        pair_domain(pr, r, beg, D, j0);
        W = (D + 31) >> 5;
        if constexpr (ENUM) {
            ec.A = pr.v.col + beg;
            ec.root = r;
        }
        rlo = pair_rlo(pr, D, j0);
        rows = arena + bt.off[b];
        rl.cap = list_cap(W);
        rl.nzc = rows + (size_t)(D - rlo) * W;
        rl.nzl = rl.nzc + (D - rlo);
    };
    for (;;) {
        uint32_t t = 0;
        if (lane == 0)
            t = atomicAdd(cursor, 1u);
        t = __shfl_sync(kFull, t, 0);
        if (t >= total)
            break;
        t += base0;
        const uint32_t b = find_batch(bt.tstart, bt.nb, t);
        setup(b);
        uint32_t x[kMaxQ];
        x[1] = j0 + (t - bt.tstart[b]);
        dc.b = b;
        dc.x1 = x[1];
        bool skip = false; // k tuples reserved: nothing left to walk
        if constexpr (ENUM) {
            unsigned full = lane == 0 ? (unsigned)enum_full(ec) : 0u;
            skip = __shfl_sync(kFull, full, 0) != 0;
        }
        if (skip) {
        } else if (dn.cap)
            dfs_warp<2, DEND, ENUM, 32, true, true>(pr.lp, rows, rlo, W, D, x, cnt, lane, ec, kFull, rl, &dc);
        else
            dfs_warp<2, DEND, ENUM, 32, true>(pr.lp, rows, rlo, W, D, x, cnt, lane, ec, kFull, rl);
        if (dn.cap && lane == 0) {
            __threadfence(); // this task's donations are counted before it is
            atomicAdd(&dn.ctl[kDonStaticDone], 1u);
        }
    }
    while (dn.cap) {
        // claim the next slot and wait until a donor fills it or no work is left
        uint32_t st = 0, idx = 0; // st: 1 a task, 2 leave
        if (lane == 0) {
            idx = atomicAdd(&dn.ctl[kDonHead], 1u);
            if (idx >= dn.cap) {
                st = 2;
            } else {
                const unsigned *ctl = dn.ctl;
                auto progress = [&]() {
                    return ld_volatile(&ctl[kDonTail]) + ld_volatile(&ctl[kDonHeartbeat]) +
                           ld_volatile(&ctl[kDonStaticDone]) + ld_volatile(&ctl[kDonDone]);
                };
                unsigned seen = progress();
                unsigned long long t0 = global_ns();
                unsigned sleep_ns = 32;
                for (;;) {
                    if (ld_volatile(&dn.ready[idx])) {
                        st = 1;
                        break;
                    }
                    if (ld_volatile(&ctl[kDonError])) {
                        st = 2;
                        break;
                    }
                    if (ld_volatile(&ctl[kDonStaticDone]) >= total) {
                        __threadfence();
                        if (ld_volatile(&ctl[kDonPending]) == 0) {
                            st = 2;
                            break;
                        }
                    }
                    const unsigned now_p = progress();
                    const unsigned long long now = global_ns();
                    if (now_p != seen) {
                        seen = now_p;
                        t0 = now;
                    } else if (now - t0 > dn.timeout_ns) {
                        atomicExch(&dn.ctl[kDonError], 1u);
                        st = 2;
                        break;
                    }
                    __nanosleep(sleep_ns);
                    if (sleep_ns < 2048)
                        sleep_ns *= 2;
                }
            }
        }
        st = __shfl_sync(kFull, st, 0);
        idx = __shfl_sync(kFull, idx, 0);
        if (st != 1)
            break;
        __threadfence();
        DonTask t;
        {
            // written by another SM: read past L1
            const unsigned *src = reinterpret_cast<const unsigned *>(dn.tasks + idx);
            unsigned *dst = reinterpret_cast<unsigned *>(&t);
#pragma unroll
            for (int i = 0; i < 16; ++i)
                dst[i] = __ldcg(src + i);
        }
        setup(t.b);
        uint32_t x[kMaxQ];
        x[1] = t.x1;
        dc.b = t.b;
        dc.x1 = t.x1;
        run_donated<2, DEND, ENUM>(pr.lp, rows, rlo, W, D, x, cnt, lane, ec, rl, dc, t);
        if (lane == 0) {
            __threadfence();
            atomicAdd(&dn.ctl[kDonDone], 1u);
            atomicSub(&dn.ctl[kDonPending], 1u);
        }
    }
    cnt = warp_sum(cnt);
    if (lane == 0)
        flush_count(pr.count, cnt);
    if (lane == 0)
        record_exit(exit_t);
}

// The large tier's 4-wheel roots (classified into depth slot kWheelSlot):
// every warp takes (root, x1) tasks from the cursor and runs wheel4_task on
// its own scratch, wstride words at wsc + warp * wstride.
__global__ void __launch_bounds__(256) k_large_wheel(const PairDev *__restrict__ pairs, Batch bt,
                                                     const uint32_t *arena, unsigned *cursor, uint32_t *wsc,
                                                     uint32_t wstride, unsigned long long *exit_t) {
    const int lane = threadIdx.x & 31;
    const uint32_t base0 = bt.tstart[0];
    const uint32_t total = bt.tstart[bt.nb] - base0;
    // four regions of Wm >= every root's W words at fixed places: U (zero on
    // entry and on exit), U's word list, x1's word list, U2 (zero on entry
    // and on exit)
    const uint32_t Wm = wstride / 4;
    uint32_t *ws = wsc + (size_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * wstride;
    PairRegs pr;
    uint32_t cur = 0xffffffffu;
    unsigned long long cnt = 0;
    for (;;) {
        uint32_t t = 0;
        if (lane == 0)
            t = atomicAdd(cursor, 1u);
        t = __shfl_sync(kFull, t, 0);
        if (t >= total)
            break;
        t += base0;
        const uint32_t b = find_batch(bt.tstart, bt.nb, t);
        const uint64_t it = bt.item[b];
        const uint32_t p = item_pair(it), r = item_root(it);
        if (p != cur) {
            cnt = warp_sum(cnt);
            if (lane == 0)
                flush_count(pr.count, cnt);
            cnt = 0;
            cur = p;
            load_pair(pairs, p, pr);
        }
        uint32_t beg, D, j0;
        pair_domain(pr, r, beg, D, j0);
        const uint32_t W = (D + 31) >> 5;
        const uint32_t *rows = arena + bt.off[b]; // rows of the whole domain: rlo == 0
        RowLists rl;
        rl.cap = list_cap(W);
        rl.nzc = rows + (size_t)D * W;
        rl.nzl = rl.nzc + D;
        wheel4_task(rows, rl, W, j0 + (t - bt.tstart[b]), ws, ws + 3 * (size_t)Wm, ws + Wm, ws + 2 * (size_t)Wm, lane,
                    cnt);
    }
    cnt = warp_sum(cnt);
    if (lane == 0)
        flush_count(pr.count, cnt);
    if (lane == 0)
        record_exit(exit_t);
}

// ---------------------------------------------------------------------------
// neighbourhood statistics (large tier, counts only)
// ---------------------------------------------------------------------------
// A five-vertex central query is a cone over a four-vertex graph H; its count
// at root v is the number of copies of H in the neighbourhood graph
// G_v = G[N(v)] whose universal vertices follow v (NbhdForm). For the forms
// here that number is a sum of per-vertex and per-edge terms of G_v, read off
// the root's bitmap rows: d_u = |row(u)|, E = sum d_u / 2 and, per edge
// (u, w), the common neighbours row(u) & row(w). The walk instead enumerates
// every (x1, x2, x3) prefix: on a hub of degree 10^5 that is ~10^13 prefixes,
// against ~10^8 edge terms here.
//
// k_large_nbdeg: d_u of every row and E of every root of the batch whose plan
// has a form (a warp per row, blocks over 256-row chunks).
__global__ void __launch_bounds__(256) k_large_nbdeg(const PairDev *__restrict__ pairs, Batch bt, uint32_t *arena) {
    const uint32_t total = bt.cstart[bt.nb];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
        const uint32_t b = find_batch(bt.cstart, bt.nb, c);
        const uint64_t it = bt.item[b];
        if (pairs[item_pair(it)].pl.nbhd == kNbNone)
            continue;
        PairRegs pr;
        load_pair(pairs, item_pair(it), pr);
        uint32_t beg, D, j0;
        pair_domain(pr, item_root(it), beg, D, j0);
        const uint32_t W = (D + 31) >> 5;
        uint32_t *base = arena + bt.off[b]; // rows of the whole domain (rlo = 0)
        uint32_t *deg = base + nb_deg_offset(D, 0);
        unsigned long long *E2 = reinterpret_cast<unsigned long long *>(base + nb_edges_offset(D, 0));
        const uint32_t i0 = (c - bt.cstart[b]) * kRowsPerChunk, i1 = min(D, i0 + kRowsPerChunk);
        unsigned long long sum = 0;
        for (uint32_t i = i0 + warp; i < i1; i += nwarps) {
            const uint32_t *row = base + (size_t)i * W;
            uint32_t d = 0;
            for (uint32_t k = lane; k < W; k += 32)
                d += (uint32_t)__popc(row[k]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                d += __shfl_xor_sync(kFull, d, o);
            if (lane == 0) {
                deg[i] = d;
                sum += d;
            }
        }
        if (lane == 0 && sum)
            atomicAdd(E2, sum); // twice the edges: E = E2 / 2
    }
}

// |row(a) & row(b)| over the shorter of a's word list (al, na) and b's own
// list; with above, only the bits after domain index lo.
__device__ __forceinline__ uint32_t common_count(const uint32_t *ra, const uint32_t *rb, const uint32_t *al,
                                                 uint32_t na, const RowLists &rl, uint32_t b, bool above,
                                                 uint32_t lo) {
    const uint32_t nbw = rl.cap ? rl.nzc[b] : 0xffffffffu;
    const bool use_b = nbw <= rl.cap && nbw < na;
    const uint32_t *lst = use_b ? rl.nzl + (size_t)b * rl.cap : al;
    const uint32_t n = use_b ? nbw : na;
    const uint32_t lw = lo >> 5, lmask = ~((2u << (lo & 31)) - 1u); // bits of word lw above lo
    uint32_t s = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t e = lst[i];
        if (above && e < lw)
            continue;
        uint32_t w = ra[e] & rb[e];
        if (above && e == lw)
            w &= lmask;
        s += (uint32_t)__popc(w);
    }
    return s;
}

// Task (root, u): u's terms of the root's form, into plus / minus (lane
// sums). la: W words of per-warp scratch for u's word list when its row has
// none.
__device__ __forceinline__ void nbhd_task(int form, const uint32_t *__restrict__ bm, const RowLists &rl,
                                          const uint32_t *__restrict__ deg, unsigned long long E, uint32_t W,
                                          uint32_t D, uint32_t u, bool first, uint32_t *la, int lane,
                                          unsigned long long &plus, unsigned long long &minus) {
    const unsigned lt = (1u << lane) - 1u;
    const unsigned long long du = deg[u], rest = D >= 3 ? D - 3 : 0;
    if (form == kNbWedgeIso) {
        if (lane == 0)
            plus = sat_add(plus, sat_mul(binom2(du), rest));
        return;
    }
    if (form == kNbTwoEdges) {
        if (lane == 0) {
            if (first) { // C(E, 2), exact through 128 bits
                const unsigned __int128 c2 = ((unsigned __int128)E * (E - (E ? 1 : 0))) / 2;
                plus = sat_add(plus, c2 >= (unsigned __int128)kCountLimit ? kCountLimit : (unsigned long long)c2);
            }
            minus = sat_add(minus, binom2(du));
        }
        return;
    }
    // the other forms sum over the edges (u, w): w after u, or every w (paw)
    const bool all_w = form == kNbPaw;
    const uint32_t *ru = bm + (size_t)u * W;
    const uint32_t uw = u >> 5;
    const uint32_t *al = la;
    uint32_t na = 0;
    if (rl.cap && rl.nzc[u] <= rl.cap) {
        al = rl.nzl + (size_t)u * rl.cap;
        na = rl.nzc[u];
    } else {
        for (uint32_t k0 = 0; k0 < W; k0 += 32) {
            const uint32_t k = k0 + (uint32_t)lane;
            const uint32_t w = k < W ? ru[k] : 0u;
            const unsigned bal = __ballot_sync(kFull, w != 0);
            if (w)
                la[na + (uint32_t)__popc(bal & lt)] = k;
            na += (uint32_t)__popc(bal);
        }
        __syncwarp();
    }
    unsigned long long tri = 0; // paw: triangles at u (lane part)
    for (uint32_t t0 = 0; t0 < na; t0 += 32) {
        uint32_t bits = 0, k = 0;
        if (t0 + (uint32_t)lane < na) {
            k = al[t0 + lane];
            bits = ru[k];
            if (!all_w)
                bits = k < uw ? 0u : (k == uw ? (bits & ~((2u << (u & 31)) - 1u)) : bits);
        }
        while (bits) {
            const uint32_t w = (k << 5) + (uint32_t)(__ffs(bits) - 1);
            bits &= bits - 1;
            const uint32_t *rw = bm + (size_t)w * W;
            switch (form) {
            case kNbTriIso: // triangles (u < w < x) once, times the isolated vertex's choices
                plus = sat_add(plus, sat_mul(common_count(ru, rw, al, na, rl, w, true, w), rest));
                break;
            case kNbPath4: // paths x - u - w - y, minus the closed ones (x = y): 3T
                plus = sat_add(plus, (du - 1) * ((unsigned long long)deg[w] - 1));
                minus = sat_add(minus, common_count(ru, rw, al, na, rl, w, false, 0));
                break;
            case kNbPaw: // triangles (u, w, x) with x after w: each once
                tri += common_count(ru, rw, al, na, rl, w, true, w);
                break;
            case kNbDiamond: { // C(common neighbours, 2) of the edge (u, w)
                const unsigned long long c = common_count(ru, rw, al, na, rl, w, false, 0);
                plus = sat_add(plus, binom2(c));
                break;
            }
            default:
                break;
            }
        }
    }
    if (form == kNbPaw) {
        tri = warp_sum(tri);
        if (lane == 0 && du >= 2)
            plus = sat_add(plus, sat_mul(tri, du - 2));
    }
    __syncwarp(); // la reused by the warp's next task
}

// The large tier's roots of neighbourhood-statistics plans (depth slot
// kNbhdSlot): every warp takes (root, u) tasks from the cursor. The task of
// the root's first domain vertex also adds the root-level term.
__global__ void __launch_bounds__(256) k_large_nbhd(const PairDev *__restrict__ pairs, Batch bt,
                                                    const uint32_t *arena, unsigned *cursor, uint32_t *wsc,
                                                    uint32_t wstride, unsigned long long *exit_t) {
    const int lane = threadIdx.x & 31;
    const uint32_t base0 = bt.tstart[0];
    const uint32_t total = bt.tstart[bt.nb] - base0;
    // the warp's scratch is shared with k_large_wheel, which needs its first
    // and fourth regions of wstride / 4 words (U and U2, for roots of any
    // width) zero on entry: this kernel writes only the third region, words
    // [2 Wm, 3 Wm)
    const uint32_t Wm = wstride / 4;
    uint32_t *ws = wsc + (size_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * wstride;
    PairRegs pr;
    uint32_t cur = 0xffffffffu;
    int form = kNbNone;
    unsigned long long plus = 0, minus = 0;
    for (;;) {
        uint32_t t = 0;
        if (lane == 0)
            t = atomicAdd(cursor, 1u);
        t = __shfl_sync(kFull, t, 0);
        if (t >= total)
            break;
        t += base0;
        const uint32_t b = find_batch(bt.tstart, bt.nb, t);
        const uint64_t it = bt.item[b];
        const uint32_t p = item_pair(it), r = item_root(it);
        if (p != cur) {
            plus = warp_sum(plus);
            minus = warp_sum(minus);
            if (lane == 0) {
                flush_count(pr.count + 2, plus);
                flush_count(pr.count + 4, minus);
            }
            plus = minus = 0;
            cur = p;
            load_pair(pairs, p, pr);
            form = pairs[p].pl.nbhd;
        }
        uint32_t beg, D, j0;
        pair_domain(pr, r, beg, D, j0);
        const uint32_t W = (D + 31) >> 5;
        const uint32_t *rows = arena + bt.off[b]; // rows of the whole domain: rlo == 0
        RowLists rl;
        rl.cap = list_cap(W);
        rl.nzc = rows + (size_t)D * W;
        rl.nzl = rl.nzc + D;
        const uint32_t *deg = rows + nb_deg_offset(D, 0);
        const unsigned long long E = *reinterpret_cast<const unsigned long long *>(rows + nb_edges_offset(D, 0)) / 2;
        const uint32_t u = j0 + (t - bt.tstart[b]);
        nbhd_task(form, rows, rl, deg, E, W, D, u, t == bt.tstart[b], ws + 2 * (size_t)Wm, lane, plus, minus);
    }
    plus = warp_sum(plus);
    minus = warp_sum(minus);
    if (lane == 0) {
        flush_count(pr.count + 2, plus);
        flush_count(pr.count + 4, minus);
        record_exit(exit_t);
    }
}

// ---------------------------------------------------------------------------
// queries without a central vertex: list walker. The neighbourhood bitmaps
// above need every position adjacent to the root; here a thread takes one
// (root, level-1 vertex) task and walks the rest of the matching order over
// the view's sorted neighbour lists: a position's candidates are the entries
// of the shortest list among its back-edge positions (the root included)
// that lie in every other such list, are not used yet and follow every
// position the symmetry chain puts before it. Counts full matches (sgm).
// ---------------------------------------------------------------------------
struct GenRegs {
    ViewDev v;
    uint32_t back[kMaxQ]; // bits q >= 1
    uint32_t sym[kMaxQ];  // bits s >= 1
    uint32_t adj0, sym0;  // bit p: position p adjacent to / after position 0
    int32_t order[kMaxQ];
    int32_t K;
    EnumDev en;
};

__device__ __forceinline__ void load_gen(const PairDev &pd, GenRegs &g) {
    g.v = pd.v;
#pragma unroll
    for (int i = 0; i < kMaxQ; ++i) {
        g.back[i] = pd.pl.back[i];
        g.sym[i] = pd.pl.sym[i];
        g.order[i] = pd.pl.order[i];
    }
    g.adj0 = pd.pl.adj0;
    g.sym0 = pd.pl.sym0;
    g.K = pd.pl.K;
    g.en = pd.en;
}

// one tuple, in query-vertex order and input ids
__device__ __forceinline__ void gen_emit(const GenRegs &g, const uint32_t (&x)[kMaxQ], int P, uint32_t w) {
    if (g.en.out == nullptr || *(volatile unsigned long long *)g.en.n >= g.en.k)
        return;
    const unsigned long long slot = atomicAdd(g.en.n, 1ull);
    if (slot >= g.en.k)
        return;
    int32_t *t = g.en.out + slot * (unsigned long long)g.K;
    for (int q = 0; q < P; ++q)
        t[g.order[q]] = (int32_t)g.v.orig[x[q]];
    t[g.order[P]] = (int32_t)g.v.orig[w];
}

template <int P, int DEND, bool ENUM>
__device__ void gen_walk(const GenRegs &g, uint32_t (&x)[kMaxQ], unsigned long long &cnt) {
    if constexpr (P >= DEND) {
        return;
    } else {
        const uint32_t bset = g.back[P] | ((g.adj0 >> P) & 1u); // bit 0: the root
        uint32_t lo = 0;
#pragma unroll
        for (int q = 1; q < P; ++q)
            if (g.sym[P] >> q & 1u)
                lo = max(lo, x[q] + 1);
        if (g.sym0 >> P & 1u)
            lo = max(lo, x[0] + 1);
        int qd = 0;
        uint32_t db = 0, de = 0, best = 0xffffffffu;
#pragma unroll
        for (int q = 0; q < P; ++q)
            if (bset >> q & 1u) {
                const uint32_t b = g.v.rp[x[q]], e = g.v.rp[x[q] + 1];
                if (e - b < best) {
                    best = e - b;
                    qd = q;
                    db = b;
                    de = e;
                }
            }
        for (uint32_t k = lower_bound_g(g.v.col, db, de, lo); k < de; ++k) {
            if constexpr (ENUM) {
                if (g.en.out && *(const volatile unsigned long long *)g.en.n >= g.en.k)
                    return;
            }
            const uint32_t w = g.v.col[k];
            bool ok = true;
#pragma unroll
            for (int q = 0; q < P; ++q)
                ok = ok && x[q] != w;
#pragma unroll
            for (int q = 0; q < P; ++q)
                if (ok && q != qd && (bset >> q & 1u))
                    ok = contains_g(g.v.col, g.v.rp[x[q]], g.v.rp[x[q] + 1], w);
            if (!ok)
                continue;
            if constexpr (P == DEND - 1) {
                if constexpr (ENUM)
                    gen_emit(g, x, P, w);
                ++cnt;
            } else {
                x[P] = w;
                gen_walk<P + 1, DEND, ENUM>(g, x, cnt);
            }
        }
    }
}

// Items of one depth; tstart[i] - tstart[0] = first task of item i
// (tstart[n] - tstart[0] tasks in all). Warps take 32 tasks at a time.
template <int DEND, bool ENUM>
__global__ void __launch_bounds__(256) k_general(const PairDev *__restrict__ pairs, const uint64_t *__restrict__ items,
                                                 const uint32_t *__restrict__ tstart, uint32_t nitems,
                                                 unsigned *cursor) {
    const int lane = threadIdx.x & 31;
    const uint32_t base0 = tstart[0], total = tstart[nitems] - base0;
    GenRegs g;
    uint32_t cur = 0xffffffffu;
    unsigned long long cnt = 0, *count_ptr = nullptr;
    for (;;) {
        uint32_t t0 = 0;
        if (lane == 0)
            t0 = atomicAdd(cursor, 32u);
        t0 = __shfl_sync(kFull, t0, 0);
        if (t0 >= total)
            break;
        const uint32_t t = t0 + (uint32_t)lane;
        if (t >= total)
            continue;
        const uint32_t b = find_batch(tstart, nitems, t + base0);
        const uint64_t it = items[b];
        const uint32_t p = item_pair(it), r = item_root(it);
        if (p != cur) {
            flush_count(count_ptr, cnt);
            cnt = 0;
            cur = p;
            load_gen(pairs[p], g);
            count_ptr = pairs[p].count;
        }
        const uint32_t j0 = (g.sym0 >> 1 & 1u) ? g.v.split[r] : 0u;
        uint32_t x[kMaxQ];
        x[0] = r;
        x[1] = g.v.col[g.v.rp[r] + j0 + (t + base0 - tstart[b])];
        gen_walk<2, DEND, ENUM>(g, x, cnt);
    }
    if (count_ptr)
        flush_count(count_ptr, cnt);
}

// task counts (D - j0) of listed items
__global__ void k_gen_tasks(const uint32_t *__restrict__ D, const uint32_t *__restrict__ j0, uint32_t n,
                            uint32_t *tasks) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        tasks[i] = D[i] - j0[i];
}

// ---------------------------------------------------------------------------
// root classification over the vertices of every pair (flattened index)
// ---------------------------------------------------------------------------
constexpr int kTiers = 5;   // 1 small (D <= 64), 2 medium (<= 256), 3 medium (<= 1024), 4 large,
                            // 5 list walker (queries without a central vertex)
constexpr int kDepths = kDepthsConst;
constexpr int kSlots = 2 * kDepths; // depth slots: counting pairs, then enumerating pairs

__device__ __forceinline__ uint32_t find_pair(const uint64_t *__restrict__ offs, uint32_t npairs, uint64_t t) {
    uint32_t lo = 0, hi = npairs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (offs[mid] <= t)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// tier[t] for flattened vertex t; dom[t] = its domain size; per tier the
// largest domain and per (tier, depth) the number of roots.
__global__ void k_classify(const PairDev *__restrict__ pairs, const uint64_t *__restrict__ offs, uint32_t npairs,
                           uint64_t N, TierCfg cfg, uint8_t *tier, uint32_t *dom, unsigned *tier_max,
                           unsigned *tier_depth, unsigned *tiny_depth, unsigned long long *large_words) {
    __shared__ unsigned s_hist[kTiers * kSlots];
    __shared__ unsigned s_tiny[kSlots];
    for (int i = threadIdx.x; i < kTiers * kSlots; i += blockDim.x)
        s_hist[i] = 0;
    for (int i = threadIdx.x; i < kSlots; i += blockDim.x)
        s_tiny[i] = 0;
    __syncthreads();
    uint32_t mx[kTiers] = {0, 0, 0, 0, 0};
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = find_pair(offs, npairs, t);
        const uint32_t r = (uint32_t)(t - offs[p]);
        const PairDev &pd = pairs[p];
        const uint32_t deg = pd.v.rp[r + 1] - pd.v.rp[r];
        const uint32_t sp = pd.v.split[r];
        uint32_t D, j0;
        if (pd.pl.restricted) {
            D = deg - sp;
            j0 = 0;
        } else {
            D = deg;
            j0 = pd.pl.pos1_after_root ? sp : 0;
        }
        uint8_t tc = 0;
        // roots: degree in [max_qdeg, cap) (subgraph_matching.cuh:1086-1098),
        // enough domain vertices for the other dend-1 positions and at least
        // one level-1 vertex
        const bool root_ok = deg >= pd.min_deg && deg < pd.cap_deg && j0 < D &&
                             (pd.shard_mod <= 1 || pd.v.orig[r] % pd.shard_mod == pd.shard_rem);
        if (!pd.pl.central) {
            if (root_ok) {
                tc = 5;
                D -= j0; // level-1 tasks of the list walker
            }
        } else if (root_ok && D + 1 >= (uint32_t)pd.pl.dend) {
            tc = D <= cfg.small_max ? 1 : (D <= cfg.med_a_max ? 2 : (D <= cfg.med_max ? 3 : 4));
        }
        tier[t] = tc;
        dom[t] = D;
        if (tc == 4) {
            const uint32_t rn = pd.pl.rows_needed, rlo = rn == 2 ? 0u : (rn == 1 ? j0 : D);
            atomicAdd(large_words, (unsigned long long)large_root_words(D, rlo, pd.pl.nbhd != kNbNone));
        }
        if (tc) {
            mx[tc - 1] = max(mx[tc - 1], D);
            const uint32_t slot = depth_slot(pd.pl, tc, pd.en.out != nullptr);
            atomicAdd(&s_hist[(tc - 1) * kSlots + slot], 1u);
            if (tc == 1 && D <= cfg.tiny_max)
                atomicAdd(&s_tiny[slot], 1u);
        }
    }
#pragma unroll
    for (int k = 0; k < kTiers; ++k) {
        const uint32_t m = __reduce_max_sync(kFull, mx[k]);
        if ((threadIdx.x & 31) == 0 && m)
            atomicMax(&tier_max[k], m);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kTiers * kSlots; i += blockDim.x)
        if (s_hist[i])
            atomicAdd(&tier_depth[i], s_hist[i]);
    for (int i = threadIdx.x; i < kSlots; i += blockDim.x)
        if (s_tiny[i])
            atomicAdd(&tiny_depth[i], s_tiny[i]);
}

// Sort keys of every flattened vertex for all item lists at once:
// (tier, depth slot, domain order) -- small roots by domain ascending, medium and
// large ones by domain descending (heaviest first), list-walker roots by
// depth only; non-roots last.
__global__ void k_list_keys(const uint8_t *__restrict__ tier, const uint32_t *__restrict__ dom,
                            const PairDev *__restrict__ pairs, const uint64_t *__restrict__ offs, uint32_t npairs,
                            uint64_t N, uint32_t *keys, uint32_t *vals) {
    constexpr uint32_t kDomMask = (1u << 24) - 1u;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t tc = tier[t];
        uint32_t key = 0xffffffffu;
        if (tc) {
            const uint32_t p = find_pair(offs, npairs, t);
            const uint32_t slot = depth_slot(pairs[p].pl, tc, pairs[p].en.out != nullptr);
            const uint32_t d = min(dom[t], kDomMask);
            const uint32_t dk = tc == 1 ? d : (tc == 5 ? 0u : kDomMask - d);
            key = ((tc - 1) << 29) | (slot << 24) | dk;
        }
        keys[t] = key;
        vals[t] = (uint32_t)t;
    }
}

// Sorted flattened indices of the roots -> items (pair << 32 | root).
__global__ void k_make_items(const uint32_t *__restrict__ sorted, uint32_t n, const uint64_t *__restrict__ offs,
                             uint32_t npairs, uint64_t *items) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t t = sorted[i];
        const uint32_t p = find_pair(offs, npairs, t);
        items[i] = ((uint64_t)p << 32) | (uint64_t)(t - offs[p]);
    }
}

// Arena words, row chunks and level-1 tasks of each listed large root
// (D, j0 from k_gather_dom).
__global__ void k_large_meta(const PairDev *__restrict__ pairs, const uint64_t *__restrict__ items, uint32_t nl,
                             const uint32_t *__restrict__ D_in, const uint32_t *__restrict__ j0_in,
                             unsigned long long *words, uint32_t *chunks, uint32_t *tasks) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += gridDim.x * blockDim.x) {
        const uint32_t D = D_in[i], j0 = j0_in[i];
        const DevPlan &pl = pairs[item_pair(items[i])].pl;
        const uint32_t rn = (uint32_t)pl.rows_needed;
        const uint32_t rlo = rn == 2 ? 0u : (rn == 1 ? j0 : D);
        words[i] = large_root_words(D, rlo, pl.nbhd != kNbNone);
        chunks[i] = (D + kRowsPerChunk - 1) / kRowsPerChunk;
        tasks[i] = D - j0;
    }
}

// (D, j0) of each listed item.
__global__ void k_gather_dom(const PairDev *__restrict__ pairs, const uint64_t *__restrict__ items, uint32_t nl,
                             uint32_t *D_out, uint32_t *j0_out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += gridDim.x * blockDim.x) {
        PairRegs pr;
        load_pair(pairs, item_pair(items[i]), pr);
        uint32_t beg, D, j0;
        pair_domain(pr, item_root(items[i]), beg, D, j0);
        D_out[i] = D;
        j0_out[i] = j0;
    }
}

// Adjacency bytes of the searched roots: row pointers and split of the root
// (12 B), its domain list (4 B each) and, per domain vertex, its row pointers
// and split (12 B) plus its higher-priority list (4 B each).
__global__ void k_alg_bytes(const PairDev *__restrict__ pairs, const uint64_t *__restrict__ offs, uint32_t npairs,
                            const uint8_t *__restrict__ tier, uint64_t N, unsigned long long *bytes) {
    unsigned long long acc[3] = {0, 0, 0}, alg[3] = {0, 0, 0};
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < N; t += warps) {
        const int tc = tier[t];
        if (!tc || tc == 5) // the list walker has no bitmap tier
            continue;
        const uint32_t p = find_pair(offs, npairs, t);
        PairRegs pr;
        load_pair(pairs, p, pr);
        uint32_t beg, D, j0;
        pair_domain(pr, (uint32_t)(t - offs[p]), beg, D, j0);
        unsigned long long a = (lane == 0) ? 12ull + 4ull * D : 0ull;
        for (uint32_t i = lane; i < D; i += 32) {
            uint32_t hb, he, xb, xe;
            hd_range(pr.v, pr.asc, pr.v.col[beg + i], i, D, hb, he, xb, xe);
            a += 12ull + 4ull * (he - hb);
        }
        // algorithmic bytes of building this root's neighbourhood bitmap from
        // the input CSR: its list and each neighbour's full list, 4 bytes an
        // entry, 4 * (deg r + sum over v in N(r) of deg v)
        const uint32_t *grp = pairs[p].g_rp, *gcol = pairs[p].g_col;
        const uint32_t u = pr.v.orig[(uint32_t)(t - offs[p])];
        const uint32_t ub = grp[u], ue = grp[u + 1];
        unsigned long long b = (lane == 0) ? 4ull * (ue - ub) : 0ull;
        for (uint32_t k = ub + lane; k < ue; k += 32) {
            const uint32_t w = gcol[k];
            b += 4ull * (grp[w + 1] - grp[w]);
        }
        const int slot = tc == 1 ? 0 : (tc == 4 ? 2 : 1);
        acc[slot] += a;
        alg[slot] += b;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const unsigned long long x = warp_sum(acc[k]), y = warp_sum(alg[k]);
        if (lane == 0 && x)
            atomicAdd(&bytes[k], x);
        if (lane == 0 && y)
            atomicAdd(&bytes[3 + k], y);
    }
}


// ---------------------------------------------------------------------------
// launch helpers (one instantiation per depth)
// ---------------------------------------------------------------------------
#define BEEP_DEPTH_SWITCH(dend, CASE)                                                                              \
    switch (dend) {                                                                                                \
        CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9) CASE(10) default                                   \
            : return fail(BEEP_ERR_UNSUPPORTED, "depth out of range");                                             \
    }

template <bool ENUM>
beep_status launch_small(int dend, int group, int grid, cudaStream_t s, const PairDev *pairs, const uint64_t *items,
                         uint32_t n, unsigned long long *exit_t) {
#define BEEP_CASE(D)                                                                                               \
    case D:                                                                                                        \
        if (group == 8)                                                                                            \
            k_small<D, ENUM, 8, kTinyMaxD><<<grid, kSmallWarps * 32, 0, s>>>(pairs, items, n, exit_t);              \
        else                                                                                                       \
            k_small<D, ENUM, 32, kSmallMaxD><<<grid, kSmallWarps * 32, 0, s>>>(pairs, items, n, exit_t);            \
        break;
    BEEP_DEPTH_SWITCH(dend, BEEP_CASE)
#undef BEEP_CASE
    BEEP_CUDA_TRY(cudaGetLastError());
    return BEEP_OK;
}

template <bool ENUM>
beep_status launch_general(int dend, int grid, cudaStream_t s, const PairDev *pairs, const uint64_t *items,
                           const uint32_t *tstart, uint32_t n, unsigned *cursor) {
#define BEEP_CASE(D)                                                                                               \
    case D:                                                                                                        \
        k_general<D, ENUM><<<grid, 256, 0, s>>>(pairs, items, tstart, n, cursor);                                   \
        break;
    BEEP_DEPTH_SWITCH(dend, BEEP_CASE)
#undef BEEP_CASE
    BEEP_CUDA_TRY(cudaGetLastError());
    return BEEP_OK;
}

// Raises a kernel's dynamic shared memory limit on the current device, never
// lowers it. A plan sets the limits its launches need when it is made and
// replays them later (eagerly or from a captured CUDA graph); a plan made in
// between for smaller domains must not leave an earlier plan's launches above
// the limit (they would fail with an invalid argument).
beep_status raise_smem_limit(const void *fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> limits;
    int dev = 0;
    BEEP_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    size_t &cur = limits[{dev, fn}];
    if (bytes <= cur)
        return BEEP_OK;
    BEEP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
    return BEEP_OK;
}

template <int D, bool ENUM> beep_status set_medium_attr(size_t smem) {
    BEEP_TRY(raise_smem_limit((const void *)k_medium<D, ENUM, 0>, smem));
    BEEP_TRY(raise_smem_limit((const void *)k_medium<D, ENUM, 32>, smem));
    return BEEP_OK;
}

template <bool ENUM>
beep_status launch_large_dfs(int dend, int grid, cudaStream_t s, const PairDev *pairs, const Batch &bt,
                             const uint32_t *arena, unsigned *cursor, const Don &dn, unsigned long long *exit_t) {
#define BEEP_CASE(D)                                                                                               \
    case D:                                                                                                        \
        k_large_dfs<D, ENUM><<<grid, 256, 0, s>>>(pairs, bt, arena, cursor, dn, exit_t);                            \
        break;
    BEEP_DEPTH_SWITCH(dend, BEEP_CASE)
#undef BEEP_CASE
    BEEP_CUDA_TRY(cudaGetLastError());
    return BEEP_OK;
}

// Blocks of k_large_dfs that are resident on one SM at once (the persistent
// grid is that many per SM).
template <bool ENUM> beep_status large_dfs_blocks_per_sm(int dend, int *out) {
    int nb = 1;
#define BEEP_CASE(D)                                                                                               \
    case D:                                                                                                        \
        BEEP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_large_dfs<D, ENUM>, 256, 0));           \
        break;
    BEEP_DEPTH_SWITCH(dend, BEEP_CASE)
#undef BEEP_CASE
    *out = std::max(nb, 1);
    return BEEP_OK;
}


} // namespace

// ---------------------------------------------------------------------------
// Plan and execution of a multi-pair call.
//
// plan_pairs does everything that needs the host: views, root classification
// (one read-back of the tier sizes), sorted item lists and the batching of
// large roots into arena-sized groups. It leaves a list of launches whose
// buffers it owns. execute_plan replays that list as a stream-ordered
// sequence of memsets and kernels with no host synchronisation, so it can be
// captured once into a CUDA graph (capture_plan) and relaunched.
// ---------------------------------------------------------------------------
struct LaunchRec {
    enum Kind { kSmall, kMedium, kLargeRows, kLargeLists, kLargeDfs, kLargeWheel, kGeneral, kMemset, kLargeNbDeg,
                kLargeNbhd } kind;
    const uint32_t *tstart = nullptr; // list walker: task prefix of the items
    int dend = 0, grid = 0, block = 0;
    int group = 32; // small tier: lanes per root
    size_t smem = 0;
    const uint64_t *items = nullptr;
    uint32_t n = 0, maxD = 0;
    unsigned *cursor = nullptr;
    Batch bt{};
    void *mptr = nullptr;
    size_t mbytes = 0;
    double *sink = nullptr;   // stats field this launch's time adds to
    uint32_t *wsc = nullptr;  // large tier: 4-wheel scratch, wstride words a warp
    uint32_t wstride = 0;
    bool enumerate = false;   // the launch writes tuples (its pairs' walks have no closed forms)
    Don don{};                // large-tier walks: the donation queue (cap 0: none)
    int tail_slot = -1;       // stats tail this launch's exit spread counts to (0 small, 1 medium, 2 large)
};

// The degree pass of the neighbourhood-statistics roots a kLargeRows record builds.
static LaunchRec nbdeg_rec(const LaunchRec &rows) {
    LaunchRec r = rows;
    r.kind = LaunchRec::kLargeNbDeg;
    r.block = 256;
    r.smem = 0;
    r.grid = rows.grid * 4;
    r.cursor = nullptr;
    return r;
}

// The list pass over the rows a kLargeRows record builds.
static LaunchRec lists_rec(const LaunchRec &rows) {
    LaunchRec r = rows;
    r.kind = LaunchRec::kLargeLists;
    r.block = 256;
    r.smem = 0;
    r.grid = rows.grid * 4;
    r.cursor = nullptr;
    return r;
}

struct LaunchPlan {
    Ctx *ctx = nullptr;
    std::vector<std::shared_ptr<View>> views; // kept alive while the plan exists
    std::vector<void *> allocs;
    std::vector<uint32_t> live; // spec index of each device pair
    uint32_t np = 0;
    PairDev *d_pairs = nullptr;
    uint64_t *d_offs = nullptr;
    uint8_t *d_tier = nullptr;
    uint64_t N = 0;
    // per pair (count, overflow flag), then np tuple counters, then kAux byte counters
    unsigned long long *d_counts = nullptr;
    // work cursors, one per launch that takes items from a counter: blocks
    // of kCursorBlock, all zeroed at the start of every run
    std::vector<unsigned *> cursor_blocks;
    uint32_t ncursors = 0;
    // pinned mirror of the (count, flag) words and the byte counters (2 np + kAux):
    // the context's buffer, or owned when captured
    unsigned long long *h_counts = nullptr;
    bool own_h_counts = false;
    std::vector<LaunchRec> recs;
    bool enumerate = false;
    // donation queue of the large tier (shared by its walk launches, which run
    // one after another on one stream) and one control block per walk launch
    DonTask *d_don_tasks = nullptr;
    unsigned *d_don_ready = nullptr;
    uint32_t don_cap = 0;
    unsigned *d_don_ctl = nullptr; // kDonWords per walk launch
    uint32_t ndon = 0;
    // earliest and latest warp exit of every launch (with BEEP_OPT_TIMING)
    unsigned long long *d_exit = nullptr;
    uint32_t nexit = 0;
    // host words after the pair counts and byte counters: donation control
    // blocks (as u32), then exit times
    size_t tel_words() const { return (size_t)ndon * kDonWords / 2 + 2 * (size_t)nexit; }
    size_t host_words() const { return kPairWords * (size_t)np + kAux + tel_words(); }
    beep_stats st{};
    cudaGraphExec_t exec = nullptr;
    ~LaunchPlan() {
        if (exec)
            cudaGraphExecDestroy(exec);
        for (void *p : allocs)
            cudaFreeAsync(p, ctx->stream);
        if (h_counts && own_h_counts)
            cudaFreeHost(h_counts);
    }
    template <typename T> beep_status alloc(T *&out, size_t count) {
        void *p = nullptr;
        const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
        cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, ctx->pool, ctx->stream);
        if (e != cudaSuccess)
            return fail(e == cudaErrorMemoryAllocation ? BEEP_ERR_OUT_OF_MEMORY : BEEP_ERR_CUDA,
                        std::string("device pool allocation of ") + std::to_string(bytes) + " bytes: " +
                            cudaGetErrorString(e));
        allocs.push_back(p);
        out = static_cast<T *>(p);
        return BEEP_OK;
    }
};

void LaunchPlanDeleter::operator()(LaunchPlan *p) const { delete p; }

// Pair i's count after the read-back: the walks' count plus the
// neighbourhood statistics' sums; BEEP_COUNT_OVERFLOW when a flag is set or
// the total reaches the limit.
static uint64_t pair_result(const LaunchPlan *lp, uint32_t i) {
    const unsigned long long *c = lp->h_counts + kPairWords * (size_t)i;
    if (c[1] || c[3] || c[5] || c[2] < c[4])
        return BEEP_COUNT_OVERFLOW;
    const uint64_t st = c[2] - c[4], v = c[0] + st;
    return (v < c[0] || v >= BEEP_COUNT_LIMIT) ? BEEP_COUNT_OVERFLOW : v;
}

beep_status plan_pairs(Ctx *ctx, const std::vector<PairSpec> &specs, uint32_t options, LaunchPlanPtr *out,
                       const TierCfg &tiers) {
    cudaStream_t s = ctx->stream;
    PhaseTrace tr("plan", s);
    LaunchPlanPtr lp(new LaunchPlan);
    lp->ctx = ctx;
    beep_stats &st = lp->st;
    std::memset(&st, 0, sizeof(st));
    if (!specs.empty()) {
        st.cutoff = specs[0].g->cutoff;
        st.ascending = specs[0].plan.dev.asc;
    }
    // views (peel + priority relabelling, cached per graph)
    std::vector<PairDev> hp;
    std::vector<uint64_t> offs{0};
    std::vector<Graph *> dropped;
    for (size_t i = 0; i < specs.size(); ++i) {
        const PairSpec &ps = specs[i];
        if (ps.g->n == 0 || ps.plan.dev.dend < 3)
            continue; // K - LUNMAT < 3: the reference's main path never reaches a counting level
        if ((options & BEEP_OPT_NO_VIEW_CACHE) && std::find(dropped.begin(), dropped.end(), ps.g) == dropped.end()) {
            ps.g->views.clear();
            dropped.push_back(ps.g);
        }
        std::shared_ptr<View> v;
        bool built = false;
        BEEP_TRY(get_view(ctx, ps.g, ps.plan.info.min_qdeg, ps.plan.dev.asc, false, &v, &built));
        lp->views.push_back(v);
        st.peel_rounds = v->peel_rounds; // view-build launches are counted where they happen
        if (v->n == 0)
            continue;
        PairDev pd;
        std::memset(&pd, 0, sizeof(pd));
        pd.v = ViewDev{v->row_ptr.as<uint32_t>(), v->col.as<uint32_t>(), v->split.as<uint32_t>(),
                       v->orig.as<uint32_t>()};
        pd.g_rp = ps.g->row_ptr.as<uint32_t>();
        pd.g_col = ps.g->col.as<uint32_t>();
        pd.pl = ps.plan.dev;
        pd.min_deg = (uint32_t)ps.plan.info.max_qdeg;
        pd.cap_deg = (options & BEEP_OPT_REFERENCE_ROOT_CAP)
                         ? (uint32_t)std::min<uint64_t>(0xffffffffull, (uint64_t)ps.g->cutoff * 100ull)
                         : 0xffffffffu;
        pd.shard_mod = ps.nshards;
        pd.shard_rem = ps.shard;
        if (ps.en && ps.en->k > 0 && ps.en->d_out) {
            lp->enumerate = true;
            pd.en.out = ps.en->d_out;
            pd.en.k = ps.en->k;
        }
        hp.push_back(pd);
        lp->live.push_back((uint32_t)i);
        offs.push_back(offs.back() + (uint64_t)v->n);
    }
    const uint32_t np = (uint32_t)hp.size();
    lp->np = np;
    tr.mark("views");
    BEEP_TRY(lp->alloc(lp->d_counts, (kPairWords + 1) * (size_t)np + kAux));
    if (np == 0) {
        BEEP_TRY(ctx->host_results(lp->host_words(), &lp->h_counts));
        *out = std::move(lp);
        return BEEP_OK;
    }
    const uint64_t N = offs.back();
    if (N >= 0xffffffffull)
        return fail(BEEP_ERR_UNSUPPORTED, "more than 2^32 vertices in one call");
    lp->N = N;
    for (uint32_t i = 0; i < np; ++i) {
        hp[i].count = lp->d_counts + kPairWords * (size_t)i;
        hp[i].en.n = lp->d_counts + kPairWords * (size_t)np + i; // every pair has a tuple counter (k = 0: none written)
        if (hp[i].en.out) { // the closed forms count; enumeration walks the matches
            hp[i].pl.wheel4 = 0;
            hp[i].pl.nbhd = kNbNone;
        }
        if (options & BEEP_OPT_NO_NBHD)
            hp[i].pl.nbhd = kNbNone;
    }
    BEEP_TRY(lp->alloc(lp->d_pairs, np));
    BEEP_TRY(lp->alloc(lp->d_offs, np + 1));
    BEEP_TRY(lp->alloc(lp->d_tier, N));
    uint32_t *d_dom, *d_sel, *d_keys, *d_keys2;
    unsigned *d_misc;
    BEEP_TRY(lp->alloc(d_dom, N));
    BEEP_TRY(lp->alloc(d_sel, N));
    BEEP_TRY(lp->alloc(d_keys, N));
    BEEP_TRY(lp->alloc(d_keys2, N));
    BEEP_TRY(lp->alloc(d_misc, 256));
    BEEP_CUDA_TRY(cudaMemcpyAsync(lp->d_pairs, hp.data(), np * sizeof(PairDev), cudaMemcpyHostToDevice, s));
    BEEP_CUDA_TRY(cudaMemcpyAsync(lp->d_offs, offs.data(), (np + 1) * 8, cudaMemcpyHostToDevice, s));
    BEEP_CUDA_TRY(cudaMemsetAsync(d_misc, 0, 256 * 4, s));
    const int gv = std::max(1, (int)std::min<uint64_t>((N + 255) / 256, (uint64_t)ctx->num_sms * 32));
    // d_misc: [0, 8) largest domain per tier, [8, 8 + kTiers * kSlots) roots
    // per (tier, depth slot), [120, 120 + kSlots) tiny small-tier roots per
    // slot, [144, 146) arena words of the large tier (u64)
    constexpr int kMiscSlots = 8, kMiscTiny = 120, kMiscLarge = 144;
    static_assert(kMiscSlots + kTiers * kSlots <= kMiscTiny && kMiscTiny + kSlots <= kMiscLarge, "d_misc layout");
    TierCfg cfg = tiers;
    cfg.tiny_max = std::min<uint32_t>(cfg.tiny_max, kTinyMaxD);
    cfg.small_max = std::min<uint32_t>(cfg.small_max, kSmallMaxD);
    cfg.med_a_max = std::min<uint32_t>(cfg.med_a_max, kMediumAMaxD);
    cfg.med_max = std::min<uint32_t>(cfg.med_max, kMediumMaxD);
    k_classify<<<gv, 256, 0, s>>>(lp->d_pairs, lp->d_offs, np, N, cfg, lp->d_tier, d_dom, d_misc,
                                  d_misc + kMiscSlots, d_misc + kMiscTiny,
                                  reinterpret_cast<unsigned long long *>(d_misc + kMiscLarge));
    BEEP_CUDA_TRY(cudaGetLastError());
    st.kernel_launches += 1;
    unsigned h_misc[kMiscLarge + 2];
    BEEP_CUDA_TRY(cudaMemcpyAsync(h_misc, d_misc, sizeof(h_misc), cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    const unsigned *tier_max = h_misc;
    const unsigned *tier_depth = h_misc + kMiscSlots; // [tier * kSlots + slot]
    const unsigned *tiny_depth = h_misc + kMiscTiny;  // [slot]
    uint64_t large_words = 0;
    std::memcpy(&large_words, h_misc + kMiscLarge, 8);
    uint32_t tier_n[kTiers];
    for (int k = 0; k < kTiers; ++k) {
        tier_n[k] = 0;
        for (int d = 0; d < kSlots; ++d)
            tier_n[k] += tier_depth[k * kSlots + d];
    }
    st.roots_small = tier_n[0];
    st.roots_medium = (int64_t)tier_n[1] + tier_n[2];
    st.roots_large = tier_n[3];
    st.roots_general = tier_n[4];
    st.roots = st.roots_small + st.roots_medium + st.roots_large + st.roots_general;
    tr.mark("classify");
    // a fresh zeroed work counter for every launch (a shared one would make a
    // later launch start past its first items and skip them)
    auto cursor = [&](unsigned *&out) -> beep_status {
        if (lp->ncursors % kCursorBlock == 0) {
            unsigned *blk = nullptr;
            BEEP_TRY(lp->alloc(blk, kCursorBlock));
            lp->cursor_blocks.push_back(blk);
        }
        const uint32_t i = lp->ncursors++;
        out = lp->cursor_blocks[i / kCursorBlock] + i % kCursorBlock;
        return BEEP_OK;
    };
    // a walk launch of the large tier: a persistent grid of resident blocks,
    // and (for k_large_dfs) the donation queue, whose ready flags are cleared
    // before the launch
    auto push_walk = [&](LaunchRec ld) -> beep_status {
        ld.tail_slot = 2;
        if (ld.kind == LaunchRec::kLargeDfs) {
            int per_sm = 1;
            if (ld.enumerate)
                BEEP_TRY(large_dfs_blocks_per_sm<true>(ld.dend, &per_sm));
            else
                BEEP_TRY(large_dfs_blocks_per_sm<false>(ld.dend, &per_sm));
            ld.grid = ctx->num_sms * per_sm;
            if (!lp->d_don_tasks) {
                lp->don_cap = kDonCap;
                BEEP_TRY(lp->alloc(lp->d_don_tasks, lp->don_cap));
                BEEP_TRY(lp->alloc(lp->d_don_ready, lp->don_cap));
                BEEP_TRY(lp->alloc(lp->d_don_ctl, (size_t)kDonWords * kMaxDonLaunches));
            }
            if (lp->ndon < kMaxDonLaunches && tiers.donate_min_iters >= 2) {
                Don &dn = ld.don;
                dn.tasks = lp->d_don_tasks;
                dn.ready = lp->d_don_ready;
                dn.ctl = lp->d_don_ctl + (size_t)kDonWords * lp->ndon++;
                dn.cap = lp->don_cap;
                dn.max_level = (uint32_t)(ld.dend + 2) / 2; // levels up to ceil((K + 1) / 2)
                dn.min_iters = tiers.donate_min_iters;
                dn.timeout_ns = (unsigned long long)(ctx->wait_timeout_ms * 1e6);
                LaunchRec ms;
                ms.kind = LaunchRec::kMemset;
                ms.mptr = lp->d_don_ready;
                ms.mbytes = (size_t)lp->don_cap * 4;
                lp->recs.push_back(ms);
            }
        }
        lp->recs.push_back(ld);
        return BEEP_OK;
    };

    // All item lists by one sort of (tier, depth, domain order) keys over the
    // flattened vertices; tier k's list is a contiguous run of the result.
    uint64_t *all_items = nullptr;
    uint32_t list_off[kTiers + 1] = {0};
    for (int k = 0; k < kTiers; ++k)
        list_off[k + 1] = list_off[k] + tier_n[k];
    BEEP_TRY(lp->alloc(all_items, list_off[kTiers]));
    if (list_off[kTiers] > 0) {
        k_list_keys<<<gv, 256, 0, s>>>(lp->d_tier, d_dom, lp->d_pairs, lp->d_offs, np, N, d_keys, d_sel);
        BEEP_CUDA_TRY(cudaGetLastError());
        size_t tb = 0;
        BEEP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_keys, d_keys2, d_sel, d_dom, N, 0, 32, s));
        BEEP_TRY(ctx->grow(ctx->scratch, tb + 1024));
        BEEP_CUDA_TRY(
            cub::DeviceRadixSort::SortPairs(ctx->scratch.ptr, tb, d_keys, d_keys2, d_sel, d_dom, N, 0, 32, s));
        k_make_items<<<std::max(1u, std::min(list_off[kTiers] / 256 + 1, 4096u)), 256, 0, s>>>(
            d_dom, list_off[kTiers], lp->d_offs, np, all_items);
        BEEP_CUDA_TRY(cudaGetLastError());
        st.kernel_launches += 2;
    }
    auto make_list = [&](int k, uint64_t *&list) -> beep_status {
        list = all_items + list_off[k];
        return BEEP_OK;
    };

    // large tier, one batch planned on the device when every root's bitmap
    // fits the arena at once (the arena words were summed by k_classify)
    size_t arena_cap = 0;
    if (tier_n[3] > 0) {
        size_t free_b = 0, total_b = 0;
        BEEP_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        arena_cap = std::max<size_t>((size_t)256 << 20, std::min<size_t>((size_t)48 << 30, free_b / 2));
    }
    // scratch of the large tier's 4-wheel tasks: U, its word list, x1's words
    // and U2 (W words each) for every warp of the DFS grid, zero on entry
    uint32_t *wsc = nullptr;
    uint32_t wstride = 0;
    {
        if (tier_depth[3 * kSlots + kWheelSlot] > 0 || tier_depth[3 * kSlots + kNbhdSlot] > 0) {
            wstride = (4 * ((tier_max[3] + 31) / 32) + 31) & ~31u;
            const size_t words = (size_t)ctx->num_sms * kLargeDfsBlocksPerSm * 8 * wstride;
            BEEP_TRY(lp->alloc(wsc, words));
            LaunchRec ms;
            ms.kind = LaunchRec::kMemset;
            ms.mptr = wsc;
            ms.mbytes = words * 4;
            lp->recs.push_back(ms);
        }
    }
    if (tier_n[3] > 0 && large_words * 4 <= arena_cap) {
        uint64_t *list = nullptr;
        BEEP_TRY(make_list(3, list));
        const uint32_t nl = tier_n[3];
        unsigned long long *words, *boff;
        uint32_t *chunks, *tasks, *cstart, *tstart, *arena;
        BEEP_TRY(lp->alloc(words, nl));
        BEEP_TRY(lp->alloc(boff, (size_t)nl + 1));
        BEEP_TRY(lp->alloc(chunks, nl));
        BEEP_TRY(lp->alloc(tasks, nl));
        BEEP_TRY(lp->alloc(cstart, (size_t)nl + 1));
        BEEP_TRY(lp->alloc(tstart, (size_t)nl + 1));
        BEEP_TRY(lp->alloc(arena, std::max<uint64_t>(large_words, 32)));
        const unsigned gl = std::max(1u, std::min(nl / 256 + 1, 1024u));
        k_gather_dom<<<gl, 256, 0, s>>>(lp->d_pairs, list, nl, d_keys, d_sel);
        k_large_meta<<<gl, 256, 0, s>>>(lp->d_pairs, list, nl, d_keys, d_sel, words, chunks, tasks);
        st.kernel_launches += 2;
        BEEP_CUDA_TRY(cudaGetLastError());
        // exclusive prefixes with the total at [nl]
        size_t tb = 0, tb2 = 0;
        BEEP_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, tb, words, boff + 1, nl, s));
        BEEP_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, tb2, chunks, cstart + 1, nl, s));
        BEEP_TRY(ctx->grow(ctx->scratch, std::max(tb, tb2) + 1024));
        tb = ctx->scratch.bytes;
        BEEP_CUDA_TRY(cub::DeviceScan::InclusiveSum(ctx->scratch.ptr, tb, words, boff + 1, nl, s));
        tb = ctx->scratch.bytes;
        BEEP_CUDA_TRY(cub::DeviceScan::InclusiveSum(ctx->scratch.ptr, tb, chunks, cstart + 1, nl, s));
        tb = ctx->scratch.bytes;
        BEEP_CUDA_TRY(cub::DeviceScan::InclusiveSum(ctx->scratch.ptr, tb, tasks, tstart + 1, nl, s));
        BEEP_CUDA_TRY(cudaMemsetAsync(boff, 0, 8, s));
        BEEP_CUDA_TRY(cudaMemsetAsync(cstart, 0, 4, s));
        BEEP_CUDA_TRY(cudaMemsetAsync(tstart, 0, 4, s));
        const uint32_t maxD_all = tier_max[3];
        const size_t smemA = std::min<size_t>(maxD_all, kLargeSmemA) * 4;
        BEEP_TRY(raise_smem_limit((const void *)k_large_rows, smemA));
        LaunchRec ms;
        ms.kind = LaunchRec::kMemset;
        ms.mptr = arena;
        ms.mbytes = large_words * 4;
        lp->recs.push_back(ms);
        st.bitmap_bytes += large_words * 4;
        LaunchRec lr;
        lr.kind = LaunchRec::kLargeRows;
        lr.grid = ctx->num_sms;
        lr.block = 512;
        lr.smem = smemA;
        lr.bt = Batch{list, reinterpret_cast<const uint64_t *>(boff), cstart, tstart, nl};
        lr.mptr = arena;
        BEEP_TRY(cursor(lr.cursor));
        lr.sink = &st.large_encode_ms;
        lp->recs.push_back(lr);
        if (list_cap((maxD_all + 31) / 32))
            lp->recs.push_back(lists_rec(lr));
        if (tier_depth[3 * kSlots + kNbhdSlot] > 0)
            lp->recs.push_back(nbdeg_rec(lr));
        uint32_t first = 0;
        for (int sl = 0; sl < kSlots; ++sl) {
            const uint32_t cnt = tier_depth[3 * kSlots + sl];
            if (!cnt)
                continue;
            const int d = sl % kDepths;
            LaunchRec ld;
            ld.kind = d == (int)kWheelSlot ? LaunchRec::kLargeWheel
                                           : (d == (int)kNbhdSlot ? LaunchRec::kLargeNbhd : LaunchRec::kLargeDfs);
            ld.dend = d;
            ld.enumerate = sl >= kDepths;
            ld.grid = ctx->num_sms * kLargeDfsBlocksPerSm;
            ld.block = 256;
            ld.bt = Batch{list + first, reinterpret_cast<const uint64_t *>(boff) + first, cstart, tstart + first,
                          cnt};
            ld.mptr = arena;
            BEEP_TRY(cursor(ld.cursor));
            ld.sink = &st.large_dfs_ms;
            ld.wsc = wsc;
            ld.wstride = wstride;
            BEEP_TRY(push_walk(ld));
            first += cnt;
        }
    } else if (tier_n[3] > 0) {
        // larger than the arena: batches planned on the host
        uint64_t *list = nullptr;
        BEEP_TRY(make_list(3, list));
        const uint32_t nl = tier_n[3];
        std::vector<uint64_t> litems(nl);
        std::vector<uint32_t> lD(nl), lj(nl);
        k_gather_dom<<<std::max(1u, std::min(nl / 256 + 1, 1024u)), 256, 0, s>>>(lp->d_pairs, list, nl, d_keys,
                                                                               d_sel);
        BEEP_CUDA_TRY(cudaGetLastError());
        st.kernel_launches += 1;
        BEEP_CUDA_TRY(cudaMemcpyAsync(litems.data(), list, 8ull * nl, cudaMemcpyDeviceToHost, s));
        BEEP_CUDA_TRY(cudaMemcpyAsync(lD.data(), d_keys, 4ull * nl, cudaMemcpyDeviceToHost, s));
        BEEP_CUDA_TRY(cudaMemcpyAsync(lj.data(), d_sel, 4ull * nl, cudaMemcpyDeviceToHost, s));
        BEEP_CUDA_TRY(cudaStreamSynchronize(s));
        struct R {
            uint64_t item;
            uint32_t D, j0, dend; // dend: the depth slot
            uint64_t words; // bitmap rows [rlo, D) of D bits and their word lists
        };
        std::vector<R> rs(nl);
        for (uint32_t i = 0; i < nl; ++i) {
            const DevPlan &pl = hp[(uint32_t)(litems[i] >> 32)].pl;
            const uint32_t D = lD[i], rlo = pl.rows_needed == 2 ? 0u : (pl.rows_needed == 1 ? lj[i] : D);
            const uint64_t words = large_root_words(D, rlo, pl.nbhd != kNbNone);
            const PairDev &pdv = hp[(uint32_t)(litems[i] >> 32)];
            rs[i] = R{litems[i], D, lj[i], depth_slot(pl, 4, pdv.en.out != nullptr), words};
        }
        std::sort(rs.begin(), rs.end(), [](const R &a, const R &b) { return a.D > b.D; });
        // batch boundaries and the arena size (largest batch)
        std::vector<std::pair<size_t, size_t>> batches;
        size_t arena_words = 0;
        for (size_t i0 = 0; i0 < rs.size();) {
            size_t words = 0, i1 = i0;
            while (i1 < rs.size()) {
                const uint64_t w = rs[i1].words;
                if (i1 > i0 && (words + w) * 4 > arena_cap)
                    break;
                words += w;
                ++i1;
            }
            if (words * 4 > arena_cap)
                return fail(BEEP_ERR_OUT_OF_MEMORY, "a root's neighbourhood bitmap (" + std::to_string(words * 4) +
                                                        " bytes) exceeds the bitmap arena");
            arena_words = std::max(arena_words, words);
            batches.push_back({i0, i1});
            i0 = i1;
        }
        uint32_t *arena = nullptr;
        BEEP_TRY(lp->alloc(arena, arena_words));
        const uint32_t maxD_all = rs[0].D;
        const size_t smemA = std::min<size_t>(maxD_all, kLargeSmemA) * 4;
        BEEP_TRY(raise_smem_limit((const void *)k_large_rows, smemA));
        for (auto &bb : batches) {
            const size_t i0 = bb.first, i1 = bb.second;
            std::stable_sort(rs.begin() + i0, rs.begin() + i1,
                             [](const R &a, const R &b) { return a.dend < b.dend; });
            const uint32_t nbt = (uint32_t)(i1 - i0);
            std::vector<uint64_t> bitem, boff;
            std::vector<uint32_t> cstart{0};
            uint64_t words = 0;
            uint32_t bmaxD = 0;
            for (size_t i = i0; i < i1; ++i) {
                bmaxD = std::max(bmaxD, rs[i].D);
                bitem.push_back(rs[i].item);
                boff.push_back(words);
                words += rs[i].words;
                cstart.push_back(cstart.back() + (rs[i].D + kRowsPerChunk - 1) / kRowsPerChunk);
            }
            std::vector<std::pair<uint32_t, uint32_t>> groups; // (first entry, count) per depth
            for (uint32_t a = 0; a < nbt;) {
                uint32_t b = a;
                while (b < nbt && rs[i0 + b].dend == rs[i0 + a].dend)
                    ++b;
                groups.push_back({a, b - a});
                a = b;
            }
            std::vector<uint32_t> ts_all, ts_off;
            for (auto &gp : groups) {
                ts_off.push_back((uint32_t)ts_all.size());
                uint32_t acc = 0;
                ts_all.push_back(0);
                for (uint32_t e = 0; e < gp.second; ++e) {
                    const R &x = rs[i0 + gp.first + e];
                    acc += x.D - x.j0;
                    ts_all.push_back(acc);
                }
            }
            uint64_t *d_bitem, *d_boff;
            uint32_t *d_cs, *d_ts;
            BEEP_TRY(lp->alloc(d_bitem, nbt));
            BEEP_TRY(lp->alloc(d_boff, nbt));
            BEEP_TRY(lp->alloc(d_cs, nbt + 1));
            BEEP_TRY(lp->alloc(d_ts, ts_all.size()));
            BEEP_CUDA_TRY(cudaMemcpyAsync(d_bitem, bitem.data(), nbt * 8, cudaMemcpyHostToDevice, s));
            BEEP_CUDA_TRY(cudaMemcpyAsync(d_boff, boff.data(), nbt * 8, cudaMemcpyHostToDevice, s));
            BEEP_CUDA_TRY(cudaMemcpyAsync(d_cs, cstart.data(), (nbt + 1) * 4, cudaMemcpyHostToDevice, s));
            BEEP_CUDA_TRY(cudaMemcpyAsync(d_ts, ts_all.data(), ts_all.size() * 4, cudaMemcpyHostToDevice, s));
            LaunchRec ms;
            ms.kind = LaunchRec::kMemset;
            ms.mptr = arena;
            ms.mbytes = words * 4;
            lp->recs.push_back(ms);
            st.bitmap_bytes += words * 4;
            LaunchRec lr;
            lr.kind = LaunchRec::kLargeRows;
            lr.grid = ctx->num_sms;
            lr.block = 512;
            lr.smem = smemA;
            lr.bt = Batch{d_bitem, d_boff, d_cs, d_ts, nbt};
            lr.mptr = arena;
            BEEP_TRY(cursor(lr.cursor));
            lr.sink = &st.large_encode_ms;
            lp->recs.push_back(lr);
            if (list_cap((bmaxD + 31) / 32))
                lp->recs.push_back(lists_rec(lr));
            bool any_nbhd = false;
            for (size_t i = i0; i < i1; ++i)
                any_nbhd |= rs[i].dend == kNbhdSlot;
            if (any_nbhd)
                lp->recs.push_back(nbdeg_rec(lr));
            for (size_t gi = 0; gi < groups.size(); ++gi) {
                LaunchRec ld;
                const uint32_t slot = rs[i0 + groups[gi].first].dend; // depth slot
                ld.dend = (int)(slot % kDepths);
                ld.enumerate = slot >= (uint32_t)kDepths;
                ld.kind = ld.dend == (int)kWheelSlot
                              ? LaunchRec::kLargeWheel
                              : (ld.dend == (int)kNbhdSlot ? LaunchRec::kLargeNbhd : LaunchRec::kLargeDfs);
                ld.grid = ctx->num_sms * kLargeDfsBlocksPerSm;
                ld.block = 256;
                ld.bt = Batch{d_bitem + groups[gi].first, d_boff + groups[gi].first, d_cs, d_ts + ts_off[gi],
                              groups[gi].second};
                ld.mptr = arena;
                BEEP_TRY(cursor(ld.cursor));
                ld.sink = &st.large_dfs_ms;
                ld.wsc = wsc;
                ld.wstride = wstride;
                BEEP_TRY(push_walk(ld));
            }
        }
    }
    tr.mark("large_batches");
    // medium tiers: block per root, bitmap in shared memory
    for (int sub = 0; sub < 2; ++sub) {
        const int k = 1 + sub;
        if (tier_n[k] == 0)
            continue;
        uint64_t *list = nullptr;
        BEEP_TRY(make_list(k, list));
        const uint32_t maxD = tier_max[k];
        // 32-bit words per row: 8 (4 x 64 bits) in the thread-mode sub-tier
        const uint32_t W = sub == 0 ? 2 * kThreadNW : (maxD + 31) / 32;
        const size_t pad = (maxD + 4) & ~3u;
        // the domain hash: nslots ids, nslots 16-bit indices and the filter
        const size_t nslots = hash_slots(maxD);
        const size_t smem = (4 * pad + nslots + nslots / 2 + nslots / 4 + (size_t)maxD * W) * 4;
        const int block = sub == 0 ? 256 : 1024;
        const int per_sm = std::max(1, (int)std::min<size_t>(2048 / block, (200 * 1024) / (smem + 1024)));
        uint32_t first = 0;
        for (int sl = 0; sl < kSlots; ++sl) {
            const uint32_t cnt = tier_depth[k * kSlots + sl];
            if (!cnt)
                continue;
            LaunchRec r;
            r.kind = LaunchRec::kMedium;
            r.dend = sl % kDepths;
            r.enumerate = sl >= kDepths;
            r.group = sub == 0 ? 0 : 32;
            r.grid = ctx->num_sms * per_sm;
            r.block = block;
            r.smem = smem;
            r.items = list + first;
            r.n = cnt;
            r.maxD = maxD;
            BEEP_TRY(cursor(r.cursor));
            r.sink = &st.medium_ms;
            r.tail_slot = 1;
            lp->recs.push_back(r);
            first += cnt;
        }
    }
    // small tier
    if (tier_n[0] > 0) {
        uint64_t *list = nullptr;
        BEEP_TRY(make_list(0, list));
        uint32_t first = 0;
        for (int sl = 0; sl < kSlots; ++sl) {
            // the list is sorted by (depth slot, domain): tiny domains first
            const uint32_t n_tiny = tiny_depth[sl], n_rest = tier_depth[sl] - tiny_depth[sl];
            for (int part = 0; part < 2; ++part) {
                const uint32_t cnt = part == 0 ? n_tiny : n_rest;
                if (!cnt)
                    continue;
                const int group = part == 0 ? 8 : 32;
                const int per_block = kSmallWarps * 32 / group;
                LaunchRec r;
                r.kind = LaunchRec::kSmall;
                r.dend = sl % kDepths;
                r.enumerate = sl >= kDepths;
                r.group = group;
                r.grid = (int)std::min<int64_t>(((int64_t)cnt + per_block - 1) / per_block,
                                                (int64_t)ctx->num_sms * 8);
                r.block = kSmallWarps * 32;
                r.items = list + first;
                r.n = cnt;
                r.sink = &st.small_ms;
                r.tail_slot = 0;
                lp->recs.push_back(r);
                first += cnt;
            }
        }
    }
    // list walker (queries without a central vertex): tasks = level-1 vertices
    if (tier_n[4] > 0) {
        uint64_t *list = nullptr;
        BEEP_TRY(make_list(4, list));
        const uint32_t nl = tier_n[4];
        uint32_t *tasks, *tstart;
        BEEP_TRY(lp->alloc(tasks, nl));
        BEEP_TRY(lp->alloc(tstart, (size_t)nl + 1));
        k_gather_dom<<<std::max(1u, std::min(nl / 256 + 1, 1024u)), 256, 0, s>>>(lp->d_pairs, list, nl, d_keys,
                                                                               d_sel);
        k_gen_tasks<<<std::max(1u, std::min(nl / 256 + 1, 1024u)), 256, 0, s>>>(d_keys, d_sel, nl, tasks);
        st.kernel_launches += 2;
        BEEP_CUDA_TRY(cudaGetLastError());
        size_t tb = 0;
        BEEP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, tasks, tstart, nl + 1, s));
        BEEP_TRY(ctx->grow(ctx->scratch, tb + 1024));
        // tasks[nl] is not written: scan nl entries, then the total into tstart[nl]
        BEEP_CUDA_TRY(cub::DeviceScan::InclusiveSum(ctx->scratch.ptr, tb, tasks, tstart + 1, nl, s));
        BEEP_CUDA_TRY(cudaMemsetAsync(tstart, 0, 4, s));
        uint32_t first = 0;
        for (int sl = 0; sl < kSlots; ++sl) {
            const uint32_t cnt = tier_depth[4 * kSlots + sl];
            if (!cnt)
                continue;
            LaunchRec r;
            r.kind = LaunchRec::kGeneral;
            r.dend = sl % kDepths;
            r.enumerate = sl >= kDepths;
            r.grid = ctx->num_sms * 8;
            r.block = 256;
            r.items = list + first;
            r.tstart = tstart + first;
            r.n = cnt;
            BEEP_TRY(cursor(r.cursor));
            r.sink = &st.general_ms;
            lp->recs.push_back(r);
            first += cnt;
        }
    }
    // shared-memory opt-ins are host calls: done here, never inside a capture
    for (auto &r : lp->recs)
        if (r.kind == LaunchRec::kMedium) {
#define BEEP_CASE(D)                                                                                               \
    case D:                                                                                                        \
        if (r.enumerate)                                                                                           \
            BEEP_TRY((set_medium_attr<D, true>(r.smem)));                                                          \
        else                                                                                                       \
            BEEP_TRY((set_medium_attr<D, false>(r.smem)));                                                         \
        break;
            BEEP_DEPTH_SWITCH(r.dend, BEEP_CASE)
#undef BEEP_CASE
        }
    lp->nexit = (uint32_t)lp->recs.size();
    BEEP_TRY(lp->alloc(lp->d_exit, 2 * (size_t)lp->nexit));
    BEEP_TRY(ctx->host_results(lp->host_words(), &lp->h_counts));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s)); // planning buffers are final
    tr.mark("lists");
    *out = std::move(lp);
    return BEEP_OK;
}

namespace {
beep_status issue(Ctx *ctx, LaunchPlan *lp, bool timing, bool serial, bool stall_test, beep_stats &st,
                  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> *ev,
                  std::vector<double *> *sinks) {
    cudaStream_t s = ctx->stream;
    const uint32_t np = lp->np;
    BEEP_CUDA_TRY(cudaMemsetAsync(lp->d_counts, 0, ((kPairWords + 1) * (size_t)np + kAux) * 8, s));
    for (unsigned *blk : lp->cursor_blocks)
        BEEP_CUDA_TRY(cudaMemsetAsync(blk, 0, kCursorBlock * 4, s));
    if (lp->ndon) {
        BEEP_CUDA_TRY(cudaMemsetAsync(lp->d_don_ctl, 0, (size_t)lp->ndon * kDonWords * 4, s));
        if (stall_test) // one phantom donated task that no donor publishes: every wait runs out
            for (uint32_t i = 0; i < lp->ndon; ++i)
                BEEP_CUDA_TRY(cudaMemsetAsync(lp->d_don_ctl + (size_t)i * kDonWords + kDonPending, 1, 1, s));
    }
    if (timing && lp->nexit)
        BEEP_CUDA_TRY(cudaMemsetAsync(lp->d_exit, 0, 2 * (size_t)lp->nexit * 8, s));
    // The tiers are independent: large on the call's stream, medium and small
    // on two side streams forked from it and joined back at the end.
    bool have_medium = false, have_small = false;
    for (auto &r : lp->recs) {
        have_medium |= r.kind == LaunchRec::kMedium;
        have_small |= r.kind == LaunchRec::kSmall;
    }
    const bool fork = (have_medium || have_small) && !serial;
    if (fork) {
        BEEP_TRY(ctx->ensure_side());
        BEEP_CUDA_TRY(cudaEventRecord(ctx->ev_fork, s));
        BEEP_CUDA_TRY(cudaStreamWaitEvent(ctx->side[0], ctx->ev_fork, 0));
        BEEP_CUDA_TRY(cudaStreamWaitEvent(ctx->side[1], ctx->ev_fork, 0));
    }
    for (size_t ri = 0; ri < lp->recs.size(); ++ri) {
        const LaunchRec &r = lp->recs[ri];
        unsigned long long *ex = timing ? lp->d_exit + 2 * ri : nullptr;
        cudaStream_t rs = s;
        if (fork && r.kind == LaunchRec::kMedium)
            rs = ctx->side[0];
        else if (fork && r.kind == LaunchRec::kSmall)
            rs = ctx->side[1];
        cudaEvent_t a = nullptr, b = nullptr;
        if (timing && r.sink) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, rs);
        }
        switch (r.kind) {
        case LaunchRec::kMemset:
            BEEP_CUDA_TRY(cudaMemsetAsync(r.mptr, 0, r.mbytes, rs));
            break;
        case LaunchRec::kLargeRows:
            k_large_rows<<<r.grid, r.block, r.smem, rs>>>(lp->d_pairs, r.bt, static_cast<uint32_t *>(r.mptr),
                                                          r.cursor);
            BEEP_CUDA_TRY(cudaGetLastError());
            st.large_encode_launches++;
            break;
        case LaunchRec::kLargeLists:
            k_large_lists<<<r.grid, r.block, 0, rs>>>(lp->d_pairs, r.bt, static_cast<uint32_t *>(r.mptr));
            BEEP_CUDA_TRY(cudaGetLastError());
            st.large_encode_launches++;
            break;
        case LaunchRec::kLargeDfs:
            if (r.enumerate)
                BEEP_TRY(launch_large_dfs<true>(r.dend, r.grid, rs, lp->d_pairs, r.bt,
                                                static_cast<const uint32_t *>(r.mptr), r.cursor, r.don, ex));
            else
                BEEP_TRY(launch_large_dfs<false>(r.dend, r.grid, rs, lp->d_pairs, r.bt,
                                                 static_cast<const uint32_t *>(r.mptr), r.cursor, r.don, ex));
            st.large_dfs_launches++;
            break;
        case LaunchRec::kLargeNbDeg:
            k_large_nbdeg<<<r.grid, r.block, 0, rs>>>(lp->d_pairs, r.bt, static_cast<uint32_t *>(r.mptr));
            BEEP_CUDA_TRY(cudaGetLastError());
            st.large_encode_launches++;
            break;
        case LaunchRec::kLargeNbhd:
            k_large_nbhd<<<r.grid, r.block, 0, rs>>>(lp->d_pairs, r.bt, static_cast<const uint32_t *>(r.mptr),
                                                     r.cursor, r.wsc, r.wstride, ex);
            BEEP_CUDA_TRY(cudaGetLastError());
            st.large_dfs_launches++;
            break;
        case LaunchRec::kLargeWheel:
            k_large_wheel<<<r.grid, r.block, 0, rs>>>(lp->d_pairs, r.bt, static_cast<const uint32_t *>(r.mptr),
                                                      r.cursor, r.wsc, r.wstride, ex);
            BEEP_CUDA_TRY(cudaGetLastError());
            st.large_dfs_launches++;
            break;
        case LaunchRec::kMedium:
#define BEEP_CASE(D)                                                                                               \
    case D:                                                                                                        \
        if (r.enumerate && r.group == 0)                                                                           \
            k_medium<D, true, 0><<<r.grid, r.block, r.smem, rs>>>(lp->d_pairs, r.items, r.n, r.cursor, r.maxD, ex); \
        else if (r.enumerate)                                                                                      \
            k_medium<D, true, 32><<<r.grid, r.block, r.smem, rs>>>(lp->d_pairs, r.items, r.n, r.cursor, r.maxD,    \
                                                                   ex);                                           \
        else if (r.group == 0)                                                                                     \
            k_medium<D, false, 0><<<r.grid, r.block, r.smem, rs>>>(lp->d_pairs, r.items, r.n, r.cursor, r.maxD,    \
                                                                   ex);                                           \
        else                                                                                                       \
            k_medium<D, false, 32><<<r.grid, r.block, r.smem, rs>>>(lp->d_pairs, r.items, r.n, r.cursor, r.maxD,   \
                                                                    ex);                                          \
        break;
            BEEP_DEPTH_SWITCH(r.dend, BEEP_CASE)
#undef BEEP_CASE
            BEEP_CUDA_TRY(cudaGetLastError());
            st.medium_launches++;
            break;
        case LaunchRec::kGeneral:
            if (r.enumerate)
                BEEP_TRY(launch_general<true>(r.dend, r.grid, rs, lp->d_pairs, r.items, r.tstart, r.n, r.cursor));
            else
                BEEP_TRY(launch_general<false>(r.dend, r.grid, rs, lp->d_pairs, r.items, r.tstart, r.n, r.cursor));
            st.general_launches++;
            break;
        case LaunchRec::kSmall:
            if (r.enumerate)
                BEEP_TRY(launch_small<true>(r.dend, r.group, r.grid, rs, lp->d_pairs, r.items, r.n, ex));
            else
                BEEP_TRY(launch_small<false>(r.dend, r.group, r.grid, rs, lp->d_pairs, r.items, r.n, ex));
            st.small_launches++;
            break;
        }
        if (r.kind != LaunchRec::kMemset)
            st.kernel_launches += 1;
        if (a) {
            cudaEventRecord(b, rs);
            ev->push_back({a, b});
            sinks->push_back(r.sink);
        }
    }
    if (fork) {
        for (int i = 0; i < 2; ++i) {
            BEEP_CUDA_TRY(cudaEventRecord(ctx->ev_join[i], ctx->side[i]));
            BEEP_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev_join[i], 0));
        }
    }
    return BEEP_OK;
}
} // namespace

// The read-back a run ends with: the (count, flag) words of every pair, the
// donation control blocks and (timing) the launches' exit times.
static cudaError_t readback(LaunchPlan *lp, cudaStream_t s, bool timing) {
    cudaError_t e =
        cudaMemcpyAsync(lp->h_counts, lp->d_counts, kPairWords * (size_t)lp->np * 8, cudaMemcpyDeviceToHost, s);
    unsigned long long *tel = lp->h_counts + kPairWords * (size_t)lp->np + kAux;
    if (e == cudaSuccess && lp->ndon)
        e = cudaMemcpyAsync(tel, lp->d_don_ctl, (size_t)lp->ndon * kDonWords * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && timing && lp->nexit)
        e = cudaMemcpyAsync(tel + (size_t)lp->ndon * kDonWords / 2, lp->d_exit, 2 * (size_t)lp->nexit * 8,
                            cudaMemcpyDeviceToHost, s);
    return e;
}

// Donation totals of the last run; BEEP_ERR_TIMEOUT when a bounded wait ran out.
static beep_status donation_result(const LaunchPlan *lp, uint64_t *donated) {
    const unsigned *ctl = reinterpret_cast<const unsigned *>(lp->h_counts + kPairWords * (size_t)lp->np + kAux);
    uint64_t d = 0;
    std::string where;
    for (uint32_t i = 0; i < lp->ndon; ++i) {
        const unsigned *c = ctl + (size_t)i * kDonWords;
        d += c[kDonCount];
        if (c[kDonError] && where.empty())
            where = "walk launch " + std::to_string(i) + " of " + std::to_string(lp->ndon) + ": slots claimed " +
                    std::to_string(c[kDonHead]) + ", reserved " + std::to_string(c[kDonTail]) + ", pending " +
                    std::to_string(c[kDonPending]) + ", static tasks done " + std::to_string(c[kDonStaticDone]) +
                    ", donated done " + std::to_string(c[kDonDone]) + ", heartbeats " +
                    std::to_string(c[kDonHeartbeat]);
    }
    if (donated)
        *donated = d;
    if (!where.empty())
        return fail(BEEP_ERR_TIMEOUT, "a warp of the large tier waited for donated work longer than the wait "
                                      "timeout with no progress anywhere (beep_ctx_set_wait_timeout); the counts of "
                                      "this run are incomplete (" + where + ")");
    return BEEP_OK;
}

beep_status capture_plan(Ctx *ctx, LaunchPlan *lp) {
    if (lp->exec)
        return BEEP_OK;
    cudaStream_t s = ctx->stream;
    // the captured read-back needs a host buffer that no other call reuses
    if (!lp->own_h_counts) {
        unsigned long long *h = nullptr;
        BEEP_CUDA_TRY(cudaMallocHost(&h, lp->host_words() * sizeof(unsigned long long)));
        lp->h_counts = h;
        lp->own_h_counts = true;
    }
    beep_stats scratch_st;
    std::memset(&scratch_st, 0, sizeof(scratch_st));
    cudaGraph_t graph = nullptr;
    BEEP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    beep_status rc = issue(ctx, lp, false, false, false, scratch_st, nullptr, nullptr);
    cudaError_t ce = readback(lp, s, false);
    cudaError_t e = cudaStreamEndCapture(s, &graph);
    if (rc != BEEP_OK) {
        if (graph)
            cudaGraphDestroy(graph);
        return rc;
    }
    BEEP_CUDA_TRY(ce);
    BEEP_CUDA_TRY(e);
    e = cudaGraphInstantiate(&lp->exec, graph, 0);
    cudaGraphDestroy(graph);
    BEEP_CUDA_TRY(e);
    return BEEP_OK;
}

beep_status execute_plan(Ctx *ctx, LaunchPlan *lp, uint32_t options, const std::vector<PairSpec> *specs_unused,
                         uint64_t *counts, size_t ncounts, beep_stats *stats) {
    (void)specs_unused;
    cudaStream_t s = ctx->stream;
    beep_stats st = lp->st;
    const bool timing = (options & BEEP_OPT_TIMING) != 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    std::vector<double *> sinks;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timing) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
    }
    if (lp->exec) {
        BEEP_CUDA_TRY(cudaGraphLaunch(lp->exec, s));
        st.kernel_launches = 0;
        for (auto &r : lp->recs)
            st.kernel_launches += r.kind != LaunchRec::kMemset;
    } else {
        st.kernel_launches = lp->st.kernel_launches;
        BEEP_TRY(issue(ctx, lp, timing, (options & BEEP_OPT_SERIAL_TIERS) != 0,
                       (options & BEEP_OPT_WAIT_STALL_TEST) != 0, st, &ev, &sinks));
        BEEP_CUDA_TRY(readback(lp, s, timing));
    }
    if (timing)
        cudaEventRecord(e1, s);
    if (lp->np > 0 && (options & BEEP_OPT_ALG_BYTES)) {
        unsigned long long *d_bytes = lp->d_counts + (kPairWords + 1) * (size_t)lp->np;
        BEEP_CUDA_TRY(cudaMemsetAsync(d_bytes, 0, kAux * 8, s));
        const int gv = std::max(1, (int)std::min<uint64_t>((lp->N + 255) / 256, (uint64_t)ctx->num_sms * 32));
        k_alg_bytes<<<gv, 256, 0, s>>>(lp->d_pairs, lp->d_offs, lp->np, lp->d_tier, lp->N, d_bytes);
        BEEP_CUDA_TRY(cudaGetLastError());
        st.kernel_launches += 1;
        BEEP_CUDA_TRY(cudaMemcpyAsync(lp->h_counts + kPairWords * (size_t)lp->np, d_bytes, kAux * 8,
                                      cudaMemcpyDeviceToHost, s));
    }
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    if (timing) {
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        st.count_ms = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        for (size_t i = 0; i < ev.size(); ++i) {
            cudaEventElapsedTime(&ms, ev[i].first, ev[i].second);
            *sinks[i] += ms;
            cudaEventDestroy(ev[i].first);
            cudaEventDestroy(ev[i].second);
        }
        // sinks point into lp->st; report through st
        st.small_ms = lp->st.small_ms;
        st.medium_ms = lp->st.medium_ms;
        st.large_encode_ms = lp->st.large_encode_ms;
        st.large_dfs_ms = lp->st.large_dfs_ms;
        st.general_ms = lp->st.general_ms;
        lp->st.small_ms = lp->st.medium_ms = lp->st.large_encode_ms = lp->st.large_dfs_ms = 0;
        lp->st.general_ms = 0;
    }
    for (size_t i = 0; i < ncounts; ++i)
        counts[i] = 0;
    st.count = 0;
    st.overflow_pairs = 0;
    for (uint32_t i = 0; i < lp->np; ++i) {
        const uint64_t c = pair_result(lp, i);
        if (lp->live[i] < ncounts)
            counts[lp->live[i]] = c;
        if (c == BEEP_COUNT_OVERFLOW)
            ++st.overflow_pairs;
        st.count = (st.count == BEEP_COUNT_OVERFLOW || c == BEEP_COUNT_OVERFLOW || st.count + c < st.count ||
                    st.count + c >= BEEP_COUNT_LIMIT)
                       ? BEEP_COUNT_OVERFLOW
                       : st.count + c;
    }
    if (options & BEEP_OPT_ALG_BYTES) {
        const unsigned long long *aux = lp->h_counts + kPairWords * (size_t)lp->np;
        st.small_bytes = aux[0];
        st.medium_bytes = aux[1];
        st.large_bytes = aux[2];
        st.adjacency_bytes = st.small_bytes + st.medium_bytes + st.large_bytes;
        st.alg_small_bytes = aux[3];
        st.alg_medium_bytes = aux[4];
        st.alg_large_bytes = aux[5];
    }
    const beep_status don_rc = donation_result(lp, &st.donated_tasks);
    if (timing && !lp->exec) {
        // per tier, the longest spread between a launch's first and last warp
        // exit: the time from "every item taken" to "every item done"
        const unsigned long long *ex =
            lp->h_counts + kPairWords * (size_t)lp->np + kAux + (size_t)lp->ndon * kDonWords / 2;
        double *tails[3] = {&st.small_tail_ms, &st.medium_tail_ms, &st.large_tail_ms};
        for (size_t ri = 0; ri < lp->recs.size(); ++ri) {
            const int slot = lp->recs[ri].tail_slot;
            if (slot < 0 || !ex[2 * ri + 1])
                continue;
            const unsigned long long first = ~ex[2 * ri], last = ex[2 * ri + 1];
            *tails[slot] = std::max(*tails[slot], (double)(last - first) / 1e6);
        }
    }
    if (stats)
        *stats = st;
    return don_rc;
}

beep_status launch_plan_async(Ctx *ctx, LaunchPlan *lp, unsigned long long *h_buf) {
    // the caller's pinned buffer (plan_host_words words) receives the
    // read-back: no pinned allocation or free on a server's latency path
    // (cudaFreeHost waits for the whole device)
    if (lp->h_counts && lp->own_h_counts)
        cudaFreeHost(lp->h_counts);
    lp->h_counts = h_buf;
    lp->own_h_counts = false;
    beep_stats st;
    std::memset(&st, 0, sizeof(st));
    BEEP_TRY(issue(ctx, lp, false, false, false, st, nullptr, nullptr));
    BEEP_CUDA_TRY(readback(lp, ctx->stream, false));
    return BEEP_OK;
}

size_t plan_host_words(const LaunchPlan *lp) { return lp->host_words(); }

beep_status plan_status(const LaunchPlan *lp) { return donation_result(lp, nullptr); }

uint64_t plan_count(const LaunchPlan *lp, size_t spec_index) {
    for (uint32_t i = 0; i < lp->np; ++i)
        if (lp->live[i] == spec_index)
            return pair_result(lp, i);
    return 0;
}

int plan_launches(const LaunchPlan *lp) {
    int n = lp->st.kernel_launches;
    for (auto &r : lp->recs)
        n += r.kind != LaunchRec::kMemset;
    return n;
}

beep_status run_pairs(Ctx *ctx, const std::vector<PairSpec> &specs, uint32_t options, beep_stats *stats,
                      uint64_t *counts) {
    cudaEvent_t p0 = nullptr, p1 = nullptr;
    const bool timing = (options & BEEP_OPT_TIMING) != 0;
    if (timing) {
        cudaEventCreate(&p0);
        cudaEventCreate(&p1);
        cudaEventRecord(p0, ctx->stream);
    }
    LaunchPlanPtr lp;
    BEEP_TRY(plan_pairs(ctx, specs, options, &lp));
    double prep_ms = 0;
    if (timing) {
        cudaEventRecord(p1, ctx->stream);
        cudaEventSynchronize(p1);
        float ms = 0;
        cudaEventElapsedTime(&ms, p0, p1);
        prep_ms = ms;
        cudaEventDestroy(p0);
        cudaEventDestroy(p1);
    }
    beep_stats st;
    PhaseTrace tr("count", ctx->stream);
    BEEP_TRY(execute_plan(ctx, lp.get(), options, &specs, counts, specs.size(), &st));
    tr.mark("execute");
    lp.reset();
    tr.mark("release");
    st.prep_ms = prep_ms;
    if (stats)
        *stats = st;
    return BEEP_OK;
}

beep_status run_count(Ctx *ctx, Graph *g, const QueryPlan &plan, uint32_t options, const EnumRequest *enreq,
                      beep_stats *stats, uint32_t shard, uint32_t nshards) {
    std::vector<PairSpec> one(1);
    one[0].g = g;
    one[0].plan = plan;
    one[0].en = enreq;
    one[0].shard = shard;
    one[0].nshards = nshards;
    uint64_t c = 0;
    return run_pairs(ctx, one, options, stats, &c);
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
    unsigned long long count;    // the match count ...
    unsigned long long overflow; // ... and its overflow flag (the word after it)
    unsigned int cursor;
    unsigned int max_domain;
    unsigned int bad_csr;        // bit 0: row pointers, bit 1: column entries
};
static_assert(sizeof(NoAllocCtrl) <= kNoAllocCtrlBytes, "control block");

// Largest search domain whose bitmap (D rows of ceil(D / 32) words, the slice
// rounded up to 64 words) fits the scratch array after the control block.
constexpr uint64_t noalloc_slice_words(uint64_t D) { return (D * ((D + 31) / 32) + 63) & ~(uint64_t)63; }
constexpr uint64_t kNoAllocArenaWords = (BEEP_NOALLOC_SCRATCH_BYTES - kNoAllocCtrlBytes) / 4;
static_assert(noalloc_slice_words(BEEP_NOALLOC_MAX_DOMAIN) <= kNoAllocArenaWords &&
                  noalloc_slice_words(BEEP_NOALLOC_MAX_DOMAIN + 1) > kNoAllocArenaWords,
              "BEEP_NOALLOC_MAX_DOMAIN is the largest domain whose bitmap fits the scratch array");

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

// A warp per row: checks the caller's CSR (row pointers non-decreasing
// within [0, m]; entries below n, strictly increasing, no self loop) before
// any kernel uses an entry as an index, and takes the largest search domain
// of the valid rows. Entries of a row are read only when its pointers are
// valid, so a bad CSR is reported, never read out of bounds.
__global__ void k_noalloc_maxdom(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ col, int64_t n,
                                 int64_t m, DevPlan pl, uint32_t min_deg, NoAllocCtrl *ctrl) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t mx = 0, bad = 0;
    for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        const uint32_t b = rp[v], e = rp[v + 1];
        if (b > e || (int64_t)e > m || (v == 0 && b != 0)) {
            bad |= 1u;
            continue;
        }
        for (uint32_t i = b + lane; i < e; i += 32) {
            const uint32_t w = col[i];
            if (!((int64_t)w < n && w != (uint32_t)v && (i == b || col[i - 1] < w)))
                bad |= 2u;
        }
        if (lane == 0) {
            uint32_t beg, D, j0, deg;
            csr_root_domain(rp, col, pl, (uint32_t)v, beg, D, j0, deg);
            if (csr_is_root(pl, deg, D, j0, min_deg))
                mx = max(mx, D);
        }
    }
    mx = __reduce_max_sync(kFull, mx);
    bad = __reduce_or_sync(kFull, bad);
    if (lane == 0 && mx)
        atomicMax(&ctrl->max_domain, mx);
    if (lane == 0 && bad)
        atomicOr(&ctrl->bad_csr, bad);
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
                dfs_warp<2, DEND, false>(lp, rows, 0u, W, D, x, cnt, lane, ec);
            }
        }
        __syncthreads();
    }
    cnt = warp_sum(cnt);
    if (lane == 0)
        flush_count(&ctrl->count, cnt);
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
    if (!plan.dev.central)
        return fail(BEEP_ERR_UNSUPPORTED, "queries without a central vertex: use beep_count");
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
        const int g0 = (int)std::max<int64_t>(1, std::min<int64_t>((n + 7) / 8, (int64_t)num_sms * 16));
        k_noalloc_maxdom<<<g0, 256, 0, s>>>(rp, col, n, m, pl, min_deg, ctrl);
        BEEP_CUDA_TRY(cudaGetLastError());
    }
    uint32_t h_ctrl[2] = {0, 0}; // max_domain, bad_csr
    BEEP_CUDA_TRY(cudaMemcpyAsync(h_ctrl, &ctrl->max_domain, sizeof(h_ctrl), cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    const uint32_t maxD = h_ctrl[0];
    if (h_ctrl[1] & 1u)
        return fail(BEEP_ERR_INVALID_ARG, "beep_count_noalloc: row_ptr must start at 0 and be non-decreasing "
                                          "within [0, m]");
    if (h_ctrl[1] & 2u)
        return fail(BEEP_ERR_INVALID_ARG, "beep_count_noalloc: every row must hold strictly increasing vertex ids "
                                          "below n with no self loop");
    if (maxD == 0) {
        *out_count = 0;
        return BEEP_OK;
    }
    const uint32_t smem_maxD = (uint32_t)kMediumMaxD;
    const uint64_t arena_words = kNoAllocArenaWords;
    uint64_t slice_words = 0;
    int grid = num_sms;
    if (maxD > smem_maxD) {
        slice_words = noalloc_slice_words(maxD);
        if (maxD > BEEP_NOALLOC_MAX_DOMAIN)
            return fail(BEEP_ERR_UNSUPPORTED,
                        "beep_count_noalloc: the largest search domain has " + std::to_string(maxD) +
                            " vertices; its bitmap needs " + std::to_string(slice_words * 4) +
                            " bytes, more than the " + std::to_string(BEEP_NOALLOC_SCRATCH_BYTES) +
                            "-byte scratch of the allocation-free path (domains up to " +
                            std::to_string(BEEP_NOALLOC_MAX_DOMAIN) + " vertices); use beep_count");
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
    unsigned long long c[2] = {0, 0}; // count, overflow flag
    BEEP_CUDA_TRY(cudaMemcpyAsync(c, &ctrl->count, sizeof(c), cudaMemcpyDeviceToHost, s));
    BEEP_CUDA_TRY(cudaStreamSynchronize(s));
    if (c[1]) {
        *out_count = BEEP_COUNT_OVERFLOW;
        return fail(BEEP_ERR_OVERFLOW, "beep_count_noalloc: the count is at least BEEP_COUNT_LIMIT (2^64 - 2^52)");
    }
    *out_count = c[0];
    return BEEP_OK;
}
