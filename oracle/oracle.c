/*
 * oracle.c — CPU restatement of BEEP's sgm/sgc counting path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA path in
 * beep_b200/. Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load it; the product never calls it.
 *
 * Parity pin: the reference ships no tests or golden vectors. The oracle is
 * pinned by closed forms on complete graphs, by brute force (embeddings /
 * |Aut(Q)|), by networkx monomorphism counts and by counts recorded from the
 * reference binary itself (tests/golden/). nauty (2.7r1, not vendored by the
 * reference) is replaced by an exact automorphism search: only the orbit
 * partition of the pointwise stabiliser is consumed, and orbits are unique,
 * labelled by their least member as nauty labels them.
 *
 * All paths in citations are relative to the reference repository root.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* Automorphisms of the position graph                                        */
/* ------------------------------------------------------------------------- */

typedef struct {
    int n;
    uint8_t adj[OR_DEPTH][OR_DEPTH];
    int deg[OR_DEPTH];
} pgraph;

/* Backtracking search for automorphisms sigma with the given pre-assignment
 * (fixed[v] = image or -1). count_all != 0 counts all of them, otherwise
 * stops at the first. */
static long aut_search(const pgraph *g, int v, int *img, uint8_t *used, const int *fixed, int count_all)
{
    if (v == g->n)
        return 1;
    long total = 0;
    for (int t = 0; t < g->n; t++) {
        if (used[t])
            continue;
        if (fixed[v] >= 0 && fixed[v] != t)
            continue;
        if (g->deg[t] != g->deg[v])
            continue;
        int ok = 1;
        for (int u = 0; u < v && ok; u++)
            if (g->adj[u][v] != g->adj[img[u]][t])
                ok = 0;
        if (!ok)
            continue;
        img[v] = t;
        used[t] = 1;
        long r = aut_search(g, v + 1, img, used, fixed, count_all);
        used[t] = 0;
        total += r;
        if (total && !count_all)
            return total;
    }
    return total;
}

/* Orbits of the pointwise stabiliser of `hist`, each labelled by its least
 * member (the convention of nauty's orbits[] used at
 * subgraph_matching/subgraph_matching.cuh:434-439). */
static void stabiliser_orbits(const pgraph *g, const int *hist, int nh, int *orbits)
{
    for (int i = 0; i < g->n; i++) {
        orbits[i] = i;
        for (int j = 0; j < i; j++) {
            int fixed[OR_DEPTH], img[OR_DEPTH];
            uint8_t used[OR_DEPTH] = {0};
            for (int k = 0; k < g->n; k++)
                fixed[k] = -1;
            for (int k = 0; k < nh; k++)
                fixed[hist[k]] = hist[k];
            if (fixed[j] >= 0 && fixed[j] != i)
                continue;
            fixed[j] = i; /* some sigma maps j to i */
            if (aut_search(g, 0, img, used, fixed, 0)) {
                orbits[i] = j;
                break;
            }
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Query plan: subgraph_matching/subgraph_matching.cuh:257-505, 555-564, 612-631 */
/* ------------------------------------------------------------------------- */

int or_plan_query(int32_t qn, const int32_t *qrow_ptr, const int32_t *qcol, int32_t sgc, or_plan *out)
{
    memset(out, 0, sizeof(*out));
    if (qn < 2 || qn > OR_DEPTH)
        return -1;
    out->K = qn;
    int degree[OR_DEPTH];
    out->max_qdeg = 0;
    out->min_qdeg = 0x7fffffff;
    /* subgraph_matching.cuh:278-286 */
    for (int i = 0; i < qn; i++) {
        degree[i] = qrow_ptr[i + 1] - qrow_ptr[i];
        if (degree[i] > out->max_qdeg)
            out->max_qdeg = degree[i];
        if (degree[i] < out->min_qdeg)
            out->min_qdeg = degree[i];
    }
    /* Matching order by d_M * n + degree, first index wins ties (:296-333). */
    int d_M[OR_DEPTH] = {0};
    out->qedge_ptr[0] = 0;
    for (int i = 0; i < qn; i++) {
        unsigned ml = 0, idx = 0;
        for (int j = 0; j < qn; j++) {
            if (d_M[j] >= 0) {
                unsigned lk = (unsigned)d_M[j] * (unsigned)qn + (unsigned)degree[j];
                if (lk > ml) {
                    ml = lk;
                    idx = (unsigned)j;
                }
            }
        }
        out->order[i] = (int32_t)idx;
        out->qdeg[i] = degree[idx];
        d_M[idx] = -1;
        for (int e = qrow_ptr[idx]; e < qrow_ptr[idx + 1]; e++) {
            int nb = qcol[e];
            if (nb >= 0 && nb < qn && d_M[nb] != -1)
                d_M[nb]++;
        }
        /* Back edges to earlier positions, ascending (:335-350). */
        out->qedge_ptr[i + 1] = out->qedge_ptr[i];
        for (int j = 0; j < i; j++)
            for (int e = qrow_ptr[idx]; e < qrow_ptr[idx + 1]; e++)
                if (qcol[e] == out->order[j]) {
                    if (out->qedge_ptr[i + 1] >= OR_DEPTH * (OR_DEPTH - 1) / 2)
                        return -2;
                    out->qedge[out->qedge_ptr[i + 1]++] = j;
                }
    }
    /* Every vertex placed exactly once (fails for disconnected queries). */
    {
        int seen[OR_DEPTH] = {0};
        for (int i = 0; i < qn; i++) {
            if (seen[out->order[i]])
                return -3;
            seen[out->order[i]] = 1;
        }
    }
    /* Position graph used for nauty (:417-426). */
    pgraph g;
    memset(&g, 0, sizeof(g));
    g.n = qn;
    for (int i = 0; i < qn; i++)
        for (int e = out->qedge_ptr[i]; e < out->qedge_ptr[i + 1]; e++) {
            int j = out->qedge[e];
            g.adj[i][j] = g.adj[j][i] = 1;
        }
    for (int i = 0; i < qn; i++)
        for (int j = 0; j < qn; j++)
            g.deg[i] += g.adj[i][j];
    {
        int img[OR_DEPTH], fixed[OR_DEPTH];
        uint8_t used[OR_DEPTH] = {0};
        for (int k = 0; k < qn; k++)
            fixed[k] = -1;
        out->aut_order = (int32_t)aut_search(&g, 0, img, used, fixed, 1);
    }
    /* Orbit chain (:431-496): take the largest orbit (first label on ties),
     * add its label as a constraint to every other member, then fix it. */
    int sym[OR_DEPTH][OR_DEPTH];
    int nsym[OR_DEPTH] = {0};
    int hist[OR_DEPTH], nh = 0;
    for (;;) {
        int orbits[OR_DEPTH], cnts[OR_DEPTH] = {0};
        stabiliser_orbits(&g, hist, nh, orbits);
        for (int i = 0; i < qn; i++)
            cnts[orbits[i]]++;
        int maxLen = 0, maxIdx = -1;
        for (int i = 0; i < qn; i++)
            if (cnts[i] > maxLen) {
                maxLen = cnts[i];
                maxIdx = i;
            }
        if (maxLen == 1)
            break;
        for (int i = 0; i < qn; i++)
            if (orbits[i] == maxIdx && i != maxIdx)
                sym[i][nsym[i]++] = maxIdx;
        hist[nh++] = maxIdx;
        if (nh > qn)
            return -4;
    }
    out->sym_ptr[0] = 0;
    for (int i = 0; i < qn; i++) {
        out->sym_ptr[i + 1] = out->sym_ptr[i];
        for (int j = 0; j < nsym[i]; j++)
            out->sym[out->sym_ptr[i + 1]++] = sym[i][j];
    }
    /* first_sym_level (:555-562). The reference leaves it unset for a query
     * with no symmetry at all; without constraints the count does not depend
     * on the order, so ascending (0) is used. */
    out->first_sym_level = 0;
    for (int i = 1; i < qn + 1; i++)
        if (out->sym_ptr[i] > 0) {
            out->first_sym_level = i;
            break;
        }
    /* check_unmat, sgc only (:357-358, 612-631). */
    out->unmat = 0;
    if (sgc) {
        int found = 0;
        for (int e = out->qedge_ptr[qn - 1]; e < out->qedge_ptr[qn]; e++)
            if (out->qedge[e] == qn - 2)
                found = 1;
        if (!found)
            out->unmat = 1;
    }
    /* Central query: position 0 adjacent to every other position
     * (README.md:51-53; the kernels skip QEDGE[QEDGE_PTR[l]] assuming it is 0,
     * subgraph_matching/include/device_utils.cuh:438). */
    out->central = 1;
    for (int i = 1; i < qn; i++)
        if (out->qedge_ptr[i + 1] == out->qedge_ptr[i] || out->qedge[out->qedge_ptr[i]] != 0)
            out->central = 0;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Degree statistics: include/utils.cuh:186-261, called at src/main.cu:132    */
/* ------------------------------------------------------------------------- */

uint32_t or_cutoff(int64_t n, const int64_t *row_ptr)
{
    if (n <= 0)
        return 0;
    double total = 0;
    for (int64_t i = 0; i < n; i++)
        total += (double)(row_ptr[i + 1] - row_ptr[i]);
    double mean = total / (double)n;
    double ss = 0;
    for (int64_t i = 0; i < n; i++) {
        double diff = (double)(row_ptr[i + 1] - row_ptr[i]) - mean;
        ss += diff * diff;
    }
    double sd = sqrt(ss / (double)n);
    return (uint32_t)ceil(mean + 6.0 * sd);
}

/* ------------------------------------------------------------------------- */
/* Peel: subgraph_matching.cuh:685-764 with bucket_scan :66-109 and kernels   */
/* subgraph_matching/include/common_utils.cuh:99-133, 189-246                 */
/* ------------------------------------------------------------------------- */

int32_t or_peel(int64_t n, const int64_t *row_ptr, const int32_t *col, int32_t min_qdeg,
                int32_t *deg, uint8_t *alive_out)
{
    uint8_t *alive = (uint8_t *)malloc((size_t)(n > 0 ? n : 1));
    uint8_t *rem = (uint8_t *)malloc((size_t)(n > 0 ? n : 1));
    for (int64_t v = 0; v < n; v++) {
        alive[v] = 1;
        deg[v] = (int32_t)(row_ptr[v + 1] - row_ptr[v]);
    }
    int32_t rounds = 0;
    for (;;) {
        /* Window [1, min_qdeg) (bucket_scan with level 1, span min_qdeg-1). */
        int64_t removed = 0;
        for (int64_t v = 0; v < n; v++) {
            rem[v] = (deg[v] >= 1 && deg[v] < min_qdeg);
            removed += rem[v];
        }
        for (int64_t v = 0; v < n; v++)
            if (rem[v])
                alive[v] = 0;
        /* Edges touching a removed vertex are dropped in both directions;
         * recount (warp_detect_deleted_edges). */
        for (int64_t v = 0; v < n; v++) {
            int32_t c = 0;
            if (alive[v])
                for (int64_t e = row_ptr[v]; e < row_ptr[v + 1]; e++)
                    c += alive[col[e]];
            deg[v] = c;
        }
        rounds++;
        /* Loop condition (:758). */
        if (!((double)removed > 0.05 * (double)n))
            break;
    }
    if (alive_out)
        for (int64_t v = 0; v < n; v++)
            alive_out[v] = alive[v] && deg[v] > 0;
    free(alive);
    free(rem);
    return rounds;
}

/* ------------------------------------------------------------------------- */
/* DFS: subgraph_matching/sgm_kernelsLD.cuh:57-126 and                        */
/* subgraph_matching/include/device_utils.cuh:99-326, 426-456                 */
/* ------------------------------------------------------------------------- */

typedef struct {
    const or_plan *plan;
    int dend;           /* positions matched: K (sgm) or K - LUNMAT (sgc) */
    int d, W;           /* root degree, words per bitmap row */
    const uint32_t *bm; /* d x W induced adjacency of the oriented neighbour list */
    uint32_t *cand;     /* OR_DEPTH x W candidate words */
    int32_t x[OR_DEPTH];
    uint64_t count;
    /* enumeration */
    const int32_t *A;
    int32_t root;
    int32_t *out;
    int64_t cap, nout;
} dfs_ctx;

static inline uint32_t low_mask(int32_t idx, int32_t k)
{
    /* get_mask (common_utils.cuh:30-38): bits below idx in word k. The
     * reference relies on a 32-bit shift by 32 giving 0 on the GPU. */
    if (idx / 32 > k)
        return 0xFFFFFFFFu;
    if (idx / 32 < k)
        return 0u;
    int r = idx - k * 32;
    return r == 0 ? 0u : (0xFFFFFFFFu >> (32 - r));
}

static void or_dfs(dfs_ctx *c, int p)
{
    const or_plan *pl = c->plan;
    const int W = c->W, d = c->d;
    uint32_t *cand = c->cand + (size_t)p * W;
    const int e0 = pl->qedge_ptr[p], e1 = pl->qedge_ptr[p + 1];
    for (int k = 0; k < W; k++) {
        uint32_t all = (k < W - 1 || (d & 31) == 0) ? 0xFFFFFFFFu : ((1u << (d & 31)) - 1u);
        uint32_t t;
        if (p == 2) {
            /* count_tri (device_utils.cuh:187-206): row j if position 2 is
             * adjacent to positions 0 and 1, else every neighbour except j. */
            if (e1 - e0 == 2)
                t = c->bm[(size_t)c->x[1] * W + k];
            else
                t = all & ~(((uint32_t)(c->x[1] / 32 == k)) << (c->x[1] & 31));
            for (int s = pl->sym_ptr[2]; s < pl->sym_ptr[3]; s++)
                if (pl->sym[s] > 0)
                    t &= ~low_mask(c->x[1], k);
        } else {
            /* compute_intersection (device_utils.cuh:426-456): remaining
             * neighbours, AND the rows of every back edge after the first
             * (position 0), then the symmetry masks of reps > 0. */
            t = all;
            for (int q = 1; q < p; q++)
                if (c->x[q] / 32 == k)
                    t &= ~(1u << (c->x[q] & 31));
            for (int e = e0 + 1; e < e1; e++)
                t &= c->bm[(size_t)c->x[pl->qedge[e]] * W + k];
            for (int s = pl->sym_ptr[p]; s < pl->sym_ptr[p + 1]; s++)
                if (pl->sym[s] > 0)
                    t &= ~low_mask(c->x[pl->sym[s]], k);
        }
        cand[k] = t;
    }
    if (p == c->dend - 1) {
        /* Last level counted by popcount (check_terminate :244-264,
         * backtrack :303-306). */
        if (c->out) {
            for (int k = 0; k < W; k++) {
                uint32_t w = cand[k];
                while (w) {
                    int b = __builtin_ctz(w);
                    w &= w - 1;
                    if (c->nout < c->cap) {
                        int32_t *t = c->out + c->nout * pl->K;
                        t[pl->order[0]] = c->root;
                        for (int q = 1; q < p; q++)
                            t[pl->order[q]] = c->A[c->x[q]];
                        t[pl->order[p]] = c->A[k * 32 + b];
                    }
                    c->nout++;
                }
            }
        }
        for (int k = 0; k < W; k++)
            c->count += (uint64_t)__builtin_popcount(cand[k]);
        return;
    }
    /* Next candidate in ascending order (get_newIndex :266-292). */
    for (int k = 0; k < W; k++) {
        uint32_t w = cand[k];
        while (w) {
            int b = __builtin_ctz(w);
            w &= w - 1;
            c->x[p] = k * 32 + b;
            or_dfs(c, p + 1);
        }
    }
}

typedef struct {
    int64_t n;
    int asc;
    const int32_t *deg;
    int64_t *rank; /* vertex -> rank in the priority order */
} order_info;

static int cmp_i32(const void *a, const void *b)
{
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return x < y ? -1 : (x > y);
}

static int cmp_u64(const void *a, const void *b)
{
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : (x > y);
}

/* Priority order of degree_ordering (subgraph_matching.cuh:1282-1336 with
 * set_priority host_utils.cuh:230-246): ascending (degree, id) when
 * first_sym_level <= 2, else descending degree with ties by id (the stable
 * sorts keep the id order of the CSR rows). */
static void build_rank(order_info *o)
{
    uint64_t *keys = (uint64_t *)malloc((size_t)(o->n > 0 ? o->n : 1) * sizeof(uint64_t));
    for (int64_t v = 0; v < o->n; v++) {
        uint64_t dk = o->asc ? (uint64_t)(uint32_t)o->deg[v] : (uint64_t)(0xFFFFFFFFu - (uint32_t)o->deg[v]);
        keys[v] = (dk << 32) | (uint64_t)v;
    }
    qsort(keys, (size_t)o->n, sizeof(uint64_t), cmp_u64);
    for (int64_t i = 0; i < o->n; i++)
        o->rank[keys[i] & 0xFFFFFFFFu] = i;
    free(keys);
}

static void sort_by_rank(int32_t *a, int d, const int64_t *rank)
{
    /* insertion sort for short lists, else qsort on (rank, id) pairs */
    if (d < 32) {
        for (int i = 1; i < d; i++) {
            int32_t v = a[i];
            int64_t rv = rank[v];
            int j = i - 1;
            while (j >= 0 && rank[a[j]] > rv) {
                a[j + 1] = a[j];
                j--;
            }
            a[j + 1] = v;
        }
        return;
    }
    uint64_t *t = (uint64_t *)malloc((size_t)d * sizeof(uint64_t));
    for (int i = 0; i < d; i++)
        t[i] = ((uint64_t)rank[a[i]] << 32) | (uint32_t)a[i];
    qsort(t, (size_t)d, sizeof(uint64_t), cmp_u64);
    for (int i = 0; i < d; i++)
        a[i] = (int32_t)(t[i] & 0xFFFFFFFFu);
    free(t);
}

typedef struct {
    int64_t v;
    int32_t d;
} root_item;

static int cmp_root_desc(const void *a, const void *b)
{
    const root_item *x = (const root_item *)a, *y = (const root_item *)b;
    if (x->d != y->d)
        return x->d > y->d ? -1 : 1;
    return x->v < y->v ? -1 : (x->v > y->v);
}

static int count_impl(int64_t n, const int64_t *row_ptr, const int32_t *col, const or_plan *plan, int32_t sgc,
                      const or_options *opt, or_result *res, int32_t *enum_out, int64_t enum_cap, int64_t *enum_n)
{
    memset(res, 0, sizeof(*res));
    if (!plan || plan->K < 3 || plan->K > OR_DEPTH || !plan->central)
        return -1;
    or_options defopt = {1, 0, 1, 0, 0, 0, 0};
    if (!opt)
        opt = &defopt;
    const int K = plan->K;
    int dend = K;
    if (sgc && !opt->full_depth)
        dend = K - plan->unmat;

    res->cutoff = or_cutoff(n, row_ptr);
    int32_t *deg = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    uint8_t *alive = (uint8_t *)malloc((size_t)(n > 0 ? n : 1));
    res->peel_rounds = or_peel(n, row_ptr, col, plan->min_qdeg, deg, alive);

    order_info o;
    o.n = n;
    o.asc = plan->first_sym_level <= 2;
    o.deg = deg;
    o.rank = (int64_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
    build_rank(&o);
    res->ascending = o.asc;

    /* Root set (subgraph_matching.cuh:1086-1098): degree in
     * [max_qdeg, 100*cutoff), scheduled heaviest first (:1110-1111). */
    uint64_t cap = (uint64_t)res->cutoff * 100u;
    root_item *roots = (root_item *)malloc((size_t)(n > 0 ? n : 1) * sizeof(root_item));
    int64_t nr = 0;
    int32_t maxdeg = 0;
    for (int64_t v = 0; v < n; v++) {
        if (deg[v] < plan->max_qdeg)
            continue;
        if (opt->root_mod > 1 && v % opt->root_mod != opt->root_rem)
            continue;
        if ((uint64_t)deg[v] >= cap) {
            res->q3_skipped++;
            if (opt->apply_root_cap)
                continue;
        }
        roots[nr].v = v;
        roots[nr].d = deg[v];
        if (deg[v] > maxdeg)
            maxdeg = deg[v];
        nr++;
    }
    qsort(roots, (size_t)nr, sizeof(root_item), cmp_root_desc);
    res->roots = nr;

    /* Q2: with ascending order and heavy roots present the reference starts
     * its heavy-root cursor at 1 (subgraph_matching.cuh:1201), skipping the
     * first root of the degree-sorted queue. That root can hold matches only
     * if a neighbour outranks it, i.e. an adjacent max-degree tie. */
    if (o.asc && nr > 0 && (uint64_t)roots[0].d > res->cutoff) {
        for (int64_t i = 0; i < nr && roots[i].d == maxdeg && !res->q2_risk; i++) {
            int64_t v = roots[i].v;
            for (int64_t e = row_ptr[v]; e < row_ptr[v + 1]; e++) {
                int32_t w = col[e];
                if (alive[w] && deg[w] == maxdeg) {
                    res->q2_risk = 1;
                    break;
                }
            }
        }
    }

    int64_t stride = opt->root_stride > 0 ? opt->root_stride : 1;
    int64_t offset = opt->root_offset;
    uint64_t total = 0;
    int64_t processed = 0;
    int64_t nout = 0;

    int nthreads = 1;
#ifdef _OPENMP
    nthreads = opt->threads > 0 ? opt->threads : omp_get_max_threads();
    if (enum_out)
        nthreads = 1;
#endif

#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads) reduction(+ : total, processed)
#endif
    {
        int32_t *pos = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
        for (int64_t v = 0; v < n; v++)
            pos[v] = -1;
        int32_t *A = (int32_t *)malloc((size_t)(maxdeg > 0 ? maxdeg : 1) * sizeof(int32_t));
        size_t bm_cap = 0, cand_cap = 0;
        uint32_t *bm = NULL, *cand = NULL;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
        for (int64_t ri = 0; ri < nr; ri++) {
            if (((ri - offset) % stride + stride) % stride != 0)
                continue;
            processed++;
            int64_t r = roots[ri].v;
            /* Oriented neighbour list (degree_ordering + map_back). */
            int d = 0;
            for (int64_t e = row_ptr[r]; e < row_ptr[r + 1]; e++)
                if (alive[col[e]])
                    A[d++] = col[e];
            sort_by_rank(A, d, o.rank);
            int split = 0;
            if (o.asc)
                while (split < d && o.rank[A[split]] < o.rank[r])
                    split++;
            const int W = (d + 31) / 32;
            size_t need = (size_t)d * (size_t)W;
            if (need > bm_cap) {
                free(bm);
                bm_cap = need;
                bm = (uint32_t *)malloc(bm_cap * sizeof(uint32_t));
            }
            if ((size_t)OR_DEPTH * W > cand_cap) {
                free(cand);
                cand_cap = (size_t)OR_DEPTH * W;
                cand = (uint32_t *)malloc(cand_cap * sizeof(uint32_t));
            }
            memset(bm, 0, need * sizeof(uint32_t));
            /* encode (device_utils.cuh:99-127, host_utils.cuh:284-316): bit k
             * of row i set iff A[i] and A[k] are adjacent. */
            for (int i = 0; i < d; i++)
                pos[A[i]] = i;
            for (int i = 0; i < d; i++) {
                int32_t u = A[i];
                for (int64_t e = row_ptr[u]; e < row_ptr[u + 1]; e++) {
                    int32_t k = pos[col[e]];
                    if (k >= 0)
                        bm[(size_t)i * W + (k >> 5)] |= 1u << (k & 31);
                }
            }
            for (int i = 0; i < d; i++)
                pos[A[i]] = -1;

            dfs_ctx c;
            memset(&c, 0, sizeof(c));
            c.plan = plan;
            c.dend = dend;
            c.d = d;
            c.W = W;
            c.bm = bm;
            c.cand = cand;
            c.A = A;
            c.root = (int32_t)r;
            c.out = enum_out;
            c.cap = enum_cap;
            c.nout = nout;
            if (dend >= 3) {
                /* Level-1 loop (sgm_kernelsLD.cuh:57-60): skip j below the
                 * split when position 1 is symmetric to position 0. */
                for (int j = 0; j < d; j++) {
                    if (plan->sym_ptr[2] == 1 && j < split)
                        continue;
                    c.x[1] = j;
                    or_dfs(&c, 2);
                }
            }
            if (enum_out)
                nout = c.nout;
            total += c.count;
        }
        free(pos);
        free(A);
        free(bm);
        free(cand);
    }
    res->count = total;
    res->roots_processed = processed;
    if (enum_n)
        *enum_n = nout;
    free(deg);
    free(alive);
    free(o.rank);
    free(roots);
    return 0;
}

int or_count(int64_t n, const int64_t *row_ptr, const int32_t *col, const or_plan *plan, int32_t sgc,
             const or_options *opt, or_result *res)
{
    return count_impl(n, row_ptr, col, plan, sgc, opt, res, NULL, 0, NULL);
}

int64_t or_enumerate(int64_t n, const int64_t *row_ptr, const int32_t *col, const or_plan *plan, int32_t *out,
                     int64_t cap)
{
    or_options opt = {0, 1, 1, 0, 1, 0, 0};
    or_result res;
    int64_t nout = 0;
    if (count_impl(n, row_ptr, col, plan, 0, &opt, &res, out, cap, &nout) != 0)
        return -1;
    return nout;
}

/* ------------------------------------------------------------------------- */
/* Brute force (independent of the reference's algorithm)                     */
/* ------------------------------------------------------------------------- */

static int has_edge(const int64_t *row_ptr, const int32_t *col, int32_t u, int32_t v)
{
    int64_t lo = row_ptr[u], hi = row_ptr[u + 1];
    while (lo < hi) {
        int64_t mid = (lo + hi) / 2;
        if (col[mid] == v)
            return 1;
        if (col[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return 0;
}

typedef struct {
    int64_t n;
    const int64_t *row_ptr;
    const int32_t *col;
    int qn;
    int ord[OR_DEPTH];
    uint8_t qadj[OR_DEPTH][OR_DEPTH];
    int32_t img[OR_DEPTH];
    uint64_t cnt;
} bf_ctx;

static void bf_rec(bf_ctx *c, int i)
{
    if (i == c->qn) {
        c->cnt++;
        return;
    }
    int qv = c->ord[i];
    /* candidates: neighbours of an already-mapped adjacent vertex, if any */
    int anchor = -1;
    for (int k = 0; k < i; k++)
        if (c->qadj[qv][c->ord[k]]) {
            anchor = c->ord[k];
            break;
        }
    int64_t lo = 0, hi = c->n;
    if (anchor >= 0) {
        lo = c->row_ptr[c->img[anchor]];
        hi = c->row_ptr[c->img[anchor] + 1];
    }
    for (int64_t t = lo; t < hi; t++) {
        int32_t v = anchor >= 0 ? c->col[t] : (int32_t)t;
        int ok = 1;
        for (int k = 0; k < i && ok; k++) {
            int qk = c->ord[k];
            if (c->img[qk] == v)
                ok = 0;
            else if (c->qadj[qv][qk] && !has_edge(c->row_ptr, c->col, v, c->img[qk]))
                ok = 0;
        }
        if (!ok)
            continue;
        c->img[qv] = v;
        bf_rec(c, i + 1);
    }
}

uint64_t or_brute_force(int64_t n, const int64_t *row_ptr, const int32_t *col, int32_t qn, const int32_t *qrow_ptr,
                        const int32_t *qcol)
{
    if (qn < 1 || qn > OR_DEPTH)
        return 0;
    bf_ctx c;
    memset(&c, 0, sizeof(c));
    c.n = n;
    c.row_ptr = row_ptr;
    c.col = col;
    c.qn = qn;
    for (int v = 0; v < qn; v++)
        for (int e = qrow_ptr[v]; e < qrow_ptr[v + 1]; e++)
            if (qcol[e] != v)
                c.qadj[v][qcol[e]] = c.qadj[qcol[e]][v] = 1;
    /* BFS order from vertex 0 for pruning */
    int seen[OR_DEPTH] = {0}, nq = 0;
    for (int s = 0; s < qn; s++) {
        if (seen[s])
            continue;
        seen[s] = 1;
        c.ord[nq++] = s;
        for (int h = nq - 1; h < nq; h++)
            for (int w = 0; w < qn; w++)
                if (c.qadj[c.ord[h]][w] && !seen[w]) {
                    seen[w] = 1;
                    c.ord[nq++] = w;
                }
    }
    bf_rec(&c, 0);
    pgraph g;
    memset(&g, 0, sizeof(g));
    g.n = qn;
    for (int i = 0; i < qn; i++)
        for (int j = 0; j < qn; j++) {
            g.adj[i][j] = c.qadj[i][j];
            g.deg[i] += c.qadj[i][j];
        }
    int img[OR_DEPTH], fixed[OR_DEPTH];
    uint8_t used[OR_DEPTH] = {0};
    for (int k = 0; k < qn; k++)
        fixed[k] = -1;
    long aut = aut_search(&g, 0, img, used, fixed, 1);
    return aut ? c.cnt / (uint64_t)aut : 0;
}

/* ------------------------------------------------------------------------- */
/* Independent clique counter (checks, not a restatement)                     */
/* ------------------------------------------------------------------------- */

static uint64_t clique_rec(const int64_t *out_ptr, const int32_t *out_col, const int32_t *cand, int nc, int left,
                           int32_t *buf)
{
    if (left == 1)
        return (uint64_t)nc;
    uint64_t total = 0;
    for (int i = 0; i < nc; i++) {
        int32_t v = cand[i];
        /* cand ∩ out(v), both ascending */
        const int32_t *a = cand + i + 1;
        int na = nc - i - 1;
        const int32_t *b = out_col + out_ptr[v];
        int nb = (int)(out_ptr[v + 1] - out_ptr[v]);
        int m = 0, x = 0, y = 0;
        while (x < na && y < nb) {
            if (a[x] < b[y])
                x++;
            else if (a[x] > b[y])
                y++;
            else {
                buf[m++] = a[x];
                x++;
                y++;
            }
        }
        if (m >= left - 1)
            total += clique_rec(out_ptr, out_col, buf, m, left - 1, buf + m);
    }
    return total;
}

uint64_t or_count_cliques(int64_t n, const int64_t *row_ptr, const int32_t *col, int32_t k, int32_t min_qdeg,
                          int64_t root_mod, int64_t root_rem, int32_t threads)
{
    if (k < 2)
        return 0;
    /* rank by ascending (peeled degree, id); out-lists hold higher-ranked
     * surviving neighbours as ranks, ascending */
    int32_t *pdeg = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * 4);
    uint8_t *alive = (uint8_t *)malloc((size_t)(n > 0 ? n : 1));
    or_peel(n, row_ptr, col, min_qdeg, pdeg, alive);
    uint64_t *keys = (uint64_t *)malloc((size_t)(n > 0 ? n : 1) * 8);
    int64_t *rank = (int64_t *)malloc((size_t)(n > 0 ? n : 1) * 8);
    for (int64_t v = 0; v < n; v++)
        keys[v] = ((uint64_t)(uint32_t)pdeg[v] << 32) | (uint64_t)v;
    qsort(keys, (size_t)n, 8, cmp_u64);
    int32_t *vert = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * 4);
    for (int64_t i = 0; i < n; i++) {
        rank[keys[i] & 0xFFFFFFFFu] = i;
        vert[i] = (int32_t)(keys[i] & 0xFFFFFFFFu);
    }
    int64_t *optr = (int64_t *)calloc((size_t)n + 1, 8);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4096)
#endif
    for (int64_t i = 0; i < n; i++) {
        int32_t v = vert[i];
        int64_t c = 0;
        if (alive[v])
            for (int64_t e = row_ptr[v]; e < row_ptr[v + 1]; e++)
                c += alive[col[e]] && rank[col[e]] > i;
        optr[i + 1] = c;
    }
    for (int64_t i = 0; i < n; i++)
        optr[i + 1] += optr[i];
    int32_t *ocol = (int32_t *)malloc((size_t)(optr[n] > 0 ? optr[n] : 1) * 4);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4096)
#endif
    for (int64_t i = 0; i < n; i++) {
        int32_t v = vert[i];
        int64_t o = optr[i];
        if (alive[v])
            for (int64_t e = row_ptr[v]; e < row_ptr[v + 1]; e++)
                if (alive[col[e]] && rank[col[e]] > i)
                    ocol[o++] = (int32_t)rank[col[e]];
        /* sort the out-list of rank i */
        int32_t *a = ocol + optr[i];
        int len = (int)(optr[i + 1] - optr[i]);
        if (len > 32) {
            qsort(a, (size_t)len, 4, cmp_i32);
            continue;
        }
        for (int x = 1; x < len; x++) {
            int32_t t = a[x];
            int y = x - 1;
            while (y >= 0 && a[y] > t) {
                a[y + 1] = a[y];
                y--;
            }
            a[y + 1] = t;
        }
    }
    uint64_t total = 0;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = threads > 0 ? threads : omp_get_max_threads();
#endif
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads) reduction(+ : total)
#endif
    {
        int64_t maxo = 0;
        for (int64_t i = 0; i < n; i++)
            if (optr[i + 1] - optr[i] > maxo)
                maxo = optr[i + 1] - optr[i];
        int32_t *buf = (int32_t *)malloc((size_t)(maxo + 1) * (size_t)k * 4 + 64);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
        for (int64_t i = 0; i < n; i++) {
            if (root_mod > 1 && (int64_t)vert[i] % root_mod != root_rem)
                continue;
            int nc = (int)(optr[i + 1] - optr[i]);
            if (nc < k - 1)
                continue;
            total += clique_rec(optr, ocol, ocol + optr[i], nc, k - 1, buf);
        }
        free(buf);
    }
    free(keys);
    free(rank);
    free(vert);
    free(optr);
    free(ocol);
    free(pdeg);
    free(alive);
    return total;
}
