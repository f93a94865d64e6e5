/*
 * oracle.h — CPU restatement of BEEP's sgm/sgc counting path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA
 * implementation in beep_b200/. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it. The product path never calls it.
 *
 * Every function cites the reference file:line whose behaviour it restates
 * (paths are relative to the reference repository root).
 *
 * Parity pin: the reference ships no tests or golden vectors. The oracle is
 * pinned by closed-form counts on complete graphs, by brute-force
 * embedding counts divided by |Aut(Q)| on small random graphs, by networkx
 * subgraph-monomorphism counts (tests/golden/make_golden.py) and, for the
 * fixtures recorded from it, by the reference's own binary built for sm_100a.
 */
#ifndef BEEP_ORACLE_H
#define BEEP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_DEPTH 10 /* subgraph_matching/include/host_utils.cuh:10 (DEPTH) */

typedef struct or_plan {
    int32_t K;                                   /* query vertices */
    int32_t order[OR_DEPTH];                     /* query vertex at each position */
    int32_t qdeg[OR_DEPTH];                      /* degree of the vertex at each position */
    int32_t qedge_ptr[OR_DEPTH + 1];             /* back edges of position i: qedge[qedge_ptr[i]..qedge_ptr[i+1]) */
    int32_t qedge[OR_DEPTH * (OR_DEPTH - 1) / 2];
    int32_t sym_ptr[OR_DEPTH + 1];               /* symmetry-breaking reps of position i */
    int32_t sym[OR_DEPTH * (OR_DEPTH - 1) / 2];
    int32_t unmat;                               /* LUNMAT: 1 if sgc stops one level early */
    int32_t first_sym_level;                     /* <=2: ascending degree order, else descending */
    int32_t min_qdeg, max_qdeg;
    int32_t central;                             /* 1 if position 0 is adjacent to every other position */
    int32_t aut_order;                           /* |Aut(Q)| (brute force) */
} or_plan;

/* Query plan from the query CSR exactly as the reference builds it from a .mtx
 * file (n = max src + 1, rows in src order). sgc != 0 selects GRAPH_COUNT.
 * Returns 0 on success, <0 on an unsupported query (K<2, K>10). */
int or_plan_query(int32_t qn, const int32_t *qrow_ptr, const int32_t *qcol, int32_t sgc, or_plan *out);

/* cutoff = ceil(mean + 6*sd) of the degree (include/utils.cuh:186-261). */
uint32_t or_cutoff(int64_t n, const int64_t *row_ptr);

/* Iterated peel of vertices with 1 <= deg < min_qdeg while more than 5% of n
 * are removed in a round (subgraph_matching.cuh:685-764). deg_out[n] receives
 * the final degrees; alive_out[n] (may be NULL) receives 1 for vertices whose
 * edges survive. Returns the number of peel rounds. */
int32_t or_peel(int64_t n, const int64_t *row_ptr, const int32_t *col, int32_t min_qdeg,
                int32_t *deg_out, uint8_t *alive_out);

/* Options for or_count. */
typedef struct or_options {
    int32_t apply_root_cap;   /* 1: skip roots with degree >= 100*cutoff (reference behaviour, subgraph_matching.cuh:1052,1098) */
    int32_t full_depth;       /* 1: count full matches even in sgc mode (sgm semantics) */
    int64_t root_stride;      /* process roots whose index in the root list is == root_offset mod root_stride */
    int64_t root_offset;
    int32_t threads;          /* OpenMP threads (0 = default) */
    int64_t root_mod;         /* > 1: only roots whose vertex id % root_mod == root_rem */
    int64_t root_rem;
} or_options;

typedef struct or_result {
    uint64_t count;
    int64_t roots;            /* roots in the root set */
    int64_t roots_processed;  /* roots this call processed (sampling) */
    uint32_t cutoff;
    int32_t peel_rounds;
    int32_t ascending;
    int32_t q2_risk;          /* 1 if the reference's skipped first heavy root could hold matches */
    int64_t q3_skipped;       /* roots with degree >= 100*cutoff */
} or_result;

/* Count matches of the planned query in the graph (CSR with both directions,
 * rows sorted by neighbour id, no duplicates, no self loops).
 * sgc selects the reference's GRAPH_COUNT semantics (LUNMAT).
 * Returns 0 on success. */
int or_count(int64_t n, const int64_t *row_ptr, const int32_t *col, const or_plan *plan,
             int32_t sgc, const or_options *opt, or_result *res);

/* Enumerate every match (full depth) as K-tuples in original query-vertex
 * order into out[cap*K]. Returns the total number of matches (may exceed cap). */
int64_t or_enumerate(int64_t n, const int64_t *row_ptr, const int32_t *col, const or_plan *plan,
                     int32_t *out, int64_t cap);

/* Independent check for cliques (not the reference's algorithm): the number
 * of k-cliques whose lowest vertex in the ascending (degree, id) order -- the
 * degrees left after or_peel with min_qdeg -- is a root with
 * id % root_mod == root_rem, by recursive intersection of sorted
 * higher-priority neighbour lists. */
uint64_t or_count_cliques(int64_t n, const int64_t *row_ptr, const int32_t *col, int32_t k, int32_t min_qdeg,
                          int64_t root_mod, int64_t root_rem, int32_t threads);

/* Brute force: injective edge-preserving maps Q -> G divided by |Aut(Q)|. */
uint64_t or_brute_force(int64_t n, const int64_t *row_ptr, const int32_t *col,
                        int32_t qn, const int32_t *qrow_ptr, const int32_t *qcol);

#ifdef __cplusplus
}
#endif
#endif
