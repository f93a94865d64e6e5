/*
 * Stand-in for the four nauty entry points the reference's query compiler
 * calls (subgraph_matching/subgraph_matching.cuh:401-434): graph, optionblk,
 * statsblk, DEFAULTOPTIONS_GRAPH, EMPTYGRAPH, ADDONEEDGE and densenauty.
 * Only the orbits of the colour-preserving automorphism group are produced,
 * each labelled by its least vertex as nauty labels them; they are found by
 * exhaustive search, which is exact for the <= 10-vertex queries.
 *
 * TEST INFRASTRUCTURE ONLY: used to compile the reference as a second oracle.
 * Written from the published meaning of the interface, header-only, and
 * includable inside a C++ namespace (it includes nothing).
 *
 * The partition is given by lab/ptn: a cell ends at an index i with
 * ptn[i] == 0, and the last cell ends at n-1 whatever ptn[n-1] holds.
 */
#ifndef BEEP_REF_SHIM_NAUTY_H
#define BEEP_REF_SHIM_NAUTY_H

#ifndef FALSE
#define FALSE 0
#endif
#ifndef TRUE
#define TRUE 1
#endif

typedef unsigned long long setword;
typedef setword graph;
typedef int boolean;

typedef struct {
    int getcanon;
    boolean digraph;
    boolean writeautoms;
    boolean writemarkers;
    boolean defaultptn;
    boolean cartesian;
    int linelength;
} optionblk;

typedef struct {
    double grpsize1;
    int grpsize2;
    int numorbits;
    int numgenerators;
    int errstatus;
} statsblk;

#define DEFAULTOPTIONS_GRAPH(opt) optionblk opt = {0, FALSE, FALSE, FALSE, TRUE, FALSE, 78}
#define SHIM_BIT(j) (((setword)1) << (j))
#define EMPTYGRAPH(g, m, n)                                                                                    \
    do {                                                                                                       \
        for (int shim_i_ = 0; shim_i_ < (m) * (n); ++shim_i_)                                                  \
            (g)[shim_i_] = 0;                                                                                  \
    } while (0)
#define ADDONEEDGE(g, i, j, m)                                                                                 \
    do {                                                                                                       \
        (g)[(size_t)(m) * (i)] |= SHIM_BIT(j);                                                                 \
        (g)[(size_t)(m) * (j)] |= SHIM_BIT(i);                                                                 \
    } while (0)

/* Extend img[0..v) to a colour- and edge-preserving bijection. pre[v] >= 0
 * forces the image of v. Returns 1 if one exists. */
static inline int shim_extend(const setword *g, int n, const int *colour, int v, int *img, setword used,
                              const int *pre)
{
    if (v == n)
        return 1;
    for (int t = 0; t < n; ++t) {
        if (used & SHIM_BIT(t))
            continue;
        if (pre[v] >= 0 && pre[v] != t)
            continue;
        if (colour[t] != colour[v])
            continue;
        int ok = 1;
        for (int u = 0; u < v && ok; ++u) {
            int a = (g[u] & SHIM_BIT(v)) != 0;
            int b = (g[img[u]] & SHIM_BIT(t)) != 0;
            if (a != b)
                ok = 0;
        }
        if (!ok)
            continue;
        img[v] = t;
        if (shim_extend(g, n, colour, v + 1, img, used | SHIM_BIT(t), pre))
            return 1;
    }
    return 0;
}

static inline void densenauty(graph *g, int *lab, int *ptn, int *orbits, optionblk *options, statsblk *stats,
                              int m, int n, graph *h)
{
    (void)h;
    (void)m;
    int colour[64];
    if (options->defaultptn) {
        for (int i = 0; i < n; ++i)
            colour[i] = 0;
    } else {
        int c = 0;
        for (int i = 0; i < n; ++i) {
            colour[lab[i]] = c;
            if (ptn[i] == 0)
                ++c;
        }
    }
    int norb = 0;
    for (int i = 0; i < n; ++i) {
        orbits[i] = i;
        for (int j = 0; j < i; ++j) {
            int pre[64], img[64];
            for (int k = 0; k < n; ++k)
                pre[k] = -1;
            pre[j] = i;
            if (shim_extend(g, n, colour, 0, img, 0, pre)) {
                orbits[i] = orbits[j];
                break;
            }
        }
        if (orbits[i] == i)
            ++norb;
    }
    if (stats) {
        stats->numorbits = norb;
        stats->errstatus = 0;
        stats->grpsize1 = 1;
        stats->grpsize2 = 0;
        stats->numgenerators = 0;
    }
}

#endif
