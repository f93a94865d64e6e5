// plan.cpp — query compiler: matching order, back edges, automorphism-based
// symmetry breaking and the sgc early-stop rule, following
// SG_Match::preprocess_query / detect_symmetry / detect_reuse / check_unmat
// (subgraph_matching/subgraph_matching.cuh:257-631 in the reference).
//
// nauty's densenauty (called at subgraph_matching.cuh:434) is replaced by an
// exact automorphism search over the <= 10 query vertices. Only the orbit
// partition of the group fixing the already-chosen representatives pointwise
// is used, and orbits are unique; like nauty, each orbit is named by its
// least member.
#include <algorithm>
#include <array>

#include "internal.h"

namespace beep {

namespace {

struct SmallGraph {
    int n = 0;
    std::array<std::array<uint8_t, kMaxQ>, kMaxQ> adj{};
    std::array<int, kMaxQ> deg{};
};

// Does an automorphism exist that extends `img` (img[v] = -1: free)?
// count != nullptr: count every automorphism instead.
bool extend_aut(const SmallGraph &g, int v, std::array<int, kMaxQ> &img, std::array<int, kMaxQ> &pre,
                uint32_t used, long *count) {
    if (v == g.n) {
        if (count) {
            ++*count;
            return false;
        }
        return true;
    }
    for (int t = 0; t < g.n; ++t) {
        if (used >> t & 1u)
            continue;
        if (pre[v] >= 0 && pre[v] != t)
            continue;
        if (g.deg[t] != g.deg[v])
            continue;
        bool ok = true;
        for (int u = 0; u < v && ok; ++u)
            ok = g.adj[u][v] == g.adj[img[u]][t];
        if (!ok)
            continue;
        img[v] = t;
        if (extend_aut(g, v + 1, img, pre, used | (1u << t), count))
            return true;
    }
    return false;
}

// Orbits of the subgroup fixing every vertex of `fixed_pts`, named by their
// least member.
std::array<int, kMaxQ> orbits_fixing(const SmallGraph &g, const std::vector<int> &fixed_pts) {
    std::array<int, kMaxQ> orb{};
    for (int i = 0; i < g.n; ++i) {
        orb[i] = i;
        for (int j = 0; j < i; ++j) {
            std::array<int, kMaxQ> pre, img;
            pre.fill(-1);
            img.fill(-1);
            for (int f : fixed_pts)
                pre[f] = f;
            if (pre[j] >= 0 && pre[j] != i)
                continue;
            pre[j] = i;
            if (extend_aut(g, 0, img, pre, 0u, nullptr)) {
                orb[i] = j;
                break;
            }
        }
    }
    return orb;
}

} // namespace

beep_status compile_plan(int32_t qn, const std::vector<int32_t> &rp, const std::vector<int32_t> &col, beep_mode mode,
                         QueryPlan *out) {
    if (qn < 3 || qn > kMaxQ)
        return fail(BEEP_ERR_UNSUPPORTED, "query must have 3.." + std::to_string(kMaxQ) + " vertices, has " +
                                              std::to_string(qn));
    beep_plan_info P;
    std::memset(&P, 0, sizeof(P));
    P.K = qn;
    std::array<int, kMaxQ> degree{};
    P.max_qdeg = 0;
    P.min_qdeg = 1 << 30;
    for (int v = 0; v < qn; ++v) {
        degree[v] = rp[v + 1] - rp[v];
        P.max_qdeg = std::max(P.max_qdeg, degree[v]);
        P.min_qdeg = std::min(P.min_qdeg, degree[v]);
    }
    // Position order: repeatedly the unplaced vertex maximising
    // (#placed neighbours) * n + degree, lowest index on ties.
    std::array<int, kMaxQ> placed_nbrs{};
    std::array<bool, kMaxQ> placed{};
    P.qedge_ptr[0] = 0;
    for (int i = 0; i < qn; ++i) {
        long best = -1;
        int pick = -1;
        for (int v = 0; v < qn; ++v) {
            if (placed[v])
                continue;
            long score = (long)placed_nbrs[v] * qn + degree[v];
            if (score > best && score > 0) {
                best = score;
                pick = v;
            }
        }
        if (pick < 0)
            return fail(BEEP_ERR_UNSUPPORTED, "query is not connected");
        placed[pick] = true;
        P.order[i] = pick;
        P.qdeg[i] = degree[pick];
        for (int e = rp[pick]; e < rp[pick + 1]; ++e)
            if (col[e] >= 0 && col[e] < qn && !placed[col[e]])
                placed_nbrs[col[e]]++;
        // back edges: earlier positions adjacent to this vertex, ascending
        P.qedge_ptr[i + 1] = P.qedge_ptr[i];
        for (int j = 0; j < i; ++j)
            for (int e = rp[pick]; e < rp[pick + 1]; ++e)
                if (col[e] == P.order[j]) {
                    if (P.qedge_ptr[i + 1] >= kMaxQ * (kMaxQ - 1) / 2)
                        return fail(BEEP_ERR_UNSUPPORTED, "query has duplicate edges");
                    P.qedge[P.qedge_ptr[i + 1]++] = j;
                }
    }
    // Position graph and its automorphisms.
    SmallGraph g;
    g.n = qn;
    for (int i = 0; i < qn; ++i)
        for (int e = P.qedge_ptr[i]; e < P.qedge_ptr[i + 1]; ++e) {
            int j = P.qedge[e];
            g.adj[i][j] = g.adj[j][i] = 1;
        }
    for (int i = 0; i < qn; ++i)
        for (int j = 0; j < qn; ++j)
            g.deg[i] += g.adj[i][j];
    for (int v = 0; v < qn; ++v)
        if (g.deg[v] != degree[P.order[v]])
            return fail(BEEP_ERR_UNSUPPORTED, "query edge list is not symmetric");
    {
        std::array<int, kMaxQ> pre, img;
        pre.fill(-1);
        img.fill(-1);
        long naut = 0;
        extend_aut(g, 0, img, pre, 0u, &naut);
        P.aut_order = (int32_t)naut;
    }
    // Orbit chain: fix the least member of the largest orbit (first on ties)
    // and require every other member of that orbit to follow it.
    std::vector<int> sym[kMaxQ];
    std::vector<int> fixed_pts;
    for (;;) {
        auto orb = orbits_fixing(g, fixed_pts);
        std::array<int, kMaxQ> size{};
        for (int i = 0; i < qn; ++i)
            size[orb[i]]++;
        int big = 0, rep = -1;
        for (int i = 0; i < qn; ++i)
            if (size[i] > big) {
                big = size[i];
                rep = i;
            }
        if (big <= 1)
            break;
        for (int i = 0; i < qn; ++i)
            if (orb[i] == rep && i != rep)
                sym[i].push_back(rep);
        fixed_pts.push_back(rep);
    }
    P.sym_ptr[0] = 0;
    for (int i = 0; i < qn; ++i) {
        P.sym_ptr[i + 1] = P.sym_ptr[i];
        for (int s : sym[i])
            P.sym[P.sym_ptr[i + 1]++] = s;
    }
    // First position with a constraint decides ascending (<= 2) or descending
    // order (subgraph_matching.cuh:555-562, 1299). With no constraint at all
    // the order cannot change the count; ascending is used.
    P.first_sym_level = 0;
    for (int i = 1; i <= qn; ++i)
        if (P.sym_ptr[i] > 0) {
            P.first_sym_level = i;
            break;
        }
    // sgc: the last position is left unmaterialised when it is not adjacent
    // to the position before it.
    P.unmat = 0;
    if (mode == BEEP_MODE_SGC) {
        bool adj_prev = false;
        for (int e = P.qedge_ptr[qn - 1]; e < P.qedge_ptr[qn]; ++e)
            adj_prev |= P.qedge[e] == qn - 2;
        P.unmat = adj_prev ? 0 : 1;
    }
    // The bitmap DFS needs position 0 adjacent to every position
    // (README.md:51-53); other queries go to the list walker, which counts
    // full matches only.
    P.central = 1;
    for (int i = 1; i < qn; ++i) {
        if (P.qedge_ptr[i + 1] == P.qedge_ptr[i])
            return fail(BEEP_ERR_UNSUPPORTED, "query is not connected");
        if (P.qedge[P.qedge_ptr[i]] != 0)
            P.central = 0;
    }
    if (!P.central && P.unmat)
        return fail(BEEP_ERR_UNSUPPORTED,
                    "sgc prefix counts (last position not adjacent to the one before) need a central query");

    // Kernel view of the plan.
    DevPlan D;
    std::memset(&D, 0, sizeof(D));
    D.K = qn;
    D.dend = (mode == BEEP_MODE_SGC) ? qn - P.unmat : qn;
    for (int p = 0; p < qn; ++p) {
        D.order[p] = P.order[p];
        for (int e = P.qedge_ptr[p]; e < P.qedge_ptr[p + 1]; ++e)
            if (P.qedge[e] >= 1)
                D.back[p] |= 1u << P.qedge[e];
        // Constraints against position 0 are enforced only at position 1
        // through the split point (sgm_kernelsLD.cuh:60); for later
        // positions they follow from the chain through position 1
        // (device_utils.cuh:448 skips them).
        for (int s = P.sym_ptr[p]; s < P.sym_ptr[p + 1]; ++s)
            if (P.sym[s] >= 1)
                D.sym[p] |= 1u << P.sym[s];
    }
    D.pos1_after_root = (P.sym_ptr[2] - P.sym_ptr[1]) == 1 ? 1 : 0;
    D.asc = P.first_sym_level <= 2 ? 1 : 0;
    // Restricted search: if position 1 follows the root and every later
    // position follows position 1 through the constraint chain, all matched
    // vertices follow the root, so only the root's later neighbours matter.
    bool restricted = D.pos1_after_root != 0 && P.central;
    std::array<uint32_t, kMaxQ> after{}; // positions that p must follow (transitively)
    for (int p = 1; p < qn; ++p) {
        uint32_t a = D.sym[p];
        for (int s = 1; s < p; ++s)
            if (D.sym[p] >> s & 1u)
                a |= after[s];
        after[p] = a;
        if (p >= 2 && !(a >> 1 & 1u))
            restricted = false;
    }
    D.restricted = restricted ? 1 : 0;
    P.restricted = D.restricted;
    // Free suffix: the last positions that all have the same back edges
    // (none of them inside the suffix) and where each follows the one before
    // it. Their completions are counted in closed form by the kernels.
    D.free_from = D.dend;
    D.free_back = 0;
    if (D.dend >= 2) {
        const uint32_t B = D.back[D.dend - 1];
        D.free_back = B;
        for (int p = D.dend - 1; p >= 1; --p) {
            if (D.back[p] != B || (B >> p & 1u))
                break;
            if (p < D.dend - 1 && !(D.sym[p + 1] >> p & 1u))
                break;
            D.free_from = p;
        }
    }
    // Rows the DFS reads: those of the positions that are back edges of a
    // later position. When that is position 1 alone, only the rows of the
    // level-1 candidates are built.
    uint32_t read = 0;
    for (int p = 2; p < D.dend; ++p)
        read |= D.back[p];
    D.rows_needed = read == 0 ? 0 : (read == 2u ? 1 : 2);
    D.central = P.central;
    for (int p = 1; p < qn; ++p) {
        for (int e = P.qedge_ptr[p]; e < P.qedge_ptr[p + 1]; ++e)
            if (P.qedge[e] == 0)
                D.adj0 |= 1u << p;
        for (int t = P.sym_ptr[p]; t < P.sym_ptr[p + 1]; ++t)
            if (P.sym[t] == 0)
                D.sym0 |= 1u << p;
    }
    // The 4-wheel: positions 1-4 a 4-cycle around the root. When its chain
    // puts every other position after x1 and x1's two cycle neighbours in
    // order (no other constraint, none against the root at position 1), x1 is
    // the cycle's first vertex and the completions of (x1, opposite vertex c)
    // are C(|row(x1) & row(c) above x1|, 2); the kernels sum that per pair.
    // The reference's chain takes this form under the labellings of the
    // 4-wheel seen so far (x2 ~ x1 ~ x4, or x2 ~ x1 ~ x3).
    D.wheel4 = 0;
    if (qn == 5 && D.dend == 5 && P.central && D.pos1_after_root == 0) {
        uint32_t adj[5] = {0, 0, 0, 0, 0};
        for (int p = 2; p <= 4; ++p)
            for (int q = 1; q < p; ++q)
                if (D.back[p] >> q & 1u) {
                    adj[p] |= 1u << q;
                    adj[q] |= 1u << p;
                }
        bool cycle = true; // four vertices of degree 2: a 4-cycle
        for (int p = 1; p <= 4; ++p)
            cycle = cycle && __builtin_popcount(adj[p]) == 2;
        if (cycle) {
            const int n1 = __builtin_ctz(adj[1]), n2 = 31 - __builtin_clz(adj[1]);
            const int o = 2 + 3 + 4 - n1 - n2;
            D.wheel4 = (D.sym[n1] == 0x2u && D.sym[o] == 0x2u && D.sym[n2] == (0x2u | 1u << n1)) ? 1 : 0;
        }
    }
    P.wheel4 = D.wheel4;
    // Neighbourhood statistics: a five-vertex central query at full depth is
    // a cone over H = positions 1-4. The forms below are those whose count at
    // a root is a sum of per-vertex and per-edge terms of G[N(root)]; the
    // other universal vertices of H (paw: its degree-3 vertex; diamond: its
    // two) must follow the root as the chain demands, so that the count at a
    // root is the walk's count at that root and the tiers can be mixed.
    D.nbhd = kNbNone;
    if (qn == 5 && D.dend == 5 && P.central && !D.wheel4) {
        uint32_t adj[5] = {0, 0, 0, 0, 0};
        int edges = 0;
        for (int p = 2; p <= 4; ++p)
            for (int q = 1; q < p; ++q)
                if (D.back[p] >> q & 1u) {
                    adj[p] |= 1u << q;
                    adj[q] |= 1u << p;
                    ++edges;
                }
        int deg[4], hub = -1, hubs = 0;
        for (int p = 1; p <= 4; ++p) {
            deg[p - 1] = __builtin_popcount(adj[p]);
            if (deg[p - 1] == 3) {
                ++hubs;
                if (hub < 0)
                    hub = p;
            }
        }
        std::sort(deg, deg + 4);
        auto seq = [&](int a, int b, int c, int d) { return deg[0] == a && deg[1] == b && deg[2] == c && deg[3] == d; };
        // position p must follow the root: position 1 through the split,
        // later ones through the chain from position 1
        auto after_root = [&](int p) { return D.pos1_after_root && (p == 1 || (after[p] >> 1 & 1u)); };
        bool universal_after = true;
        for (int p = 1; p <= 4; ++p)
            if (__builtin_popcount(adj[p]) == 3)
                universal_after = universal_after && after_root(p);
        if (edges == 2 && seq(0, 1, 1, 2) && !D.pos1_after_root)
            D.nbhd = kNbWedgeIso;
        else if (edges == 2 && seq(1, 1, 1, 1) && !D.pos1_after_root)
            D.nbhd = kNbTwoEdges;
        else if (edges == 3 && seq(0, 2, 2, 2) && !D.pos1_after_root)
            D.nbhd = kNbTriIso;
        else if (edges == 3 && seq(1, 1, 2, 2) && !D.pos1_after_root)
            D.nbhd = kNbPath4;
        else if (edges == 4 && seq(1, 2, 2, 3) && hubs == 1 && universal_after)
            D.nbhd = kNbPaw;
        else if (edges == 5 && seq(2, 2, 3, 3) && hubs == 2 && universal_after)
            D.nbhd = kNbDiamond;
    }
    if (D.nbhd)
        D.rows_needed = 2; // the statistics read every row of the neighbourhood
    P.nbhd = D.nbhd;
    out->info = P;
    out->dev = D;
    return BEEP_OK;
}

} // namespace beep
