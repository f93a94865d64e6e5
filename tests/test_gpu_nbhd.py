"""Neighbourhood statistics of the large tier: six five-vertex central
queries whose count at a root follows from degrees, edges and per-edge common
neighbours of the root's neighbourhood graph. Their counts must equal the
oracle's (bit-exact) and the walk's (the same call with BEEP_OPT_NO_NBHD),
under every labelling of the query."""
import random

import numpy as np
import pytest

import beep_b200 as B
from beep_b200 import patterns as P
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

FORMS = {6: 1, 7: 2, 9: 3, 10: 4, 11: 5, 13: 6}  # central pattern index -> beep_plan_info.nbhd


def csr_from_pairs(n, pairs):
    adj = [set() for _ in range(n)]
    for a, b in pairs:
        if a != b:
            adj[a].add(b)
            adj[b].add(a)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(x) for x in adj])
    col = np.array([w for x in adj for w in sorted(x)], np.int32)
    return rp, col


def hubs(n_leaves, p, seed, n_hubs=2):
    """n_hubs hubs over n_leaves leaves with G(n_leaves, p) among the leaves:
    the hubs are large roots (degree > 1024), the rest small."""
    rng = np.random.default_rng(seed)
    pairs = [(h, n_hubs + i) for h in range(n_hubs) for i in range(n_leaves)]
    m = int(p * n_leaves * (n_leaves - 1) / 2)
    a = rng.integers(n_hubs, n_hubs + n_leaves, size=m)
    b = rng.integers(n_hubs, n_hubs + n_leaves, size=m)
    pairs += list(zip(a.tolist(), b.tolist()))
    return csr_from_pairs(n_hubs + n_leaves, pairs)


def roots_over_hubs(nr, nh, p, seed):
    """nr roots joined to every one of nh hubs, and G(nh, p) among the hubs:
    every hub outranks every root, so each root's later neighbours are all nh
    hubs -- large roots for the forms whose other universal vertices must
    follow the root (paw, diamond)."""
    rng = np.random.default_rng(seed)
    iu = np.triu_indices(nh, 1)
    m = rng.random(len(iu[0])) < p
    pairs = list(zip((nr + iu[0][m]).tolist(), (nr + iu[1][m]).tolist()))
    pairs += [(r, nr + h) for r in range(nr) for h in range(nh)]
    return csr_from_pairs(nr + nh, pairs)


def relabel(q, seed):
    perm = list(range(5))
    random.Random(seed).shuffle(perm)
    return sorted({(perm[a], perm[b]) for a, b in q})


def test_forms_are_detected():
    pats = P.central_patterns(4) + P.central_patterns(5)
    for i, q in enumerate(pats):
        for seed in range(4):
            assert B.Query.from_edges(relabel(q, seed) if len(q) >= 8 and i >= 4 else q).plan()["nbhd"] == \
                FORMS.get(i, 0), i


@pytest.mark.parametrize("graph", ["hubs", "roots_over_hubs"])
def test_forms_match_oracle(ctx, graph):
    """Forms whose root has no constraint (wedge, two edges, triangle, path)
    on hubs of degree 1,400; forms whose other universal vertices follow the
    root (paw, diamond) on 1,100 roots of degree 1,100 below higher hubs."""
    if graph == "hubs":
        rp, col = hubs(1400, 0.012, 3)
        forms = [6, 7, 9, 10]
    else:
        rp, col = roots_over_hubs(1100, 1100, 0.05, 4)
        forms = [11, 13]
    g = B.Graph.from_csr(ctx, rp, col)
    pats = P.central_patterns(4) + P.central_patterns(5)
    for i in forms:
        for seed in (0, 1):
            q = relabel(pats[i], seed)
            exp = O.count(rp, col, q, apply_root_cap=False)["count"]
            c, st = B.count(g, q, B.SGM, B.OPT_TIMING, stats=True)
            assert c == exp, (i, seed)
            assert st["roots_large"] >= 1, (i, st["roots_large"])
            assert B.count(g, q, B.SGM, B.OPT_NO_NBHD) == exp, (i, seed)
    g.close()


def test_forms_with_word_lists_match_the_walk(ctx):
    """Hubs of degree 9,000: rows of 282 words carry non-zero-word lists. The
    batch also holds the 4-wheel, whose kernel shares the per-warp scratch
    with the statistics kernel and runs after it; each count equals the same
    pair counted alone."""
    rp, col = hubs(9000, 0.0012, 5, n_hubs=3)
    g = B.Graph.from_csr(ctx, rp, col)
    pats = P.central_patterns(4) + P.central_patterns(5)
    idx = list(FORMS) + [12]
    b = B.Batch(ctx)
    for i in idx:
        b.add(g, pats[i])
    got = b.run()
    walk = b.run(B.OPT_NO_NBHD | B.OPT_NO_GRAPH)
    alone = [B.count(g, pats[i]) for i in idx]
    assert got == walk == alone
    assert all(c > 0 for c in got)
    b.close()
    g.close()


@pytest.mark.parametrize("graph", ["hubs_thread", "hubs_warp", "roots_thread", "roots_warp"])
def test_forms_in_the_medium_tier(ctx, graph):
    """The same forms counted by the medium tier from its shared-memory rows:
    domains of 65-256 vertices (thread sub-tier, rows of 4 x 64 bits) and of
    257-1,024 (warp sub-tier). Each count equals the oracle's and the walk's,
    and the medium tier took roots."""
    if graph == "hubs_thread":
        rp, col = hubs(200, 0.06, 7, n_hubs=3)
        forms = [6, 7, 9, 10]
    elif graph == "hubs_warp":
        rp, col = hubs(700, 0.02, 8, n_hubs=2)
        forms = [6, 7, 9, 10]
    elif graph == "roots_thread":
        rp, col = roots_over_hubs(300, 200, 0.12, 9)
        forms = [11, 13]
    else:
        rp, col = roots_over_hubs(120, 600, 0.04, 10)
        forms = [11, 13]
    g = B.Graph.from_csr(ctx, rp, col)
    pats = P.central_patterns(4) + P.central_patterns(5)
    for i in forms:
        for seed in (0, 2):
            q = relabel(pats[i], seed)
            exp = O.count(rp, col, q, apply_root_cap=False)["count"]
            c, st = B.count(g, q, B.SGM, B.OPT_TIMING, stats=True)
            assert c == exp, (graph, i, seed)
            assert st["roots_medium"] >= 1 and st["roots_large"] == 0, (graph, i, st["roots_medium"])
            assert B.count(g, q, B.SGM, B.OPT_NO_NBHD) == exp, (graph, i, seed)
    g.close()
