"""Queries without a central vertex (paths, cycles, the bull, the house,
K(2,3)): counted by the list walker. The reference cannot count them
(README.md:51-53), so the checker is the oracle's brute force
(tests/golden/non_central.json, cross-checked with networkx there)."""
import itertools
import json
import math
import os

import numpy as np
import pytest

import beep_b200 as B
from beep_b200 import patterns as P
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu
GENS = {"er": B.gen_erdos_renyi, "cl": B.gen_chung_lu, "rmat": B.gen_rmat}


def load():
    with open(os.path.join(os.path.dirname(__file__), "golden", "non_central.json")) as f:
        return json.load(f)


def test_counts_match_brute_force(ctx):
    gold = load()
    for gname, rec in gold["graphs"].items():
        rp, col = GENS[rec["kind"]](*rec["args"])
        g = B.Graph.from_csr(ctx, rp, col)
        for pname, want in rec["counts"].items():
            assert B.count(g, P.NON_CENTRAL[pname], B.SGM) == want, (gname, pname)
        g.close()


@pytest.mark.parametrize("n", [8, 30])
def test_complete_graph_closed_forms(ctx, n):
    pairs = list(itertools.combinations(range(n), 2))
    adj = [set() for _ in range(n)]
    for a, b in pairs:
        adj[a].add(b)
        adj[b].add(a)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(s) for s in adj])
    col = np.array([w for s in adj for w in sorted(s)], np.int32)
    g = B.Graph.from_csr(ctx, rp, col)
    want = {"path4": 12 * math.comb(n, 4), "cycle4": 3 * math.comb(n, 4), "path5": 60 * math.comb(n, 5),
            "cycle5": 12 * math.comb(n, 5), "k23": 10 * math.comb(n, 5)}
    for name, w in want.items():
        assert B.count(g, P.NON_CENTRAL[name], B.SGM) == w, name
    g.close()


def test_enumeration_and_batch(ctx):
    rp, col = B.gen_chung_lu(300, 6.0, 2.1, 9)
    g = B.Graph.from_csr(ctx, rp, col)
    edges = set()
    for v in range(len(rp) - 1):
        for w in col[rp[v]:rp[v + 1]]:
            edges.add((v, int(w)))
    for name in ["cycle4", "house"]:
        q = P.NON_CENTRAL[name]
        total = B.count(g, q, B.SGM)
        assert total == O.brute_force(rp, col, q)
        tup, tot = B.enumerate_matches(g, q, 50, ctx=ctx)
        n_out = len(tup)
        assert tot == total and n_out == min(50, total)
        assert len({tuple(t) for t in tup.tolist()}) == n_out
        for t in tup.tolist():
            assert len(set(t)) == len(t)
            for a, b in q:
                assert (t[a], t[b]) in edges
    # central and non-central pairs in one planned call
    b = B.Batch(ctx)
    qs = [P.K4, P.NON_CENTRAL["cycle4"], P.DIAMOND, P.NON_CENTRAL["path5"]]
    for q in qs:
        b.add(g, q, B.SGM)
    got = b.run()
    assert got == [B.count(g, q, B.SGM) for q in qs]
    assert got[1] == O.brute_force(rp, col, qs[1]) and got[3] == O.brute_force(rp, col, qs[3])
    b.close()
    g.close()


def test_sgc_prefix_needs_central_query(ctx):
    with pytest.raises(B.BeepError) as e:
        B.Query.from_edges(P.NON_CENTRAL["path4"]).plan(B.SGC)
    assert e.value.status == B.ERR_UNSUPPORTED
    # cycle4's last position is adjacent to the one before: sgc counts full matches
    rp, col = B.gen_erdos_renyi(80, 0.1, 2)
    g = B.Graph.from_csr(ctx, rp, col)
    assert B.count(g, P.NON_CENTRAL["cycle4"], B.SGC) == O.brute_force(rp, col, P.NON_CENTRAL["cycle4"])
    g.close()
