"""Batched counting: many (graph, pattern, mode) pairs in one set of launches,
captured into a CUDA graph and replayed. Every count must equal the plain
per-pair count and the oracle."""
import numpy as np
import pytest

import beep_b200 as B
from beep_b200 import patterns as P
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


def graphs():
    return [
        B.gen_chung_lu(1 << 10, 8.0, 2.1, 13),
        B.gen_chung_lu(1 << 11, 10.0, 2.1, 14),
        B.gen_rmat(11, 8, 0.57, 0.19, 0.19, 3),
        B.gen_erdos_renyi(600, 0.03, 4),
    ]


def test_batch_matches_plain_and_oracle(ctx):
    pats = P.central_patterns(4) + P.central_patterns(5) + [P.TRIANGLE]
    gs = [(rp, col, B.Graph.from_csr(ctx, rp, col)) for rp, col in graphs()]
    batch = B.Batch(ctx)
    want = []
    for rp, col, g in gs:
        for q in pats:
            for mode in (B.SGM, B.SGC):
                batch.add(g, q, mode)
                want.append(O.count(rp, col, q, sgc=(mode == B.SGC), apply_root_cap=False)["count"])
    assert len(batch) == len(want)
    got1 = batch.run()                    # plans, captures the CUDA graph, replays it
    got2 = batch.run()                    # replays again: counters start at zero
    got3 = batch.run(B.OPT_NO_GRAPH)      # same plan, launched directly
    assert got1 == want
    assert got2 == want
    assert got3 == want
    # plain per-pair counts agree
    i = 0
    for rp, col, g in gs:
        for q in pats[:4]:
            for mode in (B.SGM, B.SGC):
                assert B.count(g, q, mode) == want[i + pats.index(q) * 2 + (mode == B.SGC)]
        i += len(pats) * 2
    batch.close()
    for _, _, g in gs:
        g.close()


def test_batch_mixed_depths_and_large_roots(ctx):
    # a hub of degree 1500 (large tier) next to small graphs, K = 3..5
    rng = np.random.default_rng(7)
    n = 1501
    adj = [set() for _ in range(n)]
    for i in range(1, n):
        adj[0].add(i)
        adj[i].add(0)
    for a, b in zip(rng.integers(1, n, 12000).tolist(), rng.integers(1, n, 12000).tolist()):
        if a != b:
            adj[a].add(b)
            adj[b].add(a)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(x) for x in adj])
    col = np.array([w for x in adj for w in sorted(x)], np.int32)
    g1 = B.Graph.from_csr(ctx, rp, col)
    rp2, col2 = B.gen_erdos_renyi(300, 0.05, 9)
    g2 = B.Graph.from_csr(ctx, rp2, col2)
    batch = B.Batch(ctx)
    want = []
    for (r, c, g) in [(rp, col, g1), (rp2, col2, g2)]:
        for name in ["triangle", "diamond", "k4", "tailed_triangle", "w5", "k5", "claw"]:
            batch.add(g, P.NAMED[name], B.SGM)
            want.append(O.count(r, c, P.NAMED[name], apply_root_cap=False)["count"])
    got, st = batch.run(stats=True)
    assert got == want
    assert st["roots_large"] >= 1
    assert batch.run() == want
    batch.close()
    g1.close()
    g2.close()


def test_tier_limits_and_autotune_keep_counts(ctx):
    """Counts do not depend on which tier a root runs in: every limit set the
    autotuner can pick, and the one it picks, give the same counts."""
    gs = [(rp, col, B.Graph.from_csr(ctx, rp, col)) for rp, col in graphs()[:3]]
    pats = [P.TRIANGLE, P.DIAMOND, P.K4, P.W5, P.NAMED["tailed_triangle"]]
    batch = B.Batch(ctx)
    for _, _, g in gs:
        for q in pats:
            batch.add(g, q, B.SGM)
    base = batch.run()
    for tiers in [dict(tiny_max=0, small_max=32, med_a_max=128, med_max=512),
                  dict(tiny_max=8, small_max=64, med_a_max=256, med_max=512),
                  dict(tiny_max=16, small_max=32, med_a_max=256, med_max=1024)]:
        batch.set_tiers(tiers)
        assert batch.run() == base, tiers
    best = batch.autotune()
    assert best["small_max"] in (32, 64) and best["count_ms"] > 0
    assert batch.run() == base
    assert batch.run(B.OPT_NO_GRAPH) == base
    batch.close()
    for _, _, g in gs:
        g.close()


def test_batch_with_hub_roots_equals_plain_loop(ctx):
    """A small slice of the batched workload whose graphs have hubs above
    degree 1,024: every large-tier kernel (walks with donation, the 4-wheel,
    the neighbourhood statistics) runs in one plan over all 15 central
    patterns, and each count equals the same pair counted alone. The plain
    counts in between plan smaller launches; the captured replay after them
    still runs the batch's own (shared memory limits only grow)."""
    gs = [B.gen_chung_lu(1 << 14, 32.0, 2.1, 13000 + i) for i in range(3)]
    assert all(np.diff(rp).max() > 1024 for rp, _ in gs)
    graphs = [B.Graph.from_csr(ctx, rp, col) for rp, col in gs]
    pats = P.central_patterns(4) + P.central_patterns(5)
    batch = B.Batch(ctx)
    for g in graphs:
        for q in pats:
            batch.add(g, q)
    got, st = batch.run(B.OPT_NO_GRAPH, stats=True)
    assert st["roots_large"] > 0
    plain = [B.count(g, q) for g in graphs for q in pats]
    assert got == plain
    assert batch.run() == plain  # the captured graph
    batch.close()
    for g in graphs:
        g.close()
