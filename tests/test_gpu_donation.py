"""Work donation of the large tier and its bounded waits.

Warps of the large tier's walk that run out of (root, x1) tasks wait for
donated subtrees; running walks hand over half of their remaining iterations
at shallow levels. Counts must not change whether or not anything is donated
(bit-exact against the oracle), and a wait that can never be served ends the
kernel with BEEP_ERR_TIMEOUT after the context's wait bound, leaving the
context usable."""
import numpy as np
import pytest

import beep_b200 as B
from beep_b200 import patterns as P
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


def roots_over_hubs(nr, nh, p, seed):
    """nr roots joined to every one of nh hubs, and G(nh, p) among the hubs.
    Every hub outranks every root in the ascending degree order, so each
    root's higher-priority neighbours are all nh hubs: nr large-tier roots
    (nh > 1024) whose walks differ with the random hub neighbourhoods."""
    rng = np.random.default_rng(seed)
    iu = np.triu_indices(nh, 1)
    m = rng.random(len(iu[0])) < p
    a, b = nr + iu[0][m], nr + iu[1][m]
    ra, hb = np.repeat(np.arange(nr), nh), nr + np.tile(np.arange(nh), nr)
    s, d = np.concatenate([a, b, ra, hb]), np.concatenate([b, a, hb, ra])
    n = nr + nh
    key = np.unique(s.astype(np.int64) * n + d)
    s, d = key // n, key % n
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, s + 1, 1)
    return np.cumsum(rp).astype(np.int32), d.astype(np.int32)


@pytest.fixture(scope="module")
def graph():
    rp, col = roots_over_hubs(1000, 1050, 0.12, 3)
    exp = {"k4": O.count(rp, col, P.K4, apply_root_cap=False)["count"],
           "k5": O.count_cliques(rp, col, 5),
           "diamond": O.count(rp, col, P.DIAMOND, apply_root_cap=False)["count"]}
    return rp, col, exp


def test_counts_with_donation_match_oracle(ctx, graph):
    rp, col, exp = graph
    g = B.Graph.from_csr(ctx, rp, col)
    donated = 0
    for name in ("k4", "k5", "diamond"):
        c, st = B.count(g, P.NAMED[name], B.SGM, B.OPT_TIMING, stats=True)
        assert c == exp[name], name
        if name != "diamond":
            assert st["roots_large"] >= 1000, (name, st["roots_large"])
        donated += st["donated_tasks"]
    assert donated > 0
    g.close()


def test_donation_off_gives_the_same_counts(ctx, graph):
    """The same pairs in a batch with donation (captured replay too) and with
    the donation threshold at 0 (none): equal counts."""
    rp, col, exp = graph
    g = B.Graph.from_csr(ctx, rp, col)
    names = ["k5", "k4", "diamond"]
    b = B.Batch(ctx)
    for name in names:
        b.add(g, P.NAMED[name])
    want = [exp[n] for n in names]
    got, st = b.run(B.OPT_NO_GRAPH, stats=True)
    assert got == want
    assert st["donated_tasks"] > 0, st["donated_tasks"]
    assert b.run() == want  # the captured CUDA graph replays the donation protocol
    assert b.run() == want
    b.set_tiers({"tiny_max": 8, "small_max": 64, "med_a_max": 256, "med_max": 1024, "donate_min_iters": 0})
    got0, st0 = b.run(B.OPT_NO_GRAPH, stats=True)
    assert got0 == want and st0["donated_tasks"] == 0
    b.close()
    g.close()


def test_wait_that_cannot_be_served_times_out(graph):
    """A phantom donated task that no donor publishes: every waiting warp runs
    out its bound, the call reports BEEP_ERR_TIMEOUT (no trap, no hang), and
    the same context counts correctly afterwards."""
    rp, col, exp = graph
    with B.Context(0) as c:
        c.set_wait_timeout(50.0)
        g = B.Graph.from_csr(c, rp, col)
        with pytest.raises(B.BeepError) as e:
            B.count(g, P.K4, B.SGM, B.OPT_WAIT_STALL_TEST, ctx=c)
        assert e.value.status == B.ERR_TIMEOUT
        assert B.count(g, P.K4, B.SGM, 0, ctx=c) == exp["k4"]
        g.close()
