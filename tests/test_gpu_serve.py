"""Serving with continuous batching: requests submitted while earlier ones run
are admitted into later batches; every result must equal the same request
run alone (exact counts; enumerations return min(k, count) distinct valid
matches)."""
import time

import numpy as np
import pytest

import beep_b200 as B
from beep_b200 import patterns as P
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

NAMES = ["triangle", "diamond", "k4", "tailed_triangle", "w5", "k5"]


def test_serve_results_match_alone(ctx):
    specs = [B.gen_chung_lu(1 << 10, 8.0, 2.1, 21), B.gen_chung_lu(1 << 11, 12.0, 2.1, 22),
             B.gen_rmat(11, 8, 0.57, 0.19, 0.19, 23)]
    graphs = [B.Graph.from_csr(ctx, rp, col) for rp, col in specs]
    queries = {n: B.Query.from_edges(P.NAMED[n]) for n in NAMES}
    alone = {(gi, n): B.count(g, queries[n]) for gi, g in enumerate(graphs) for n in NAMES}
    full_sets = {}
    srv = B.Server(ctx, max_batch=8, streams=3)
    gids = [srv.add_graph(g) for g in graphs]
    rng = np.random.default_rng(17)
    reqs = []
    for i in range(120):
        gi = int(rng.integers(0, len(graphs)))
        n = NAMES[int(rng.integers(0, len(NAMES)))]
        k = 200 if rng.random() < 0.2 else 0
        reqs.append((srv.submit(gids[gi], queries[n], B.SGM, k), gi, n, k))
        if i % 10 == 0:
            time.sleep(0.002)  # arrivals spread over time: later ones join later batches
    for rid, gi, n, k in reqs:
        res = srv.wait(rid, k)
        assert res["count"] == alone[(gi, n)], (gi, n)
        if k:
            tup = res["tuples"]
            assert len(tup) == min(k, res["count"])
            assert len(set(map(tuple, tup.tolist()))) == len(tup)
            if (gi, n) not in full_sets:
                rp, col = specs[gi]
                full_sets[(gi, n)] = set(map(tuple, O.enumerate_matches(rp, col, P.NAMED[n]).tolist()))
            assert set(map(tuple, tup.tolist())) <= full_sets[(gi, n)]
    st = srv.stats()
    assert st["requests"] == len(reqs)
    assert st["batches"] >= 2
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    srv.close()
    for g in graphs:
        g.close()


def test_serve_sgc_and_errors(ctx):
    rp, col = B.gen_erdos_renyi(300, 0.05, 5)
    g = B.Graph.from_csr(ctx, rp, col)
    srv = B.Server(ctx)
    gid = srv.add_graph(g)
    rid = srv.submit(gid, P.DIAMOND, B.SGC)
    assert srv.wait(rid)["count"] == B.count(g, P.DIAMOND, B.SGC)
    with pytest.raises(B.BeepError):
        srv.submit(gid + 5, P.TRIANGLE)
    srv.drain()
    srv.close()
    g.close()


def test_serve_admission_back_pressure_and_refusal(ctx):
    """A budget that holds one small request at a time: requests queue behind
    the batch in flight instead of running out of memory, each result is
    still exact, and a request whose estimate exceeds the whole budget is
    refused with BEEP_ERR_OUT_OF_MEMORY."""
    import torch

    small_rp, small_col = B.gen_erdos_renyi(300, 0.05, 5)
    hub_rp, hub_col = B.gen_chung_lu(1 << 14, 32.0, 2.1, 9)  # hubs above degree 1024: a large-tier arena
    assert np.diff(hub_rp).max() > 1024
    small = B.Graph.from_csr(ctx, small_rp, small_col)
    hub = B.Graph.from_csr(ctx, hub_rp, hub_col)
    want = B.count(small, P.TRIANGLE)
    n, m = len(small_rp) - 1, len(small_col)
    one = n * 64 + m * 4  # the estimate of one count request on the small graph
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    srv = B.Server(ctx, max_batch=8, streams=4, hbm_reserve_bytes=free - int(1.5 * one))
    g_small, g_hub = srv.add_graph(small), srv.add_graph(hub)
    st0 = srv.stats()
    assert one <= st0["budget_bytes"] < 2 * one
    big = srv.submit(g_hub, P.TRIANGLE)
    rids = [srv.submit(g_small, P.TRIANGLE) for _ in range(20)]
    with pytest.raises(B.BeepError) as e:
        srv.wait(big)
    assert e.value.status == B.ERR_OUT_OF_MEMORY
    for rid in rids:
        assert srv.wait(rid)["count"] == want
    st = srv.stats()
    assert st["refused"] == 1
    assert st["requests"] == 20
    assert st["max_inflight_bytes"] <= st["budget_bytes"]
    assert st["batches"] == 20  # one request per batch, one batch at a time
    srv.close()
    small.close()
    hub.close()
