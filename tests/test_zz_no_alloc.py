"""The allocation-free entry point (beep_count_noalloc), for callers that
cannot let a library call cudaMalloc (device memory owned by their own pool or
caching allocator, or loops that cannot take cudaMalloc's synchronisation).

Its counts are compared with the regular entry point's (exact integer
equality, the tolerance of every count test here) on two calls in a row,
since the shared scratch array keeps the previous call's contents. This file
is named to be collected last; it passes alone in a fresh process and after
the other tests."""
import math

import numpy as np
import pytest

import beep_b200 as B
from beep_b200 import patterns as P

pytestmark = pytest.mark.gpu


def hub_graph(n_leaves, p, seed):
    rng = np.random.default_rng(seed)
    adj = [set() for _ in range(n_leaves + 1)]
    for i in range(1, n_leaves + 1):
        adj[0].add(i)
        adj[i].add(0)
    m = int(p * n_leaves * (n_leaves - 1) / 2)
    for a, b in zip(rng.integers(1, n_leaves + 1, size=m).tolist(), rng.integers(1, n_leaves + 1, size=m).tolist()):
        if a != b:
            adj[a].add(b)
            adj[b].add(a)
    rp = np.zeros(n_leaves + 2, np.int32)
    rp[1:] = np.cumsum([len(x) for x in adj])
    col = np.array([w for x in adj for w in sorted(x)], np.int32)
    return rp, col


CASES = [
    ("er_c1", lambda: B.gen_erdos_renyi(4096, 0.004, 1)),
    ("rmat_12", lambda: B.gen_rmat(12, 8, 0.57, 0.19, 0.19, 1)),
    # a hub of degree 1500: its bitmap lives in the scratch array, not in shared memory
    ("hub_1500", lambda: hub_graph(1500, 0.01, 3)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_count(name, make):
    import torch

    rp, col = make()
    d_rp = torch.from_numpy(np.ascontiguousarray(rp, np.int32)).cuda()
    d_col = torch.from_numpy(np.ascontiguousarray(col, np.int32)).cuda()
    torch.cuda.synchronize()
    n, m = len(rp) - 1, len(col)
    with B.Context(0) as ctx:
        g = B.Graph.from_csr(ctx, rp, col)
        for pname in ["triangle", "diamond", "k4", "tailed_triangle", "w5", "claw"]:
            q = B.Query.from_edges(P.NAMED[pname])
            for mode in (B.SGM, B.SGC):
                if mode == B.SGC and q.plan(B.SGC)["unmat"]:
                    continue
                want = B.count(g, q, mode)
                for call in range(2):
                    got = B.count_noalloc(0, n, m, d_rp.data_ptr(), d_col.data_ptr(), q, mode)
                    assert got == want, (name, pname, mode, call, got, want)
        g.close()


def star(leaves):
    """Vertex 0 joined to vertices 1..leaves (the hub's domain has `leaves` vertices)."""
    rp = np.zeros(leaves + 2, np.int32)
    rp[1] = leaves
    rp[2:] = leaves + np.arange(1, leaves + 1)
    col = np.concatenate([np.arange(1, leaves + 1), np.zeros(leaves)]).astype(np.int32)
    return rp, col


def test_noalloc_domain_limit_boundary():
    """The largest domain whose bitmap fits the scratch array is counted; one
    vertex more is refused before any counting work."""
    import torch

    leaves = B.NOALLOC_MAX_DOMAIN
    rp, col = star(leaves)
    d_rp = torch.from_numpy(rp).cuda()
    d_col = torch.from_numpy(col).cuda()
    torch.cuda.synchronize()
    with B.Context(0) as ctx:
        g = B.Graph.from_csr(ctx, rp, col)
        want = B.count(g, P.CLAW, B.SGM)
        g.close()
    assert want == math.comb(leaves, 3)
    for call in range(2):
        assert B.count_noalloc(0, leaves + 1, len(col), d_rp.data_ptr(), d_col.data_ptr(), P.CLAW, B.SGM) == want
    rp, col = star(leaves + 1)
    d_rp = torch.from_numpy(rp).cuda()
    d_col = torch.from_numpy(col).cuda()
    torch.cuda.synchronize()
    with pytest.raises(B.BeepError) as e:
        B.count_noalloc(0, leaves + 2, len(col), d_rp.data_ptr(), d_col.data_ptr(), P.CLAW, B.SGM)
    assert e.value.status == B.ERR_UNSUPPORTED
    assert "scratch" in str(e.value) and str(B.NOALLOC_MAX_DOMAIN) in str(e.value)


def test_noalloc_rejects_bad_csr():
    """A CSR the caller got wrong is refused by the device-side check before
    any kernel uses an entry as an index: an id at or above n, an unsorted
    row, a self loop, row pointers beyond m."""
    import torch

    rp, col = B.gen_erdos_renyi(200, 0.05, 2)
    n, m = len(rp) - 1, len(col)
    bad_cases = []
    c = col.copy()
    c[rp[5]] = n + 7  # an id out of range
    bad_cases.append((rp, c))
    c = col.copy()
    v = int(np.argmax(np.diff(rp) >= 2))
    c[rp[v]], c[rp[v] + 1] = c[rp[v] + 1], c[rp[v]]  # an unsorted row
    bad_cases.append((rp, c))
    loop = next((u, i) for u in range(n) for i in range(rp[u] + 1, rp[u + 1] - 1) if col[i - 1] < u < col[i + 1])
    c = col.copy()
    c[loop[1]] = loop[0]  # a self loop, the row still strictly increasing
    bad_cases.append((rp, c))
    r = rp.copy()
    r[3] = m + 5  # a row pointer beyond m
    bad_cases.append((r, col))
    for rpb, cb in bad_cases:
        d_rp = torch.from_numpy(np.ascontiguousarray(rpb, np.int32)).cuda()
        d_col = torch.from_numpy(np.ascontiguousarray(cb, np.int32)).cuda()
        torch.cuda.synchronize()
        with pytest.raises(B.BeepError) as e:
            B.count_noalloc(0, n, m, d_rp.data_ptr(), d_col.data_ptr(), P.TRIANGLE, B.SGM)
        assert e.value.status == B.ERR_INVALID_ARG, str(e.value)
    # the check leaves the path usable: a valid CSR right after counts as before
    d_rp = torch.from_numpy(rp).cuda()
    d_col = torch.from_numpy(col).cuda()
    torch.cuda.synchronize()
    with B.Context(0) as ctx:
        g = B.Graph.from_csr(ctx, rp, col)
        want = B.count(g, P.TRIANGLE, B.SGM)
        g.close()
    assert B.count_noalloc(0, n, m, d_rp.data_ptr(), d_col.data_ptr(), P.TRIANGLE, B.SGM) == want


def test_noalloc_refuses_oversized_domain():
    import torch

    leaves = 30000  # a star: the hub's domain is 30000 > BEEP_NOALLOC_MAX_DOMAIN vertices
    rp, col = star(leaves)
    d_rp = torch.from_numpy(rp).cuda()
    d_col = torch.from_numpy(col).cuda()
    torch.cuda.synchronize()
    with pytest.raises(B.BeepError) as e:
        B.count_noalloc(0, leaves + 1, len(col), d_rp.data_ptr(), d_col.data_ptr(), P.CLAW, B.SGM)
    assert e.value.status == B.ERR_UNSUPPORTED
    assert "scratch" in str(e.value)
    # sgc whose last level is unmaterialised is refused too
    rp2, col2 = B.gen_erdos_renyi(200, 0.05, 2)
    d2 = torch.from_numpy(rp2).cuda()
    c2 = torch.from_numpy(col2).cuda()
    torch.cuda.synchronize()
    with pytest.raises(B.BeepError) as e:
        B.count_noalloc(0, len(rp2) - 1, len(col2), d2.data_ptr(), c2.data_ptr(), P.DIAMOND, B.SGC)
    assert e.value.status == B.ERR_UNSUPPORTED
