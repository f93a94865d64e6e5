"""The large tier counts the 4-wheel per (x1, x3) pair in closed form
(k_large_wheel in beep_b200/csrc/count.cu): under the reference's chain for
the 4-wheel (x2, x3, x4 > x1 and x4 > x2), the completions of (x1, x3) are
C(|row(x1) & row(x3) above x1|, 2), summed over the x3 > x1 reached from a
neighbour of x1 above x1. This restates that sum in Python, over every root's
neighbourhood in the priority order of the plan, and checks it against the
oracle's walk of every match. CPU only."""
from math import comb

import pytest

import beep_b200 as B
from beep_b200 import patterns as P
from oracle import pyoracle as O


def wheel_pairs_count(rp, col):
    n = len(rp) - 1
    adj = [set(col[rp[v]:rp[v + 1]].tolist()) for v in range(n)]
    # descending degree, ties by id: the 4-wheel plan's order (first_sym_level 3)
    prio = sorted(range(n), key=lambda v: (-len(adj[v]), v))
    rank = {v: i for i, v in enumerate(prio)}
    total = 0
    for r in range(n):
        if len(adj[r]) < 4:
            continue
        A = sorted(adj[r], key=lambda v: rank[v])
        idx = {v: i for i, v in enumerate(A)}
        rows = [{idx[w] for w in adj[v] if w in idx} for v in A]
        for a in range(len(A)):
            U = set()
            for b in rows[a]:
                if b > a:
                    U |= {c for c in rows[b] if c > a}
            for c in U:
                total += comb(sum(1 for x in rows[a] & rows[c] if x > a), 2)
    return total


def test_plan_is_the_closed_form_chain():
    pl = B.Query.from_edges(P.W5).plan()
    # x2 after x1; x3 after x1; x4 after x1 and x2 (positions 2, 3, 4)
    sym = {p: sorted(pl["sym"][pl["sym_ptr"][p]:pl["sym_ptr"][p + 1]]) for p in range(5)}
    assert sym == {0: [], 1: [], 2: [1], 3: [1], 4: [1, 2]}
    assert pl["first_sym_level"] == 3 and pl["unmat"] == 0


@pytest.mark.parametrize("gen,args", [
    ("er", (120, 0.12, 1)), ("er", (150, 0.1, 2)), ("cl", (300, 12.0, 2.1, 3)), ("rmat", (9, 8, 0.57, 0.19, 0.19, 4)),
])
def test_closed_form_equals_the_walk(built, gen, args):
    rp, col = {"er": B.gen_erdos_renyi, "cl": B.gen_chung_lu, "rmat": B.gen_rmat}[gen](*args)
    exp = O.count(rp, col, P.W5, apply_root_cap=False)["count"]
    assert wheel_pairs_count(rp, col) == exp
    # the oracle walks the other form of the chain (another labelling) to the same count
    w5b = P.central_patterns(5)[8]
    assert sorted(w5b) != sorted(P.W5)
    assert O.count(rp, col, w5b, apply_root_cap=False)["count"] == exp
