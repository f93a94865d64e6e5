"""Counts at or above BEEP_COUNT_LIMIT (2^64 - 2^52) are reported as
overflow, never as a residue mod 2^64; counts just below it stay exact.

A star with L leaves has C(L, 4) matches of the 4-star (hub + 4 leaves):
C(140000, 4) ~ 1.60e19 lies between 2^63 and the limit, C(145500, 4) ~ 1.87e19
is above 2^64."""
import math

import numpy as np
import pytest

import beep_b200 as B
from beep_b200 import patterns as P

pytestmark = pytest.mark.gpu

STAR4 = P.central_patterns(5)[0]  # the cone over 4 isolated vertices


def star(leaves):
    rp = np.zeros(leaves + 2, np.int64)
    rp[1] = leaves
    rp[2:] = leaves + np.arange(1, leaves + 1)
    col = np.concatenate([np.arange(1, leaves + 1), np.zeros(leaves)])
    return rp.astype(np.int32), col.astype(np.int32)


def test_star_pattern_is_the_4_star():
    edges = {tuple(sorted(e)) for e in STAR4}
    assert edges == {(0, 1), (0, 2), (0, 3), (0, 4)}


def test_count_below_limit_is_exact(ctx):
    rp, col = star(140000)
    exp = math.comb(140000, 4)
    assert 2 ** 63 < exp < B.COUNT_LIMIT
    g = B.Graph.from_csr(ctx, rp, col)
    assert B.count(g, STAR4) == exp
    g.close()


def test_count_above_limit_is_refused(ctx):
    rp, col = star(145500)
    assert math.comb(145500, 4) >= 2 ** 64
    g = B.Graph.from_csr(ctx, rp, col)
    with pytest.raises(B.BeepError) as e:
        B.count(g, STAR4)
    assert e.value.status == B.ERR_OVERFLOW
    # the 3-star (claw) on the same graph is far below the limit and exact
    assert B.count(g, P.CLAW) == math.comb(145500, 3)
    g.close()


def test_batch_flags_only_the_overflowing_pair(ctx):
    small = B.Graph.from_csr(ctx, *star(140000))
    big = B.Graph.from_csr(ctx, *star(145500))
    b = B.Batch(ctx)
    b.add(small, STAR4)
    b.add(big, STAR4)
    b.add(big, P.CLAW)
    for opts in (0, B.OPT_NO_GRAPH):
        counts, st = b.run(opts, stats=True)
        assert counts == [math.comb(140000, 4), B.COUNT_OVERFLOW, math.comb(145500, 3)]
        assert st["overflow_pairs"] == 1
    b.close()
    small.close()
    big.close()
