"""Named query patterns, as .mtx-style directed edge lists (0-based, both
directions listed, as README.md:55-64 of the reference shows for the
triangle). The patterns in NAMED have a central vertex adjacent to all
others, which the reference requires (README.md:51-53); those in
NON_CENTRAL do not and are counted by the library's list walker."""
from __future__ import annotations

import itertools


def _undirected(pairs):
    out = []
    for a, b in pairs:
        out.append((a, b))
        out.append((b, a))
    out.sort()
    return out


# The reference README's triangle query file (README.md:55-64).
TRIANGLE = [(0, 1), (0, 2), (1, 0), (1, 2), (2, 0), (2, 1)]
# K4 minus one edge; vertices 0 and 1 are adjacent to all others.
DIAMOND = _undirected([(0, 1), (0, 2), (0, 3), (1, 2), (1, 3)])
K4 = _undirected([(a, b) for a, b in itertools.combinations(range(4), 2)])
# Triangle with a pendant vertex on vertex 0 (the "paw").
TAILED_TRIANGLE = _undirected([(0, 1), (0, 2), (0, 3), (1, 2)])
# Hub 0 plus the 4-cycle 1-2-3-4-1.
W5 = _undirected([(0, 1), (0, 2), (0, 3), (0, 4), (1, 2), (2, 3), (3, 4), (4, 1)])
K5 = _undirected([(a, b) for a, b in itertools.combinations(range(5), 2)])
# Star with three leaves (central vertex 0).
CLAW = _undirected([(0, 1), (0, 2), (0, 3)])
# Hub 0 plus a path on 2 vertices (a "wedge" with apex 0 is CLAW minus a leaf).
WEDGE = _undirected([(0, 1), (0, 2)])

# Queries without a central vertex.
PATH4 = _undirected([(0, 1), (1, 2), (2, 3)])
CYCLE4 = _undirected([(0, 1), (1, 2), (2, 3), (3, 0)])
PATH5 = _undirected([(0, 1), (1, 2), (2, 3), (3, 4)])
CYCLE5 = _undirected([(0, 1), (1, 2), (2, 3), (3, 4), (4, 0)])
# Triangle 0-1-2 with pendants on 1 and 2.
BULL = _undirected([(0, 1), (0, 2), (1, 2), (1, 3), (2, 4)])
# 4-cycle 0-1-2-3 with a roof vertex 4 on the edge 0-1.
HOUSE = _undirected([(0, 1), (1, 2), (2, 3), (3, 0), (0, 4), (1, 4)])
# Complete bipartite K(2,3).
K23 = _undirected([(a, b) for a in (0, 1) for b in (2, 3, 4)])

NON_CENTRAL = {
    "path4": PATH4,
    "cycle4": CYCLE4,
    "path5": PATH5,
    "cycle5": CYCLE5,
    "bull": BULL,
    "house": HOUSE,
    "k23": K23,
}

NAMED = {
    "triangle": TRIANGLE,
    "diamond": DIAMOND,
    "k4": K4,
    "tailed_triangle": TAILED_TRIANGLE,
    "w5": W5,
    "k5": K5,
    "claw": CLAW,
}


def _canon(n, edges):
    """Canonical form of a small graph: the lexicographically least sorted
    edge tuple over all vertex permutations."""
    best = None
    for perm in itertools.permutations(range(n)):
        e = tuple(sorted(tuple(sorted((perm[a], perm[b]))) for a, b in edges))
        if best is None or e < best:
            best = e
    return best


def central_patterns(k: int):
    """All connected k-vertex patterns with a universal vertex, up to
    isomorphism: the cone over each graph on k-1 vertices. There are 4 for
    k = 4 and 11 for k = 5 (15 in total)."""
    m = k - 1
    pairs = list(itertools.combinations(range(m), 2))
    seen = set()
    out = []
    for mask in range(1 << len(pairs)):
        h = [pairs[i] for i in range(len(pairs)) if mask >> i & 1]
        c = _canon(m, h)
        if c in seen:
            continue
        seen.add(c)
        cone = [(0, a + 1) for a in range(m)] + [(a + 1, b + 1) for a, b in c]
        out.append(_undirected(cone))
    out.sort(key=lambda e: (len(e), e))
    return out


def to_mtx(edges) -> str:
    """The .mtx text the reference reads (header 'n n m', then 'row col')."""
    n = max(max(a, b) for a, b in edges) + 1
    lines = [f"{n} {n} {len(edges)}"] + [f"{a} {b}" for a, b in edges]
    return "\n".join(lines) + "\n"
