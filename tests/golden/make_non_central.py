"""Generate tests/golden/non_central.json: counts of the queries without a
central vertex (beep_b200.patterns.NON_CENTRAL) on the small seeded graphs of
golden.json, by the oracle's brute force (injective maps / |Aut|), checked
against networkx monomorphism counts where the graph is small.

The reference cannot count these queries (its DFS needs a vertex adjacent to
all others, README.md:51-53), so the brute force is the checker.

Run from the repository root:  python tests/golden/make_non_central.py
"""
from __future__ import annotations

import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import beep_b200 as B  # noqa: E402
from beep_b200 import patterns as P  # noqa: E402
from oracle import pyoracle as O  # noqa: E402

import make_golden as G  # noqa: E402

GRAPHS = ["er_60_p15_s3", "er_200_p05_s4", "cl_300_d12_s5"]


def main():
    out = {"patterns": dict(P.NON_CENTRAL), "graphs": {}}
    for gname in GRAPHS:
        kind, args = G.SMALL[gname]
        rp, col = G.gen(kind, args)
        rec = {"kind": kind, "args": list(args), "counts": {}}
        for pname, q in P.NON_CENTRAL.items():
            c = O.brute_force(rp, col, q)
            if len(rp) - 1 <= 200:
                nxc = G.nx_count(rp, col, q)
                assert c == nxc, (gname, pname, c, nxc)
            rec["counts"][pname] = int(c)
        out["graphs"][gname] = rec
        print(gname, rec["counts"], flush=True)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "non_central.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
