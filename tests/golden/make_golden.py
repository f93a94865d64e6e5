"""Generate tests/golden/golden.json: match counts for seeded synthetic graphs,
computed by the CPU oracle (oracle/), cross-checked here by brute force and
networkx monomorphism counts on the small graphs.

Run from the repository root:  python tests/golden/make_golden.py
Needs the built library (for the generators) and the oracle; networkx is used
only here, not at test time.
"""
from __future__ import annotations

import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import beep_b200 as B  # noqa: E402
from beep_b200 import patterns as P  # noqa: E402
from oracle import pyoracle as O  # noqa: E402

# Small graphs: name -> (generator, args)
SMALL = {
    "er_60_p15_s3": ("er", (60, 0.15, 3)),
    "er_200_p05_s4": ("er", (200, 0.05, 4)),
    "cl_300_d12_s5": ("cl", (300, 12.0, 2.1, 5)),
    "rmat_9_8_s6": ("rmat", (9, 8, 0.57, 0.19, 0.19, 6)),
}
# Seeded full-size inputs of the plain-method workloads.
LARGE = {
    "c1_er_4096_p004_s1": (("er", (4096, 0.004, 1)), ["triangle"]),
    "c2_rmat_20_3_s7": (("rmat", (20, 3, 0.57, 0.19, 0.19, 7)), ["k4", "diamond"]),
}


def gen(kind, args):
    if kind == "er":
        return B.gen_erdos_renyi(*args)
    if kind == "cl":
        return B.gen_chung_lu(*args)
    if kind == "rmat":
        return B.gen_rmat(*args)
    raise ValueError(kind)


def nx_count(rp, col, q):
    import networkx as nx
    from networkx.algorithms import isomorphism as iso

    G = nx.Graph()
    n = len(rp) - 1
    G.add_nodes_from(range(n))
    for v in range(n):
        for e in range(rp[v], rp[v + 1]):
            G.add_edge(v, int(col[e]))
    Q = nx.Graph()
    Q.add_edges_from((a, b) for a, b in q if a != b)
    gm = iso.GraphMatcher(G, Q)
    mono = sum(1 for _ in gm.subgraph_monomorphisms_iter())
    aut = sum(1 for _ in iso.GraphMatcher(Q, Q).isomorphisms_iter())
    return mono // aut


def main():
    out = {"small": {}, "large": {}, "patterns": {}}
    allpat = dict(P.NAMED)
    for i, q in enumerate(P.central_patterns(4)):
        allpat[f"c4_{i}"] = q
    for i, q in enumerate(P.central_patterns(5)):
        allpat[f"c5_{i}"] = q
    out["patterns"] = {k: v for k, v in allpat.items()}
    for gname, (kind, args) in SMALL.items():
        rp, col = gen(kind, args)
        rec = {"kind": kind, "args": list(args), "n": int(len(rp) - 1), "m": int(len(col)), "counts": {}}
        for pname, q in allpat.items():
            sgm = O.count(rp, col, q, sgc=False, apply_root_cap=False)["count"]
            sgc = O.count(rp, col, q, sgc=True, apply_root_cap=False)["count"]
            bf = O.brute_force(rp, col, q)
            assert sgm == bf, (gname, pname, sgm, bf)
            if len(rp) - 1 <= 200:
                nxc = nx_count(rp, col, q)
                assert sgm == nxc, (gname, pname, sgm, nxc)
            rec["counts"][pname] = {"sgm": int(sgm), "sgc": int(sgc)}
        out["small"][gname] = rec
        print(gname, "done", flush=True)
    for gname, ((kind, args), pats) in LARGE.items():
        rp, col = gen(kind, args)
        rec = {"kind": kind, "args": list(args), "n": int(len(rp) - 1), "m": int(len(col)),
               "cutoff": O.cutoff(rp), "counts": {}}
        for pname in pats:
            r1 = O.count(rp, col, P.NAMED[pname], sgc=False)
            r2 = O.count(rp, col, P.NAMED[pname], sgc=True)
            assert r1["q2_risk"] == 0 and r1["q3_skipped"] == 0
            rec["counts"][pname] = {"sgm": int(r1["count"]), "sgc": int(r2["count"]), "roots": int(r1["roots"]),
                                    "peel_rounds": int(r1["peel_rounds"])}
        out["large"][gname] = rec
        print(gname, rec["counts"], flush=True)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
