"""Oracle counts of the 4-wheel on a root shard of the large config, for the
GPU parity test of that config (tests/test_gpu_parity.py).

The large config is R-MAT scale 22, edge factor 28, (a, b, c) = (0.57, 0.19,
0.19), seed 11 (220 M directed edges, max degree ~240 K). The oracle's dense
per-root bitmaps cannot take its hub roots, so the test compares one shard of
the roots (input id % 997 == 754: 1,701 roots of degree up to 5,140, 31 of
them above 1,024, which the large tier takes) with the oracle's count of the
same roots. It takes the OpenMP oracle about 6 minutes on 8 cores, which is
why its result is a fixture rather than computed at test time.

  python tests/golden/make_c3_samples.py
"""
from __future__ import annotations

import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import beep_b200 as B  # noqa: E402
from beep_b200 import patterns as P  # noqa: E402
from oracle import pyoracle as O  # noqa: E402

GRAPH = (22, 28, 0.57, 0.19, 0.19, 11)
SAMPLES = [("w5", 997, 754)]


def main():
    rp, col = B.gen_rmat(*GRAPH)
    out = {"graph": {"kind": "rmat", "args": list(GRAPH), "n": len(rp) - 1, "m_directed": len(col)},
           "samples": []}
    for name, mod, rem in SAMPLES:
        t0 = time.time()
        r = O.count(rp, col, P.NAMED[name], apply_root_cap=False, root_mod=mod, root_rem=rem)
        deg = np.diff(rp)[rem::mod]
        out["samples"].append({"pattern": name, "mode": "sgm", "root_mod": mod, "root_rem": rem,
                               "count": int(r["count"]), "roots": int(r["roots"]),
                               "max_root_degree": int(deg.max()), "oracle_s": round(time.time() - t0, 1)})
        print(out["samples"][-1], flush=True)
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "c3_samples.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
