"""Record the reference implementation's own counts on the seeded inputs.

Runs oracle/_ref/beep_ref (the reference's src/main.cu built for sm_100a by
oracle/refbuild.py) on a GPU machine: writes each seeded graph as .bel and
each query as .mtx, runs `beep_ref -g G.bel -t Q.mtx -m sgm|sgc -d 0`, parses
"------------- Counter = N" and its timing lines, and writes
tests/golden/reference_counts.json. The tests compare the oracle with these
recorded counts; nothing at test time runs the reference.

  python tests/golden/make_reference_counts.py [--timeout 300] [--cases c1,c2]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import beep_b200 as B  # noqa: E402
from beep_b200 import patterns as P  # noqa: E402

CASES = {
    # the large config: recorded to show how the reference fails on it
    "c3": ("c3_rmat_22_28_s11", ("rmat", (22, 28, 0.57, 0.19, 0.19, 11)), [("k5", "sgm")]),
    "c1": ("c1_er_4096_p004_s1", ("er", (4096, 0.004, 1)), [("triangle", "sgc"), ("triangle", "sgm")]),
    "small": ("rmat_9_8_s6", ("rmat", (9, 8, 0.57, 0.19, 0.19, 6)),
              [(p, m) for p in ["triangle", "diamond", "k4", "tailed_triangle", "w5", "k5"] for m in ("sgm", "sgc")]),
    "c2": ("c2_rmat_20_3_s7", ("rmat", (20, 3, 0.57, 0.19, 0.19, 7)),
           [("k4", "sgm"), ("diamond", "sgm"), ("k4", "sgc"), ("diamond", "sgc")]),
}


def gen(kind, args):
    return {"er": B.gen_erdos_renyi, "rmat": B.gen_rmat, "cl": B.gen_chung_lu}[kind](*args)


def parse(out: str) -> dict:
    r = {}
    m = re.search(r"Counter = (\d+)", out)
    r["count"] = int(m.group(1)) if m else None
    for key, pat in [("transfer_s", r"Transfer Time: ([0-9.eE+-]+) s"),
                     ("preprocessing_ms", r"Preprocessing TIME: ([0-9.eE+-]+) ms"),
                     ("final_count_s", r"final count time ([0-9.eE+-]+) s")]:
        m = re.search(pat, out)
        r[key] = float(m.group(1)) if m else None
    return r


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--timeout", type=float, default=300)
    ap.add_argument("--cases", default="small,c1,c2")
    ap.add_argument("--repeat", default="",
                    help="comma-separated graph/pattern/mode keys to run several times (runs_repeated)")
    ap.add_argument("--repeats", type=int, default=5)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                  "reference_counts.json"))
    args = ap.parse_args()
    binary = os.path.join(ROOT, "oracle", "_ref", "beep_ref")
    result = {"binary": "reference src/main.cu built for sm_100a (oracle/refbuild.py)", "runs": {}}
    if os.path.exists(args.out):
        with open(args.out) as f:
            result = json.load(f)
    with tempfile.TemporaryDirectory() as td:
        for case in args.cases.split(","):
            gname, (kind, gargs), runs = CASES[case]
            rp, col = gen(kind, gargs)
            bel = os.path.join(td, f"{gname}.bel")
            B.write_bel(bel, rp, col)
            for pname, mode in runs:
                mtx = os.path.join(td, f"{pname}.mtx")
                B.write_mtx(mtx, P.NAMED[pname])
                key = f"{gname}/{pname}/{mode}"
                reps = args.repeats if key in args.repeat.split(",") else 1
                recs = []
                for _ in range(reps):
                    try:
                        r = subprocess.run([binary, "-g", bel, "-t", mtx, "-m", mode, "-d", "0"],
                                           capture_output=True, text=True, timeout=args.timeout)
                        rec = parse(r.stdout)
                        rec["returncode"] = r.returncode
                        if r.returncode != 0:
                            rec["stderr_tail"] = r.stderr[-600:]
                            rec["stdout_tail"] = r.stdout[-600:]
                    except subprocess.TimeoutExpired:
                        rec = {"count": None, "timeout_s": args.timeout}
                    recs.append(rec)
                    print(key, rec, flush=True)
                if reps > 1:
                    result.setdefault("runs_repeated", {})[key] = recs
                else:
                    result["runs"][key] = recs[0]
                with open(args.out, "w") as f:
                    json.dump(result, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
