"""Generate tests/golden/converters/: inputs for the file converters and the
outputs the reference's own binary writes for them (src/main.cu:40-67,
-m txt-bel | mtx-bel | tsv-bel | tsv-mtx | bel-mtx -g <in> -r <out>).

The reference binary is built by oracle/refbuild.py into oracle/_ref/beep_ref.
It links the CUDA driver, so it loads only on a machine with a GPU driver,
although the converters themselves make no CUDA call. Run from the repository
root on such a machine:  python tests/golden/make_converter_golden.py

Only inputs the reference reads to the end are used (no empty lines, lines
under 100 characters, non-empty Matrix Market outputs). A case whose run does
not produce the output file is recorded in index.json under "failed".
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.join(ROOT, "tests", "golden", "converters")
REF = os.path.join(ROOT, "oracle", "_ref", "beep_ref")
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)

import test_convert as T  # noqa: E402


def main():
    if not os.path.exists(REF):
        sys.exit(f"missing {REF}: build it with python oracle/refbuild.py")
    os.makedirs(OUT, exist_ok=True)
    inputs = []
    for name, text in T.TXT_CASES.items():
        inputs.append(("txt-bel", f"txt_{name}.txt", text.encode()))
    for name, text in T.MTX_CASES.items():
        inputs.append(("mtx-bel", f"mtx_{name}.mtx", text.encode()))
    for name, text in T.TSV_CASES.items():
        inputs.append(("tsv-bel", f"tsv_{name}.tsv", text.encode()))
        inputs.append(("tsv-mtx", f"tsv_{name}.tsv", text.encode()))
    # a small .bel with non-zero weight words for bel-mtx
    import struct
    recs = [(1, 0, 0), (0, 1, 3), (2, 1, 0xFFFFFFFF), (1, 2, (1 << 32) | 9)]
    inputs.append(("bel-mtx", "bel_small.bel", b"".join(struct.pack("<QQQ", *r) for r in recs)))
    cases, failed = [], []
    for task, fname, data in inputs:
        src = os.path.join(OUT, fname)
        with open(src, "wb") as f:
            f.write(data)
        out_name = f"{os.path.splitext(fname)[0]}.{task}.out"
        dst = os.path.join(OUT, out_name)
        if os.path.exists(dst):
            os.remove(dst)
        r = subprocess.run([REF, "-m", task, "-g", src, "-r", dst], capture_output=True, text=True, timeout=60)
        name = f"{task}:{fname}"
        if os.path.exists(dst):
            cases.append({"name": name, "task": task, "input": fname, "output": out_name})
        else:
            failed.append({"name": name, "returncode": r.returncode, "stderr": r.stderr[-400:]})
        print(name, "ok" if os.path.exists(dst) else f"FAILED rc={r.returncode}", flush=True)
    with open(os.path.join(OUT, "index.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_converter_golden.py", "reference": "oracle/_ref/beep_ref",
                   "cases": cases, "failed": failed}, f, indent=1)


if __name__ == "__main__":
    main()
