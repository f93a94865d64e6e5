"""File converters (-m txt-bel | mtx-bel | tsv-bel | tsv-mtx | bel-mtx):
beep_convert must write the bytes of the CPU restatement of the reference's
converters (oracle/convert_ref.py), and the outputs the reference binary itself
wrote for the committed inputs (tests/golden/converters/). CPU only."""
import json
import os
import subprocess

import numpy as np
import pytest

import beep_b200 as B
from oracle import convert_ref as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "converters")

TXT_CASES = {
    "plain": "0 1\n1 2\n2 0\n",
    "comments_loops_dups": "% a comment\n%% another\n3 3\n0 5\n5 0\n0 5\n2 7 9\n7 2\n",
    "unsorted_wide_ids": "4000000000 1\n17 4\n4 17\n1 4000000000\n",
    "garbage_lines": "x y\n1\n2 3\n-1 4\n 5 6\n",
    "crlf": "1 2\r\n2 3\r\n",
}
# lines the reference cannot read (its fscanf loop stalls on an empty line,
# its line buffer holds 99 characters): compared with the restatement only
TXT_OWN_CASES = {
    "empty_lines": "1 2\n\n2 3\n\n",
    "long_line": "1 2 " + "9" * 200 + "\n3 4\n",
    "empty": "",
}
MTX_CASES = {
    "general": "%%MatrixMarket matrix coordinate pattern general\n4 4 3\n1 2\n2 3\n3 1\n",
    "symmetric_values": "%%MatrixMarket matrix coordinate real symmetric\n% c\n5 5 4\n1 2 0.5\n3 3 1\n4 1 2\n2 5 -1\n",
    "last_comment_wins": "%%MatrixMarket matrix coordinate pattern symmetric\n% plain\n3 3 2\n0 1\n1 2\n",
    "short_body": "%%MatrixMarket matrix coordinate pattern general\n3 3 5\n0 1\n1 2\n",
    "bad_entry_stops": "%%MatrixMarket matrix coordinate integer general\n3 3 4\n0 1 1\n1\n2 0 1\n",
    "duplicates_kept": "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 3\n0 1\n1 0\n0 1\n",
    "array": "%%MatrixMarket matrix array real general\n2 2\n1.0\n0\n3\n4\n",
}
MTX_ERRORS = {
    "not_square": "%%MatrixMarket matrix coordinate pattern general\n3 4 1\n0 1\n",
    "no_size": "%%MatrixMarket matrix coordinate pattern general\n",
}
TSV_CASES = {
    "plain": "1 0 0\n2 1 0\n0 2 7\n",
    "one_line": "5 6 1 7 8 2 9 10 3\n",
    "trailing_partial": "1 2 3\n4 5\n",
    "garbage_stops": "1 2 3\n4 5x 6\n7 8 9\n",
    "big_weight": "1 2 4294967297\n3 4 18446744073709551615\n",
}


def run(task, src_bytes, tmp_path, name="in"):
    src = tmp_path / f"{name}.src"
    src.write_bytes(src_bytes)
    dst = tmp_path / f"{name}.dst"
    n = B.convert(task, str(src), str(dst))
    return n, dst.read_bytes()


@pytest.mark.parametrize("name", sorted(TXT_CASES) + sorted(TXT_OWN_CASES))
def test_txt_bel(built, tmp_path, name):
    text = {**TXT_CASES, **TXT_OWN_CASES}[name]
    n, out = run("txt-bel", text.encode(), tmp_path)
    want = R.txt_bel(text)
    assert out == want
    assert n * 24 == len(out)


@pytest.mark.parametrize("name", sorted(MTX_CASES))
def test_mtx_bel(built, tmp_path, name):
    n, out = run("mtx-bel", MTX_CASES[name].encode(), tmp_path)
    assert out == R.mtx_bel(MTX_CASES[name])
    assert n * 24 == len(out)


@pytest.mark.parametrize("name", sorted(MTX_ERRORS))
def test_mtx_bel_errors(built, tmp_path, name):
    with pytest.raises(ValueError):
        R.mtx_bel(MTX_ERRORS[name])
    with pytest.raises(B.BeepError) as e:
        run("mtx-bel", MTX_ERRORS[name].encode(), tmp_path)
    assert e.value.status == B.ERR_PARSE


@pytest.mark.parametrize("name", sorted(TSV_CASES))
def test_tsv_bel_and_mtx(built, tmp_path, name):
    text = TSV_CASES[name]
    _, out = run("tsv-bel", text.encode(), tmp_path, "a")
    assert out == R.tsv_bel(text)
    _, out = run("tsv-mtx", text.encode(), tmp_path, "b")
    assert out.decode() == R.tsv_mtx(text)


def test_bel_mtx_roundtrip(built, tmp_path):
    rp, col = B.gen_erdos_renyi(40, 0.2, 3)
    B.write_bel(str(tmp_path / "g.bel"), rp, col)
    data = (tmp_path / "g.bel").read_bytes()
    n = B.convert("bel-mtx", str(tmp_path / "g.bel"), str(tmp_path / "g.mtx"))
    text = (tmp_path / "g.mtx").read_text()
    assert text == R.bel_mtx(data)
    assert n == len(col)
    # weights: low 32 bits of the third word as a signed int
    recs = np.frombuffer(data, dtype=np.uint64).reshape(-1, 3).copy()
    recs[:, 2] = [0xFFFFFFFF, 1 << 32 | 5] * (len(recs) // 2) + [7] * (len(recs) % 2)
    (tmp_path / "w.bel").write_bytes(recs.tobytes() + b"\x01\x02")  # trailing partial record ignored
    B.convert("bel-mtx", str(tmp_path / "w.bel"), str(tmp_path / "w.mtx"))
    assert (tmp_path / "w.mtx").read_text() == R.bel_mtx(recs.tobytes())


def test_empty_inputs_to_market_fail(built, tmp_path):
    for task in ("tsv-mtx", "bel-mtx"):
        with pytest.raises(B.BeepError) as e:
            run(task, b"", tmp_path)
        assert e.value.status == B.ERR_PARSE


def test_txt_bel_output_loads_as_graph(built, tmp_path):
    """A converted edge list is a valid .bel data graph: the loader reads it
    back to the same undirected edge set."""
    rng = np.random.default_rng(5)
    pairs = rng.integers(0, 60, size=(300, 2))
    text = "".join(f"{a} {b}\n" for a, b in pairs)
    run("txt-bel", text.encode(), tmp_path, "t")
    raw = np.frombuffer((tmp_path / "t.dst").read_bytes(), dtype=np.uint64).reshape(-1, 3)
    got = set(zip(raw[:, 1].tolist(), raw[:, 0].tolist()))
    want = {(int(a), int(b)) for a, b in pairs if a != b} | {(int(b), int(a)) for a, b in pairs if a != b}
    assert got == want
    assert np.all(np.diff(raw[:, 1].astype(np.int64)) >= 0)


def test_cli_converts(built, tmp_path):
    src = tmp_path / "e.txt"
    src.write_text(TXT_CASES["comments_loops_dups"])
    r = subprocess.run([os.path.join(ROOT, "beep_b200", "beep"), "-m", "txt-bel", "-g", str(src), "-r",
                        str(tmp_path / "e.bel")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "e.bel").read_bytes() == R.txt_bel(TXT_CASES["comments_loops_dups"])


def golden_cases():
    path = os.path.join(GOLDEN, "index.json")
    if not os.path.exists(path):
        return []
    with open(path) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c["name"])
def test_matches_reference_binary_outputs(built, tmp_path, case):
    """Outputs written by the reference's own converters
    (tests/golden/make_converter_golden.py runs them)."""
    src = os.path.join(GOLDEN, case["input"])
    dst = tmp_path / "out"
    B.convert(case["task"], src, str(dst))
    with open(os.path.join(GOLDEN, case["output"]), "rb") as f:
        assert dst.read_bytes() == f.read()
