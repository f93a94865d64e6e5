"""Host-side checks of the C ABI: the library loads and exports every symbol
include/beep.h declares, the query compiler agrees with the oracle, file
formats and generators behave. No device calls. CPU only."""
import ctypes
import itertools
import os
import re
import struct
import subprocess

import numpy as np
import pytest

import beep_b200 as B
from beep_b200 import patterns as P
from oracle import pyoracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "beep.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(beep_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(built):
    declared = header_functions()
    assert len(declared) >= 20
    lib = ctypes.CDLL(B.LIB_PATH)
    for name in declared:
        assert hasattr(lib, name), name
    # the Python bindings cover the whole header
    assert sorted(B.exported_names()) == declared


def all_patterns():
    out = list(P.NAMED.items())
    out += [(f"c4_{i}", q) for i, q in enumerate(P.central_patterns(4))]
    out += [(f"c5_{i}", q) for i, q in enumerate(P.central_patterns(5))]
    return out


def test_fifteen_central_patterns():
    assert len(P.central_patterns(4)) == 4
    assert len(P.central_patterns(5)) == 11


@pytest.mark.parametrize("mode", [B.SGM, B.SGC])
def test_query_plan_matches_oracle(built, mode):
    keys = ["K", "order", "qedge_ptr", "qedge", "sym_ptr", "sym", "unmat", "first_sym_level", "min_qdeg",
            "max_qdeg", "aut_order"]
    for name, q in all_patterns():
        a = B.Query.from_edges(q).plan(mode)
        o = O.plan(q, sgc=(mode == B.SGC))
        for k in keys:
            assert a[k] == o[k], (name, k)


def test_restricted_flag():
    assert B.Query.from_edges(P.K4).plan()["restricted"] == 1
    assert B.Query.from_edges(P.K5).plan()["restricted"] == 1
    assert B.Query.from_edges(P.TRIANGLE).plan()["restricted"] == 1
    assert B.Query.from_edges(P.DIAMOND).plan()["restricted"] == 0
    assert B.Query.from_edges(P.W5).plan()["restricted"] == 0


def test_wheel4_flag():
    """Only the 4-wheel's plan takes the per-(x1, x3) closed form: under every
    labelling of its edge list (the reference's chain comes out in two forms)
    and in both modes (its last position is adjacent to the one before, so
    sgc counts full matches)."""
    plans = set()
    for perm in itertools.permutations(range(5)):
        pl = B.Query.from_edges([(perm[a], perm[b]) for a, b in P.W5]).plan()
        assert pl["wheel4"] == 1
        plans.add((tuple(pl["qedge"]), tuple(pl["sym"])))
    assert len(plans) == 2
    assert B.Query.from_edges(P.W5).plan(B.SGC)["wheel4"] == 1
    for q in [P.K4, P.DIAMOND, P.TAILED_TRIANGLE, P.TRIANGLE] + P.central_patterns(5):
        pl = B.Query.from_edges(q).plan()
        assert pl["wheel4"] == (1 if pl["qdeg"] == [4, 3, 3, 3, 3] and pl["aut_order"] == 8 else 0), q


def test_unsupported_queries_fail_cleanly(built):
    # path 0-1-2-3: no central vertex; counted (sgm) by the list walker, but
    # its sgc form stops before a last position that is not adjacent to the
    # one before it, which is defined for central queries only
    path = [(0, 1), (1, 0), (1, 2), (2, 1), (2, 3), (3, 2)]
    assert B.Query.from_edges(path).plan(B.SGM)["central"] == 0
    with pytest.raises(B.BeepError) as e:
        B.Query.from_edges(path).plan(B.SGC)
    assert e.value.status == B.ERR_UNSUPPORTED
    # disconnected
    with pytest.raises(B.BeepError):
        B.Query.from_edges([(0, 1), (1, 0), (2, 3), (3, 2)]).plan()
    # 11 vertices
    star11 = [(0, i) for i in range(1, 11)] + [(i, 0) for i in range(1, 11)]
    with pytest.raises(B.BeepError) as e:
        B.Query.from_edges(star11)
    assert e.value.status == B.ERR_UNSUPPORTED
    # asymmetric edge list
    with pytest.raises(B.BeepError):
        B.Query.from_edges([(0, 1), (0, 2), (1, 0), (1, 2), (2, 0)]).plan()


def test_mtx_reader(tmp_path, built):
    p = tmp_path / "tri.mtx"
    p.write_text(P.to_mtx(P.TRIANGLE))
    assert B.Query.load_mtx(str(p)).plan()["order"] == [0, 1, 2]
    # %%...symmetric banner adds the reverse edges; comments are skipped
    p2 = tmp_path / "k4sym.mtx"
    lines = ["%%MatrixMarket matrix coordinate pattern symmetric", "% a comment", "4 4 6"]
    lines += [f"{a} {b}" for a in range(4) for b in range(a + 1, 4)]
    p2.write_text("\n".join(lines) + "\n")
    pl = B.Query.load_mtx(str(p2)).plan()
    assert pl["K"] == 4 and pl["aut_order"] == 24
    # errors
    bad = tmp_path / "bad.mtx"
    bad.write_text("3 4 2\n0 1\n1 0\n")
    with pytest.raises(B.BeepError) as e:
        B.Query.load_mtx(str(bad))
    assert e.value.status == B.ERR_PARSE
    with pytest.raises(B.BeepError) as e:
        B.Query.load_mtx(str(tmp_path / "missing.mtx"))
    assert e.value.status == B.ERR_IO


def test_bel_writer_byte_layout(tmp_path, built):
    rp, col = B.gen_erdos_renyi(50, 0.2, 9)
    path = tmp_path / "g.bel"
    B.write_bel(str(path), rp, col)
    raw = path.read_bytes()
    assert len(raw) == 24 * len(col)
    recs = np.frombuffer(raw, dtype=np.uint64).reshape(-1, 3)
    # {u64 dst @0, u64 src @8, u64 weight @16} (include/FIleReader.cuh:63-89)
    src = np.repeat(np.arange(50), np.diff(rp))
    assert np.array_equal(recs[:, 1], src.astype(np.uint64))
    assert np.array_equal(recs[:, 0], col.astype(np.uint64))
    assert struct.unpack("<Q", raw[8:16])[0] == recs[0, 1]


def test_generators_deterministic_and_simple(built):
    for fn, args in [(B.gen_erdos_renyi, (500, 0.02, 3)), (B.gen_rmat, (10, 8, 0.57, 0.19, 0.19, 5)),
                     (B.gen_chung_lu, (1000, 10.0, 2.1, 7))]:
        rp1, c1 = fn(*args)
        rp2, c2 = fn(*args)
        assert np.array_equal(rp1, rp2) and np.array_equal(c1, c2)
        n = len(rp1) - 1
        for v in range(n):
            row = c1[rp1[v]:rp1[v + 1]]
            assert np.all(np.diff(row) > 0)
            assert not np.any(row == v)
        # symmetric
        src = np.repeat(np.arange(n), np.diff(rp1))
        fwd = set(zip(src.tolist(), c1.tolist()))
        assert all((b, a) in fwd for a, b in fwd)


def test_cli_help(built):
    r = subprocess.run([os.path.join(ROOT, "beep_b200", "beep"), "-h"], capture_output=True, text=True)
    assert r.returncode == 0
    assert "-g" in r.stdout and "sgc" in r.stdout
    r = subprocess.run([os.path.join(ROOT, "beep_b200", "beep"), "-m", "tc", "-g", "x", "-t", "y"],
                       capture_output=True, text=True)
    assert r.returncode != 0 and "Unrecognized" in r.stderr


def test_tune_cache_round_trip(tmp_path):
    """The autotuner's choice persisted per workload key in a JSON file: a
    stored entry reads back exactly, other keys are kept, and a missing file,
    key or limit reads as nothing."""
    import beep_b200 as B

    path = str(tmp_path / "tiers.json")
    assert B.tune_cache_get(path, "c4") is None
    t1 = {"tiny_max": 8, "small_max": 64, "med_a_max": 256, "med_max": 1024, "donate_min_iters": 2,
          "count_ms": 12.5}
    t2 = {"tiny_max": 16, "small_max": 32, "med_a_max": 128, "med_max": 512, "donate_min_iters": 0}
    B.tune_cache_put(path, "c4", t1)
    B.tune_cache_put(path, "other", t2)
    assert B.tune_cache_get(path, "c4") == t1
    assert B.tune_cache_get(path, "other") == t2
    assert B.tune_cache_get(path, "missing") is None
    with open(path, "w") as f:
        f.write('{"c4": {"tiny_max": 8}}')
    assert B.tune_cache_get(path, "c4") is None
