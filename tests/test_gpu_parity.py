"""Parity of the CUDA path with the oracle (bit-exact integer counts).
Every call goes through the C ABI (libbeep_b200.so)."""
import itertools
import math
import os
import subprocess

import numpy as np
import pytest

import beep_b200 as B
from beep_b200 import patterns as P
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

GENS = {"er": B.gen_erdos_renyi, "cl": B.gen_chung_lu, "rmat": B.gen_rmat}


def csr_from_pairs(n, pairs):
    adj = [set() for _ in range(n)]
    for a, b in pairs:
        if a != b:
            adj[a].add(b)
            adj[b].add(a)
    rp = [0]
    col = []
    for v in range(n):
        col += sorted(adj[v])
        rp.append(len(col))
    return np.array(rp, np.int32), np.array(col, np.int32)


def gpu_count(ctx, rp, col, q, mode=B.SGM, options=0):
    g = B.Graph.from_csr(ctx, rp, col)
    try:
        return B.count(g, q, mode, options)
    finally:
        g.close()


def test_small_fixtures_all_patterns(ctx, golden):
    for gname, rec in golden["small"].items():
        rp, col = GENS[rec["kind"]](*rec["args"])
        g = B.Graph.from_csr(ctx, rp, col)
        for pname, c in rec["counts"].items():
            q = [tuple(e) for e in golden["patterns"][pname]]
            assert B.count(g, q, B.SGM) == c["sgm"], (gname, pname, "sgm")
            assert B.count(g, q, B.SGC) == c["sgc"], (gname, pname, "sgc")
        g.close()


@pytest.mark.parametrize("n", [10, 40, 66, 100])
def test_complete_graphs(ctx, n):
    rp, col = csr_from_pairs(n, itertools.combinations(range(n), 2))
    g = B.Graph.from_csr(ctx, rp, col)
    exp = {
        "triangle": math.comb(n, 3), "k4": math.comb(n, 4), "k5": math.comb(n, 5),
        "diamond": 6 * math.comb(n, 4), "tailed_triangle": 12 * math.comb(n, 4), "claw": 4 * math.comb(n, 4),
    }
    if n <= 66:
        exp["w5"] = 15 * math.comb(n, 5)
    for name, e in exp.items():
        assert B.count(g, P.NAMED[name]) == e, name
    g.close()


def hub_graph(n_leaves, p, seed):
    rng = np.random.default_rng(seed)
    pairs = [(0, i) for i in range(1, n_leaves + 1)]
    m = int(p * n_leaves * (n_leaves - 1) / 2)
    a = rng.integers(1, n_leaves + 1, size=m)
    b = rng.integers(1, n_leaves + 1, size=m)
    pairs += list(zip(a.tolist(), b.tolist()))
    return csr_from_pairs(n_leaves + 1, pairs)


def test_large_tier_hub(ctx):
    """A hub of degree 1500 exercises the global-bitmap (large) tier. It is a
    root only for plans whose position 1 need not follow the root: with the
    diamond (position 1 symmetric to the root) the hub, last in ascending
    order, has no later neighbour and is not searched."""
    rp, col = hub_graph(1500, 0.01, 3)
    g = B.Graph.from_csr(ctx, rp, col)
    try:
        for name in ["triangle", "diamond", "k4", "tailed_triangle", "w5", "k5", "claw"]:
            for mode, sgc in [(B.SGM, False), (B.SGC, True)]:
                exp = O.count(rp, col, P.NAMED[name], sgc=sgc, apply_root_cap=False)["count"]
                c, st = B.count(g, P.NAMED[name], mode, B.OPT_TIMING, stats=True)
                assert c == exp, (name, mode)
                if name in ("w5", "tailed_triangle", "claw"):
                    assert st["roots_large"] >= 1, (name, st)
    finally:
        g.close()


def wide_hub_graph(seed):
    """Hub 0 with 12,000 leaves (its neighbourhood rows are 12,000 bits wide,
    so the large tier walks their non-zero-word lists), a sparse random graph
    on the leaves, a second hub on 3,000 of them (a row too dense for its
    list, walked word by word) and a 20-clique among the leaves."""
    rng = np.random.default_rng(seed)
    n = 12000
    pairs = [(0, i) for i in range(1, n + 1)]
    a = rng.integers(1, n + 1, size=48000)
    b = rng.integers(1, n + 1, size=48000)
    pairs += list(zip(a.tolist(), b.tolist()))
    pairs += [(1, int(v)) for v in rng.choice(np.arange(2, n + 1), size=3000, replace=False)]
    clique = rng.choice(np.arange(2, n + 1), size=20, replace=False).tolist()
    pairs += list(itertools.combinations(clique, 2))
    return csr_from_pairs(n + 1, pairs)


def test_large_tier_word_lists(ctx):
    rp, col = wide_hub_graph(5)
    g = B.Graph.from_csr(ctx, rp, col)
    try:
        # the 4-wheel under its second labelling too (the other form of the reference's chain)
        w5b = P.central_patterns(5)[8]
        assert B.Query.from_edges(w5b).plan()["wheel4"] == 1 and sorted(w5b) != sorted(P.W5)
        queries = {name: P.NAMED[name] for name in ["w5", "diamond", "tailed_triangle", "k4", "k5", "triangle"]}
        queries["w5_relabelled"] = w5b
        for name, q in queries.items():
            exp = O.count(rp, col, q, apply_root_cap=False)["count"]
            c, st = B.count(g, q, B.SGM, B.OPT_TIMING, stats=True)
            assert c == exp, name
            if name in ("w5", "w5_relabelled", "tailed_triangle"):
                assert st["roots_large"] >= 1, (name, st)
        # enumeration through the lists: the same set of matches as the oracle
        total = O.count(rp, col, P.W5, apply_root_cap=False)["count"]
        tuples, t = B.enumerate_matches(g, P.W5, total + 5)
        assert t == total and len(tuples) == total
        assert canon(tuples) == canon(O.enumerate_matches(rp, col, P.W5))
    finally:
        g.close()


@pytest.mark.parametrize("scale,ef,seed", [(12, 8, 1), (14, 6, 2)])
def test_rmat_named_patterns(ctx, scale, ef, seed):
    rp, col = B.gen_rmat(scale, ef, 0.57, 0.19, 0.19, seed)
    g = B.Graph.from_csr(ctx, rp, col)
    for name in ["triangle", "diamond", "k4", "tailed_triangle", "k5", "w5"]:
        for mode, sgc in [(B.SGM, False), (B.SGC, True)]:
            exp = O.count(rp, col, P.NAMED[name], sgc=sgc, apply_root_cap=False)["count"]
            assert B.count(g, P.NAMED[name], mode) == exp, (name, mode)
    g.close()


def test_c1_triangle(ctx, golden):
    rec = golden["large"]["c1_er_4096_p004_s1"]
    rp, col = B.gen_erdos_renyi(*rec["args"])
    g = B.Graph.from_csr(ctx, rp, col)
    assert g.info()["cutoff"] == rec["cutoff"]
    assert B.count(g, P.TRIANGLE, B.SGC) == rec["counts"]["triangle"]["sgc"]
    assert B.count(g, P.TRIANGLE, B.SGM) == rec["counts"]["triangle"]["sgm"]
    g.close()


def test_c2_k4_diamond(ctx, golden):
    rec = golden["large"]["c2_rmat_20_3_s7"]
    rp, col = B.gen_rmat(*rec["args"])
    g = B.Graph.from_csr(ctx, rp, col)
    assert g.info()["cutoff"] == rec["cutoff"]
    for name in ["k4", "diamond"]:
        c, st = B.count(g, P.NAMED[name], B.SGM, B.OPT_TIMING, stats=True)
        assert c == rec["counts"][name]["sgm"], name
        # roots that can hold a match (the oracle's figure counts every vertex of degree >= max_qdeg)
        assert 0 < st["roots"] <= rec["counts"][name]["roots"]
        assert st["peel_rounds"] == rec["counts"][name]["peel_rounds"]
        assert B.count(g, P.NAMED[name], B.SGC) == rec["counts"][name]["sgc"], name
    g.close()


def canon(rows):
    return sorted(map(tuple, np.asarray(rows).tolist()))


def test_enumerate_matches_oracle_set(ctx, golden):
    rec = golden["small"]["er_60_p15_s3"]
    rp, col = B.gen_erdos_renyi(*rec["args"])
    g = B.Graph.from_csr(ctx, rp, col)
    for name in ["triangle", "diamond", "k4", "tailed_triangle", "w5", "claw"]:
        total = rec["counts"][name]["sgm"]
        tuples, t = B.enumerate_matches(g, P.NAMED[name], total + 5)
        assert t == total and len(tuples) == total, name
        exp = O.enumerate_matches(rp, col, P.NAMED[name])
        assert canon(tuples) == canon(exp), name
        # every tuple is an embedding
        adj = {(int(s), int(d)) for s in range(len(rp) - 1) for d in col[rp[s]:rp[s + 1]]}
        for tup in tuples[:50]:
            for a, b in P.NAMED[name]:
                assert (int(tup[a]), int(tup[b])) in adj
    g.close()


def test_enumerate_first_k(ctx):
    rp, col = B.gen_rmat(12, 8, 0.57, 0.19, 0.19, 1)
    g = B.Graph.from_csr(ctx, rp, col)
    for name in ["diamond", "k4"]:
        total = O.count(rp, col, P.NAMED[name], apply_root_cap=False)["count"]
        k = 1000
        tuples, t = B.enumerate_matches(g, P.NAMED[name], k)
        assert t == total and len(tuples) == min(k, total)
        assert len(set(map(tuple, tuples.tolist()))) == len(tuples)
        full = set(map(tuple, O.enumerate_matches(rp, col, P.NAMED[name]).tolist()))
        assert set(map(tuple, tuples.tolist())) <= full
    g.close()


def test_dirty_csr_is_deduped(ctx):
    rp, col = B.gen_erdos_renyi(300, 0.05, 5)
    clean = gpu_count(ctx, rp, col, P.DIAMOND)
    # shuffle each row, duplicate some entries, add self loops
    rng = np.random.default_rng(0)
    rows = []
    for v in range(len(rp) - 1):
        r = list(col[rp[v]:rp[v + 1]])
        r += r[: len(r) // 3] + [v]
        rng.shuffle(r)
        rows.append(r)
    rp2 = np.zeros(len(rows) + 1, np.int32)
    rp2[1:] = np.cumsum([len(r) for r in rows])
    col2 = np.array([x for r in rows for x in r], np.int32)
    g = B.Graph.from_csr(ctx, rp2, col2)
    assert g.info()["m"] == len(col)
    rpb, colb = g.csr()
    assert np.array_equal(rpb, rp) and np.array_equal(colb, col)
    assert B.count(g, P.DIAMOND) == clean
    g.close()


def test_edges_and_bel_paths(ctx, tmp_path):
    rp, col = B.gen_chung_lu(2000, 10.0, 2.1, 4)
    exp = O.count(rp, col, P.K4, apply_root_cap=False)["count"]
    src = np.repeat(np.arange(len(rp) - 1), np.diff(rp)).astype(np.uint32)
    g = B.Graph.from_edges(ctx, src, col.astype(np.uint32))
    assert B.count(g, P.K4) == exp
    g.close()
    path = tmp_path / "g.bel"
    B.write_bel(str(path), rp, col)
    g = B.Graph.load_bel(ctx, str(path))
    assert B.count(g, P.K4) == exp
    g.close()


def test_device_csr_input(ctx):
    import torch

    rp, col = B.gen_rmat(11, 8, 0.57, 0.19, 0.19, 3)
    exp = O.count(rp, col, P.TRIANGLE, apply_root_cap=False)["count"]
    drp = torch.from_numpy(rp).cuda()
    dcol = torch.from_numpy(col).cuda()
    torch.cuda.synchronize()
    g = B.Graph.from_device_csr(ctx, len(rp) - 1, len(col), drp.data_ptr(), dcol.data_ptr())
    assert B.count(g, P.TRIANGLE) == exp
    g.close()
    # the caller's buffers are not modified
    assert torch.equal(drp.cpu(), torch.from_numpy(rp))


def test_edge_cases(ctx):
    # isolated vertices only
    rp = np.zeros(11, np.int32)
    assert gpu_count(ctx, rp, np.zeros(0, np.int32), P.TRIANGLE) == 0
    # one edge
    rp, col = csr_from_pairs(2, [(0, 1)])
    assert gpu_count(ctx, rp, col, P.TRIANGLE) == 0
    # one triangle, every pattern larger than it gives 0
    rp, col = csr_from_pairs(3, [(0, 1), (1, 2), (0, 2)])
    assert gpu_count(ctx, rp, col, P.TRIANGLE) == 1
    assert gpu_count(ctx, rp, col, P.K4) == 0
    assert gpu_count(ctx, rp, col, P.DIAMOND) == 0
    # star: claws only
    rp, col = csr_from_pairs(40, [(0, i) for i in range(1, 40)])
    assert gpu_count(ctx, rp, col, P.CLAW) == math.comb(39, 3)
    assert gpu_count(ctx, rp, col, P.TRIANGLE) == 0
    # sgc with K - LUNMAT < 3 (wedge) counts 0, like the reference's main path
    assert gpu_count(ctx, rp, col, P.WEDGE, B.SGC) == 0
    assert gpu_count(ctx, rp, col, P.WEDGE, B.SGM) == math.comb(39, 2)


def test_reference_root_cap_option(ctx):
    """Roots with degree >= 100*cutoff are skipped only with the option."""
    n = 400000
    hub_leaves = 5000
    rng = np.random.default_rng(2)
    pairs = [(0, i) for i in range(1, hub_leaves + 1)]
    a = rng.integers(1, hub_leaves + 1, size=15000)
    b = rng.integers(1, hub_leaves + 1, size=15000)
    pairs += list(zip(a.tolist(), b.tolist()))
    rp, col = csr_from_pairs(n, pairs)
    cut = O.cutoff(rp)
    assert np.diff(rp).max() >= 100 * cut
    for name in ["triangle", "diamond"]:
        capped = O.count(rp, col, P.NAMED[name], apply_root_cap=True)
        full = O.count(rp, col, P.NAMED[name], apply_root_cap=False)
        assert capped["q3_skipped"] >= 1
        assert gpu_count(ctx, rp, col, P.NAMED[name], B.SGM, B.OPT_REFERENCE_ROOT_CAP) == capped["count"]
        assert gpu_count(ctx, rp, col, P.NAMED[name], B.SGM) == full["count"]


def test_cli_counter_line(built, tmp_path):
    rp, col = B.gen_erdos_renyi(4096, 0.004, 1)
    bel = tmp_path / "c1.bel"
    mtx = tmp_path / "tri.mtx"
    B.write_bel(str(bel), rp, col)
    mtx.write_text(P.to_mtx(P.TRIANGLE))
    r = subprocess.run([os.path.join(ROOT, "beep_b200", "beep"), "-g", str(bel), "-t", str(mtx), "-m", "sgc",
                        "-d", "0"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    exp = O.count(rp, col, P.TRIANGLE, sgc=True)["count"]
    assert f"------------- Counter = {exp}" in r.stdout


def test_sg_match_mirror(built, capsys):
    rp, col = B.gen_erdos_renyi(4096, 0.004, 1)
    sg = B.SG_Match(B.GRAPH_COUNT, "node", 0, 768, 1)
    c = sg.run((rp, col), P.TRIANGLE)
    assert c == O.count(rp, col, P.TRIANGLE, sgc=True)["count"]
    assert f"------------- Counter = {c}" in capsys.readouterr().out


def test_root_shards_sum_and_match_oracle(ctx):
    rp, col = B.gen_rmat(12, 8, 0.57, 0.19, 0.19, 1)
    g = B.Graph.from_csr(ctx, rp, col)
    for name in ["triangle", "diamond", "k4", "w5", "claw"]:
        full = B.count(g, P.NAMED[name])
        parts = [B.count_shard(g, P.NAMED[name], r, 5) for r in range(5)]
        assert sum(parts) == full, name
        for r in range(5):
            exp = O.count(rp, col, P.NAMED[name], apply_root_cap=False, root_mod=5, root_rem=r)["count"]
            assert parts[r] == exp, (name, r)
    g.close()


def test_c3_sampled_roots(ctx):
    """Full-size R-MAT s22 ef28 (seed 11): the 5-clique count of 1 root in
    997 (by input id) against the oracle's independent clique counter on the
    same roots, and the 4-wheel count of another shard of 1,701 roots (degrees
    up to 5,140, 31 of them in the large tier) against the oracle's count of
    those roots, recorded in tests/golden/c3_samples.json by
    tests/golden/make_c3_samples.py."""
    import json

    rp, col = B.gen_rmat(22, 28, 0.57, 0.19, 0.19, 11)
    g = B.Graph.from_csr(ctx, rp, col)
    info = g.info()
    assert info["n"] == 1 << 22 and info["m"] == len(col)
    mod, rem = 997, 5
    got = B.count_shard(g, P.K5, rem, mod)
    exp = O.count_cliques(rp, col, 5, mod, rem)
    assert got == exp
    assert got > 0
    with open(os.path.join(ROOT, "tests", "golden", "c3_samples.json")) as f:
        fx = json.load(f)
    assert fx["graph"]["m_directed"] == len(col)
    for smp in fx["samples"]:
        c, st = B.count_shard(g, P.NAMED[smp["pattern"]], smp["root_rem"], smp["root_mod"], options=B.OPT_TIMING,
                              stats=True)
        assert c == smp["count"], smp
        assert st["roots_large"] >= 1, st
    g.close()
