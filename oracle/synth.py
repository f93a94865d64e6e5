"""Seeded synthetic graphs and the reference's input files, in numpy.

TEST INFRASTRUCTURE ONLY. A restatement of the library's generators
(beep_gen_erdos_renyi / beep_gen_rmat / beep_gen_chung_lu: splitmix64 streams
keyed by (seed, row or edge index)) and of its .bel / .mtx writers, so that
the benchmark's reference arm can write the inputs the reference binary reads
without loading the library, and so that the tests can check the library's
generators against an independent implementation. The product never imports
this module.

File formats follow the reference's readers: .bel records are three
little-endian u64 {dst, src, weight} (include/FIleReader.cuh:51-95), sorted
by source, both directions of every edge; .mtx is a "rows cols nnz" line then
0-based "row col" lines (include/FIleReader.cuh:130-212, README.md:55-64).
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
_GOLD = np.uint64(0x9E3779B97F4A7C15)
_KEYMIX = np.uint64(0x632BE59BD9B4E019)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser, elementwise on uint64 (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        x = x + _GOLD
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return x ^ (x >> np.uint64(31))


def _stream_base(seed: int, keys: np.ndarray) -> np.ndarray:
    """Base word of the counter stream (seed, key) for each key."""
    with np.errstate(over="ignore"):
        k = _splitmix64(keys.astype(np.uint64) + _KEYMIX)
        return _splitmix64(np.uint64(seed) ^ k)


def _stream_value(base: np.ndarray, i: int) -> np.ndarray:
    """Value i (1-based) of each stream."""
    with np.errstate(over="ignore"):
        return _splitmix64(base + _GOLD * np.uint64(i))


def _uniform(base: np.ndarray, i: int) -> np.ndarray:
    """Uniform double in [0, 1) from the top 53 bits of value i."""
    return (_stream_value(base, i) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def to_csr(n: int, u: np.ndarray, v: np.ndarray):
    """Undirected simple graph: loops dropped, both directions, rows sorted,
    duplicates removed. Returns int32 (row_ptr, col)."""
    u = np.asarray(u, dtype=np.int64)
    v = np.asarray(v, dtype=np.int64)
    keep = u != v
    u, v = u[keep], v[keep]
    src = np.concatenate([u, v])
    dst = np.concatenate([v, u])
    keys = np.unique((src << np.int64(32)) | dst)
    src = keys >> np.int64(32)
    dst = keys & np.int64(0xFFFFFFFF)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rp, src + 1, 1)
    rp = np.cumsum(rp)
    if rp[-1] >= 2 ** 31:
        raise ValueError("graph exceeds an int32 CSR")
    return rp.astype(np.int32), dst.astype(np.int32)


def rmat(scale: int, edge_factor: int, a: float, b: float, c: float, seed: int, chunk: int = 1 << 22):
    """R-MAT: edge e descends `scale` quadrant levels with the uniforms
    1..scale of stream (seed, e)."""
    n = 1 << scale
    ne = edge_factor << scale
    ab, abc = a + b, a + b + c
    us, vs = [], []
    for e0 in range(0, ne, chunk):
        e = np.arange(e0, min(ne, e0 + chunk), dtype=np.uint64)
        base = _stream_base(seed, e)
        u = np.zeros(len(e), dtype=np.int64)
        v = np.zeros(len(e), dtype=np.int64)
        for lvl in range(scale):
            r = _uniform(base, lvl + 1)
            bu = (r >= ab).astype(np.int64)
            bv = (((r >= a) & (r < ab)) | (r >= abc)).astype(np.int64)
            u = (u << 1) | bu
            v = (v << 1) | bv
        us.append(u)
        vs.append(v)
    return to_csr(n, np.concatenate(us), np.concatenate(vs))


def erdos_renyi(n: int, p: float, seed: int):
    """G(n, p): row u draws its neighbours v > u by geometric skips
    floor(log1p(-r) / log1p(-p)) from stream (seed, u)."""
    if p <= 0.0:
        return to_csr(n, np.zeros(0, np.int64), np.zeros(0, np.int64))
    rows = np.arange(n, dtype=np.int64)
    base = _stream_base(seed, rows.astype(np.uint64))
    lq = np.log1p(-p) if p < 1.0 else -np.inf
    pos = rows.copy()
    active = np.ones(n, dtype=bool)
    us, vs = [], []
    i = 0
    while active.any():
        i += 1
        idx = np.nonzero(active)[0]
        if p < 1.0:
            r = _uniform(base[idx], i)
            skip = np.floor(np.log1p(-r) / lq).astype(np.int64)
        else:
            skip = np.zeros(len(idx), dtype=np.int64)
        pos[idx] += skip + 1
        ok = pos[idx] < n
        us.append(idx[ok])
        vs.append(pos[idx][ok])
        active[idx[~ok]] = False
    return to_csr(n, np.concatenate(us), np.concatenate(vs))


def chung_lu(n: int, avg_degree: float, exponent: float, seed: int, chunk: int = 1 << 22):
    """Chung-Lu: n * avg / 2 edges, each endpoint drawn by the weights
    (i + 1)^(-1 / (exponent - 1)) through the inverse CDF with uniforms 1 and 2
    of stream (seed, e)."""
    ex = -1.0 / (exponent - 1.0)
    w = np.power(np.arange(1, n + 1, dtype=np.float64), ex)
    cdf = np.add.accumulate(w)
    cdf = cdf / cdf[-1]
    ne = int(np.rint(n * avg_degree / 2.0))
    us, vs = [], []
    for e0 in range(0, ne, chunk):
        e = np.arange(e0, min(ne, e0 + chunk), dtype=np.uint64)
        base = _stream_base(seed, e)
        r1, r2 = _uniform(base, 1), _uniform(base, 2)
        us.append(np.minimum(np.searchsorted(cdf, r1, side="left"), n - 1))
        vs.append(np.minimum(np.searchsorted(cdf, r2, side="left"), n - 1))
    return to_csr(n, np.concatenate(us), np.concatenate(vs))


def write_bel(path: str, row_ptr, col) -> None:
    """.bel records {u64 dst, u64 src, u64 weight = 0}, rows in order."""
    rp = np.asarray(row_ptr, dtype=np.int64)
    c = np.asarray(col, dtype=np.int64)
    src = np.repeat(np.arange(len(rp) - 1, dtype=np.uint64), np.diff(rp))
    rec = np.zeros((len(c), 3), dtype="<u8")
    rec[:, 0] = c.astype(np.uint64)
    rec[:, 1] = src
    rec.tofile(path)


def write_mtx(path: str, edges) -> None:
    """The query file: 'n n nnz', then one 0-based 'row col' line per listed
    (directed) edge."""
    edges = [(int(a), int(b)) for a, b in edges]
    n = max(max(a, b) for a, b in edges) + 1
    with open(path, "w") as f:
        f.write(f"{n} {n} {len(edges)}\n")
        for a, b in edges:
            f.write(f"{a} {b}\n")
