"""ctypes wrapper around the CPU oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py to check the CUDA path. The product never
imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

OR_DEPTH = 10


class OrPlan(ctypes.Structure):
    _fields_ = [
        ("K", ctypes.c_int32),
        ("order", ctypes.c_int32 * OR_DEPTH),
        ("qdeg", ctypes.c_int32 * OR_DEPTH),
        ("qedge_ptr", ctypes.c_int32 * (OR_DEPTH + 1)),
        ("qedge", ctypes.c_int32 * (OR_DEPTH * (OR_DEPTH - 1) // 2)),
        ("sym_ptr", ctypes.c_int32 * (OR_DEPTH + 1)),
        ("sym", ctypes.c_int32 * (OR_DEPTH * (OR_DEPTH - 1) // 2)),
        ("unmat", ctypes.c_int32),
        ("first_sym_level", ctypes.c_int32),
        ("min_qdeg", ctypes.c_int32),
        ("max_qdeg", ctypes.c_int32),
        ("central", ctypes.c_int32),
        ("aut_order", ctypes.c_int32),
    ]


class OrOptions(ctypes.Structure):
    _fields_ = [
        ("apply_root_cap", ctypes.c_int32),
        ("full_depth", ctypes.c_int32),
        ("root_stride", ctypes.c_int64),
        ("root_offset", ctypes.c_int64),
        ("threads", ctypes.c_int32),
        ("root_mod", ctypes.c_int64),
        ("root_rem", ctypes.c_int64),
    ]


class OrResult(ctypes.Structure):
    _fields_ = [
        ("count", ctypes.c_uint64),
        ("roots", ctypes.c_int64),
        ("roots_processed", ctypes.c_int64),
        ("cutoff", ctypes.c_uint32),
        ("peel_rounds", ctypes.c_int32),
        ("ascending", ctypes.c_int32),
        ("q2_risk", ctypes.c_int32),
        ("q3_skipped", ctypes.c_int64),
    ]


_lib = None


def build() -> str:
    """Compile liboracle.so with the Makefile next to this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        L.or_plan_query.argtypes = [ctypes.c_int32, P(ctypes.c_int32), P(ctypes.c_int32), ctypes.c_int32, P(OrPlan)]
        L.or_plan_query.restype = ctypes.c_int
        L.or_cutoff.argtypes = [ctypes.c_int64, P(ctypes.c_int64)]
        L.or_cutoff.restype = ctypes.c_uint32
        L.or_peel.argtypes = [ctypes.c_int64, P(ctypes.c_int64), P(ctypes.c_int32), ctypes.c_int32,
                              P(ctypes.c_int32), P(ctypes.c_uint8)]
        L.or_peel.restype = ctypes.c_int32
        L.or_count.argtypes = [ctypes.c_int64, P(ctypes.c_int64), P(ctypes.c_int32), P(OrPlan), ctypes.c_int32,
                               P(OrOptions), P(OrResult)]
        L.or_count.restype = ctypes.c_int
        L.or_enumerate.argtypes = [ctypes.c_int64, P(ctypes.c_int64), P(ctypes.c_int32), P(OrPlan),
                                   P(ctypes.c_int32), ctypes.c_int64]
        L.or_enumerate.restype = ctypes.c_int64
        L.or_count_cliques.argtypes = [ctypes.c_int64, P(ctypes.c_int64), P(ctypes.c_int32), ctypes.c_int32,
                                       ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32]
        L.or_count_cliques.restype = ctypes.c_uint64
        L.or_brute_force.argtypes = [ctypes.c_int64, P(ctypes.c_int64), P(ctypes.c_int32), ctypes.c_int32,
                                     P(ctypes.c_int32), P(ctypes.c_int32)]
        L.or_brute_force.restype = ctypes.c_uint64
        _lib = L
    return _lib


def _i32p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _i64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


def query_csr(edges):
    """Query CSR as CSRCOO::from_edgelist builds it (include/CSRCOO.cuh:37-80):
    self loops dropped, n = max src + 1, rows in src order (edges are sorted
    by src first; the reference asserts that order), file order within a row."""
    edges = [(int(a), int(b)) for a, b in edges if int(a) != int(b)]
    edges.sort(key=lambda e: e[0])  # stable: keeps file order within a row
    n = max(a for a, _ in edges) + 1
    rp = np.zeros(n + 1, dtype=np.int32)
    for a, _ in edges:
        rp[a + 1] += 1
    rp = np.cumsum(rp).astype(np.int32)
    col = np.array([b for _, b in edges], dtype=np.int32)
    return n, rp, col


def plan(edges, sgc=False) -> dict:
    n, rp, col = query_csr(edges)
    p = OrPlan()
    rc = lib().or_plan_query(n, _i32p(rp), _i32p(col), int(bool(sgc)), ctypes.byref(p))
    if rc != 0:
        raise ValueError(f"unsupported query (or_plan_query returned {rc})")
    K = p.K
    return {
        "K": K,
        "order": list(p.order[:K]),
        "qdeg": list(p.qdeg[:K]),
        "qedge_ptr": list(p.qedge_ptr[: K + 1]),
        "qedge": list(p.qedge[: p.qedge_ptr[K]]),
        "sym_ptr": list(p.sym_ptr[: K + 1]),
        "sym": list(p.sym[: p.sym_ptr[K]]),
        "unmat": p.unmat,
        "first_sym_level": p.first_sym_level,
        "min_qdeg": p.min_qdeg,
        "max_qdeg": p.max_qdeg,
        "central": p.central,
        "aut_order": p.aut_order,
        "_raw": p,
    }


def _graph_arrays(row_ptr, col):
    rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
    c = np.ascontiguousarray(col, dtype=np.int32)
    return len(rp) - 1, rp, c


def count(row_ptr, col, query_edges, sgc=False, apply_root_cap=True, full_depth=False,
          root_stride=1, root_offset=0, threads=0, root_mod=0, root_rem=0) -> dict:
    n, rp, c = _graph_arrays(row_ptr, col)
    p = plan(query_edges, sgc)["_raw"]
    opt = OrOptions(int(apply_root_cap), int(full_depth), int(root_stride), int(root_offset), int(threads),
                    int(root_mod), int(root_rem))
    res = OrResult()
    rc = lib().or_count(n, _i64p(rp), _i32p(c), ctypes.byref(p), int(bool(sgc)), ctypes.byref(opt),
                        ctypes.byref(res))
    if rc != 0:
        raise ValueError(f"or_count failed ({rc})")
    return {f: getattr(res, f) for f, _ in OrResult._fields_}


def enumerate_matches(row_ptr, col, query_edges, cap=None) -> np.ndarray:
    n, rp, c = _graph_arrays(row_ptr, col)
    p = plan(query_edges, False)["_raw"]
    if cap is None:
        cap = int(count(row_ptr, col, query_edges, apply_root_cap=False)["count"])
    out = np.zeros((max(cap, 1), p.K), dtype=np.int32)
    got = lib().or_enumerate(n, _i64p(rp), _i32p(c), ctypes.byref(p), _i32p(out), int(cap))
    if got < 0:
        raise ValueError("or_enumerate failed")
    return out[: min(got, cap)]


def count_cliques(row_ptr, col, k, root_mod=0, root_rem=0, threads=0) -> int:
    """Independent k-clique count (recursive intersection on the peeled
    degree order, peel threshold k-1 as for a k-clique query), restricted to
    lowest vertices with id % root_mod == root_rem."""
    n, rp, c = _graph_arrays(row_ptr, col)
    return int(lib().or_count_cliques(n, _i64p(rp), _i32p(c), int(k), int(k) - 1, int(root_mod), int(root_rem),
                                      int(threads)))


def brute_force(row_ptr, col, query_edges) -> int:
    n, rp, c = _graph_arrays(row_ptr, col)
    qn, qrp, qcol = query_csr(query_edges)
    return int(lib().or_brute_force(n, _i64p(rp), _i32p(c), qn, _i32p(qrp), _i32p(qcol)))


def peel(row_ptr, col, min_qdeg):
    n, rp, c = _graph_arrays(row_ptr, col)
    deg = np.zeros(max(n, 1), dtype=np.int32)
    alive = np.zeros(max(n, 1), dtype=np.uint8)
    rounds = lib().or_peel(n, _i64p(rp), _i32p(c), int(min_qdeg), _i32p(deg),
                           alive.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    return deg[:n], alive[:n].astype(bool), rounds


def view(row_ptr, col, min_qdeg, asc=True):
    """The peeled, priority-relabelled CSR: or_peel, then every vertex that
    kept an edge in build_rank's order (ascending (degree, id), or descending
    degree with ties by ascending id; subgraph_matching.cuh:1282-1336,
    host_utils.cuh:230-246) and each row the sorted new ids of its kept
    neighbours. Returns int32 (row_ptr, col, orig)."""
    deg, keep, _ = peel(row_ptr, col, min_qdeg)
    rp = np.asarray(row_ptr, dtype=np.int64)
    c = np.asarray(col, dtype=np.int64)
    n = len(rp) - 1
    ids = np.nonzero(keep)[0].astype(np.int64)
    d = deg[ids].astype(np.int64)
    orig = ids[np.lexsort((ids, d if asc else -d))]
    rank = np.full(max(n, 1), -1, dtype=np.int64)
    rank[orig] = np.arange(len(orig), dtype=np.int64)
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    ok = (rank[src] >= 0) & (rank[c] >= 0)
    keys = np.sort((rank[src][ok] << np.int64(32)) | rank[c][ok])
    nrp = np.zeros(len(orig) + 1, dtype=np.int64)
    nrp[1:] = np.cumsum(np.bincount(keys >> np.int64(32), minlength=len(orig)))
    return nrp.astype(np.int32), (keys & np.int64(0xFFFFFFFF)).astype(np.int32), orig.astype(np.int32)


def cutoff(row_ptr) -> int:
    rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
    return int(lib().or_cutoff(len(rp) - 1, _i64p(rp)))
