"""beep_b200 — B200-native subgraph counting and enumeration (BEEP's sgm/sgc
path) behind a C ABI (include/beep.h), with ctypes bindings.

The library is the compiled CUDA code in libbeep_b200.so next to this file.
There is no CPU fallback: if the library is missing, importing the bindings
raises, and every call that reaches the device needs a CUDA GPU.

Host-side mirror of the reference's entry point:
  SG_Match(task, by, dev, cutoff, ndev).run(data_graph, query_graph)
(subgraph_matching/subgraph_matching.cuh:113-231), which prints
"------------- Counter = N" (subgraph_matching.cuh:1277).
"""
from __future__ import annotations

import ctypes
import os
from typing import Iterable, Sequence

import numpy as np

from . import patterns  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbeep_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "beep.h")

MAX_QUERY = 10

# beep_status
(OK, ERR_INVALID_ARG, ERR_IO, ERR_PARSE, ERR_UNSUPPORTED, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_TIMEOUT, ERR_INTERNAL,
 ERR_OVERFLOW) = range(10)
# counts are exact below COUNT_LIMIT; a batch slot holds COUNT_OVERFLOW for a count at or above it
COUNT_LIMIT = 0xFFF0000000000000
COUNT_OVERFLOW = 0xFFFFFFFFFFFFFFFF
NOALLOC_MAX_DOMAIN = 23168
# beep_mode
SGM, SGC = 0, 1
# options
OPT_REFERENCE_ROOT_CAP = 1 << 0
OPT_TIMING = 1 << 1
OPT_NO_VIEW_CACHE = 1 << 2
OPT_ALG_BYTES = 1 << 3
OPT_NO_GRAPH = 1 << 4
OPT_SERIAL_TIERS = 1 << 5
OPT_WAIT_STALL_TEST = 1 << 6
OPT_NO_NBHD = 1 << 7


class BeepError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_status_name(status)}: {message}")
        self.status = status


def _status_name(s: int) -> str:
    names = ["ok", "invalid argument", "i/o error", "parse error", "unsupported", "cuda error", "out of memory",
             "timeout", "internal error", "count overflow"]
    return names[s] if 0 <= s < len(names) else f"status {s}"


class GraphInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("m", ctypes.c_int64), ("max_degree", ctypes.c_int64),
                ("cutoff", ctypes.c_uint32), ("reserved", ctypes.c_int32)]


class PlanInfo(ctypes.Structure):
    _fields_ = [
        ("K", ctypes.c_int32),
        ("order", ctypes.c_int32 * MAX_QUERY),
        ("qdeg", ctypes.c_int32 * MAX_QUERY),
        ("qedge_ptr", ctypes.c_int32 * (MAX_QUERY + 1)),
        ("qedge", ctypes.c_int32 * (MAX_QUERY * (MAX_QUERY - 1) // 2)),
        ("sym_ptr", ctypes.c_int32 * (MAX_QUERY + 1)),
        ("sym", ctypes.c_int32 * (MAX_QUERY * (MAX_QUERY - 1) // 2)),
        ("unmat", ctypes.c_int32),
        ("first_sym_level", ctypes.c_int32),
        ("min_qdeg", ctypes.c_int32),
        ("max_qdeg", ctypes.c_int32),
        ("aut_order", ctypes.c_int32),
        ("restricted", ctypes.c_int32),
        ("central", ctypes.c_int32),
        ("wheel4", ctypes.c_int32),
        ("nbhd", ctypes.c_int32),
    ]


class ServeOptions(ctypes.Structure):
    _fields_ = [("max_batch", ctypes.c_uint32), ("streams", ctypes.c_uint32), ("hbm_reserve_bytes", ctypes.c_uint64),
                ("count_options", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class ServeResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("K", ctypes.c_int32), ("count", ctypes.c_uint64),
                ("n_tuples", ctypes.c_uint64), ("latency_ms", ctypes.c_double), ("queue_ms", ctypes.c_double)]


class ServeStats(ctypes.Structure):
    _fields_ = [("requests", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("matches", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint64), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("span_s", ctypes.c_double),
                ("max_batch", ctypes.c_double), ("refused", ctypes.c_uint64), ("max_inflight_bytes", ctypes.c_uint64),
                ("budget_bytes", ctypes.c_uint64)]


class Stats(ctypes.Structure):
    _fields_ = [
        ("count", ctypes.c_uint64),
        ("roots", ctypes.c_int64),
        ("roots_small", ctypes.c_int64),
        ("roots_medium", ctypes.c_int64),
        ("roots_large", ctypes.c_int64),
        ("peel_rounds", ctypes.c_int32),
        ("ascending", ctypes.c_int32),
        ("cutoff", ctypes.c_uint32),
        ("kernel_launches", ctypes.c_int32),
        ("prep_ms", ctypes.c_double),
        ("count_ms", ctypes.c_double),
        ("small_ms", ctypes.c_double),
        ("medium_ms", ctypes.c_double),
        ("large_encode_ms", ctypes.c_double),
        ("large_dfs_ms", ctypes.c_double),
        ("small_launches", ctypes.c_int32),
        ("medium_launches", ctypes.c_int32),
        ("large_encode_launches", ctypes.c_int32),
        ("large_dfs_launches", ctypes.c_int32),
        ("adjacency_bytes", ctypes.c_uint64),
        ("bitmap_bytes", ctypes.c_uint64),
        ("small_bytes", ctypes.c_uint64),
        ("medium_bytes", ctypes.c_uint64),
        ("large_bytes", ctypes.c_uint64),
        ("roots_general", ctypes.c_int64),
        ("general_ms", ctypes.c_double),
        ("general_launches", ctypes.c_int32),
        ("overflow_pairs", ctypes.c_int32),
        ("alg_small_bytes", ctypes.c_uint64),
        ("alg_medium_bytes", ctypes.c_uint64),
        ("alg_large_bytes", ctypes.c_uint64),
        ("small_tail_ms", ctypes.c_double),
        ("medium_tail_ms", ctypes.c_double),
        ("large_tail_ms", ctypes.c_double),
        ("donated_tasks", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None

# (name, restype, argtypes) of every exported function in include/beep.h
_P = ctypes.POINTER
_vp = ctypes.c_void_p
_SIGNATURES = [
    ("beep_last_error", ctypes.c_size_t, [ctypes.c_char_p, ctypes.c_size_t]),
    ("beep_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("beep_ctx_create", ctypes.c_int, [ctypes.c_int, _vp, _P(_vp)]),
    ("beep_ctx_destroy", ctypes.c_int, [_vp]),
    ("beep_ctx_set_wait_timeout", ctypes.c_int, [_vp, ctypes.c_double]),
    ("beep_ctx_kernel_launches", ctypes.c_int, [_vp, _P(ctypes.c_uint64)]),
    ("beep_graph_load_bel", ctypes.c_int, [_vp, ctypes.c_char_p, _P(_vp)]),
    ("beep_graph_from_csr", ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int64, _P(ctypes.c_int32),
                                           _P(ctypes.c_int32), _P(_vp)]),
    ("beep_graph_from_device_csr", ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int64, _vp, _vp, _P(_vp)]),
    ("beep_graph_from_edges", ctypes.c_int, [_vp, ctypes.c_int64, _P(ctypes.c_uint32), _P(ctypes.c_uint32),
                                             _P(_vp)]),
    ("beep_graph_info_get", ctypes.c_int, [_vp, _P(GraphInfo)]),
    ("beep_graph_csr", ctypes.c_int, [_vp, _P(ctypes.c_int32), _P(ctypes.c_int32)]),
    ("beep_graph_view", ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32, _P(ctypes.c_int64),
                                       _P(ctypes.c_int64), _P(ctypes.c_int32), _P(ctypes.c_int32),
                                       _P(ctypes.c_int32)]),
    ("beep_graph_destroy", ctypes.c_int, [_vp]),
    ("beep_query_load_mtx", ctypes.c_int, [ctypes.c_char_p, _P(_vp)]),
    ("beep_query_from_edges", ctypes.c_int, [ctypes.c_int32, _P(ctypes.c_int32), _P(ctypes.c_int32), _P(_vp)]),
    ("beep_query_destroy", ctypes.c_int, [_vp]),
    ("beep_query_plan", ctypes.c_int, [_vp, ctypes.c_int, _P(PlanInfo)]),
    ("beep_count", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _P(ctypes.c_uint64)]),
    ("beep_count_ex", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_uint32, _P(Stats)]),
    ("beep_count_shard", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_uint32, _P(Stats)]),
    ("beep_enumerate", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_uint64, _P(ctypes.c_int32), _P(ctypes.c_uint64),
                                      _P(ctypes.c_uint64)]),
    ("beep_batch_create", ctypes.c_int, [_vp, _P(_vp)]),
    ("beep_batch_add", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _P(ctypes.c_uint32)]),
    ("beep_batch_run", ctypes.c_int, [_vp, ctypes.c_uint32, _P(ctypes.c_uint64), _P(Stats)]),
    ("beep_batch_size", ctypes.c_int, [_vp, _P(ctypes.c_uint32)]),
    ("beep_batch_destroy", ctypes.c_int, [_vp]),
    ("beep_serve_create", ctypes.c_int, [_vp, _P(ServeOptions), _P(_vp)]),
    ("beep_serve_add_graph", ctypes.c_int, [_vp, _vp, _P(ctypes.c_int32)]),
    ("beep_serve_submit", ctypes.c_int, [_vp, ctypes.c_int32, _vp, ctypes.c_int, ctypes.c_uint64,
                                         _P(ctypes.c_uint64)]),
    ("beep_serve_wait", ctypes.c_int, [_vp, ctypes.c_uint64, _P(ServeResult), _P(ctypes.c_int32), ctypes.c_uint64]),
    ("beep_serve_drain", ctypes.c_int, [_vp]),
    ("beep_serve_stats_get", ctypes.c_int, [_vp, _P(ServeStats)]),
    ("beep_serve_destroy", ctypes.c_int, [_vp]),
    ("beep_count_noalloc", ctypes.c_int, [ctypes.c_int, _vp, ctypes.c_int64, ctypes.c_int64, _vp, _vp, _vp,
                                          ctypes.c_int, _P(ctypes.c_uint64)]),
    ("beep_gen_erdos_renyi", ctypes.c_int, [ctypes.c_int64, ctypes.c_double, ctypes.c_uint64, _P(ctypes.c_int64),
                                            _P(ctypes.c_int64), _P(ctypes.c_int32), _P(ctypes.c_int32)]),
    ("beep_gen_rmat", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_uint64, _P(ctypes.c_int64), _P(ctypes.c_int64),
                                     _P(ctypes.c_int32), _P(ctypes.c_int32)]),
    ("beep_gen_chung_lu", ctypes.c_int, [ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_uint64,
                                         _P(ctypes.c_int64), _P(ctypes.c_int64), _P(ctypes.c_int32),
                                         _P(ctypes.c_int32)]),
    ("beep_write_bel", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int64, _P(ctypes.c_int32), _P(ctypes.c_int32)]),
    ("beep_convert", ctypes.c_int, [ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p, _P(ctypes.c_uint64)]),
    ("beep_batch_autotune", ctypes.c_int, [_vp, ctypes.c_uint32, _P(ctypes.c_uint32 * 5), _P(ctypes.c_double)]),
    ("beep_batch_set_tiers", ctypes.c_int, [_vp, _P(ctypes.c_uint32 * 5)]),
]


def lib() -> ctypes.CDLL:
    """Load libbeep_b200.so. Raises if it has not been built: there is no
    fallback implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m beep_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_names() -> list[str]:
    return [n for n, _, _ in _SIGNATURES]


def last_error() -> str:
    buf = ctypes.create_string_buffer(4096)
    lib().beep_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def _check(status: int) -> None:
    if status != OK:
        raise BeepError(status, last_error())


def _i32p(a: np.ndarray):
    return a.ctypes.data_as(_P(ctypes.c_int32))


def _u32p(a: np.ndarray):
    return a.ctypes.data_as(_P(ctypes.c_uint32))


# ---------------------------------------------------------------------------
# handles
# ---------------------------------------------------------------------------
class Context:
    """A device plus a CUDA stream (cuda_stream: an integer cudaStream_t, or
    None for a stream the context owns)."""

    def __init__(self, device: int = 0, cuda_stream: int | None = None):
        h = _vp()
        _check(lib().beep_ctx_create(int(device), _vp(cuda_stream) if cuda_stream else None, ctypes.byref(h)))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def set_wait_timeout(self, ms: float) -> None:
        _check(lib().beep_ctx_set_wait_timeout(self._h, float(ms)))

    def kernel_launches(self) -> int:
        n = ctypes.c_uint64()
        _check(lib().beep_ctx_kernel_launches(self._h, ctypes.byref(n)))
        return int(n.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().beep_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Graph:
    """A data graph resident on the device (deduped CSR)."""

    def __init__(self, ctx: Context, handle):
        self.ctx = ctx
        self._h = handle

    @classmethod
    def from_csr(cls, ctx: Context, row_ptr, col_ind) -> "Graph":
        rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
        ci = np.ascontiguousarray(col_ind, dtype=np.int32)
        n = len(rp) - 1
        h = _vp()
        _check(lib().beep_graph_from_csr(ctx.handle, n, len(ci), _i32p(rp), _i32p(ci) if len(ci) else None,
                                         ctypes.byref(h)))
        return cls(ctx, h)

    @classmethod
    def from_device_csr(cls, ctx: Context, n: int, m: int, d_row_ptr: int, d_col_ind: int) -> "Graph":
        h = _vp()
        _check(lib().beep_graph_from_device_csr(ctx.handle, int(n), int(m), _vp(d_row_ptr), _vp(d_col_ind),
                                                ctypes.byref(h)))
        return cls(ctx, h)

    @classmethod
    def from_edges(cls, ctx: Context, src, dst) -> "Graph":
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        h = _vp()
        _check(lib().beep_graph_from_edges(ctx.handle, len(s), _u32p(s), _u32p(d), ctypes.byref(h)))
        return cls(ctx, h)

    @classmethod
    def load_bel(cls, ctx: Context, path: str) -> "Graph":
        h = _vp()
        _check(lib().beep_graph_load_bel(ctx.handle, os.fsencode(path), ctypes.byref(h)))
        return cls(ctx, h)

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        gi = GraphInfo()
        _check(lib().beep_graph_info_get(self._h, ctypes.byref(gi)))
        return {f: getattr(gi, f) for f, _ in GraphInfo._fields_ if f != "reserved"}

    def csr(self):
        inf = self.info()
        rp = np.zeros(inf["n"] + 1, dtype=np.int32)
        ci = np.zeros(max(inf["m"], 1), dtype=np.int32)
        _check(lib().beep_graph_csr(self._h, _i32p(rp), _i32p(ci)))
        return rp, ci[: inf["m"]]

    def view(self, min_qdeg: int, asc: bool = True):
        """The peeled, priority-relabelled CSR the counting kernels read for
        this peel threshold and order: (row_ptr, col, orig), orig[i] being
        the input id of new vertex i."""
        n, m = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().beep_graph_view(self._h, int(min_qdeg), 1 if asc else 0, ctypes.byref(n), ctypes.byref(m),
                                     None, None, None))
        rp = np.zeros(n.value + 1, dtype=np.int32)
        ci = np.zeros(max(m.value, 1), dtype=np.int32)
        orig = np.zeros(max(n.value, 1), dtype=np.int32)
        _check(lib().beep_graph_view(self._h, int(min_qdeg), 1 if asc else 0, ctypes.byref(n), ctypes.byref(m),
                                     _i32p(rp), _i32p(ci), _i32p(orig)))
        return rp, ci[: m.value], orig[: n.value]

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().beep_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Query:
    """A query graph; must have a central vertex adjacent to all others."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_edges(cls, edges: Iterable[Sequence[int]]) -> "Query":
        e = np.asarray(list(edges), dtype=np.int32).reshape(-1, 2)
        s = np.ascontiguousarray(e[:, 0])
        d = np.ascontiguousarray(e[:, 1])
        h = _vp()
        _check(lib().beep_query_from_edges(len(s), _i32p(s), _i32p(d), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def load_mtx(cls, path: str) -> "Query":
        h = _vp()
        _check(lib().beep_query_load_mtx(os.fsencode(path), ctypes.byref(h)))
        return cls(h)

    @property
    def handle(self):
        return self._h

    def plan(self, mode: int = SGM) -> dict:
        p = PlanInfo()
        _check(lib().beep_query_plan(self._h, int(mode), ctypes.byref(p)))
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
            "aut_order": p.aut_order,
            "restricted": p.restricted,
            "central": p.central,
            "wheel4": p.wheel4,
            "nbhd": p.nbhd,
        }

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().beep_query_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _as_query(q) -> Query:
    return q if isinstance(q, Query) else Query.from_edges(q)


def count(graph: Graph, query, mode: int = SGM, options: int = 0, ctx: Context | None = None,
          stats: bool = False):
    """Exact number of matches. With stats=True returns (count, stats dict)."""
    q = _as_query(query)
    st = Stats()
    _check(lib().beep_count_ex(ctx.handle if ctx else None, graph.handle, q.handle, int(mode), int(options),
                               ctypes.byref(st)))
    return (int(st.count), st.as_dict()) if stats else int(st.count)


_TUNE_KEYS = ("tiny_max", "small_max", "med_a_max", "med_max", "donate_min_iters")


def tune_cache_get(path: str, key: str) -> dict | None:
    """The tier limits stored under key in the JSON file at path, or None
    (no file, no such key, or an entry without every limit)."""
    import json

    try:
        with open(path) as f:
            entry = json.load(f).get(key)
    except (OSError, ValueError, AttributeError):
        return None
    if not isinstance(entry, dict) or any(k not in entry for k in _TUNE_KEYS):
        return None
    return {k: int(entry[k]) for k in _TUNE_KEYS} | ({"count_ms": float(entry["count_ms"])}
                                                     if "count_ms" in entry else {})


def tune_cache_put(path: str, key: str, tiers: dict) -> None:
    """Store the tier limits under key in the JSON file at path (other keys
    kept; written to a temporary file and renamed into place)."""
    import json

    try:
        with open(path) as f:
            data = json.load(f)
        if not isinstance(data, dict):
            data = {}
    except (OSError, ValueError):
        data = {}
    data[key] = {k: int(tiers[k]) for k in _TUNE_KEYS} | ({"count_ms": float(tiers["count_ms"])}
                                                          if "count_ms" in tiers else {})
    tmp = f"{path}.tmp{os.getpid()}"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


class Batch:
    """Many (graph, query, mode) pairs counted by one set of launches,
    captured into a CUDA graph on the first run and replayed afterwards."""

    def __init__(self, ctx: Context):
        h = _vp()
        _check(lib().beep_batch_create(ctx.handle, ctypes.byref(h)))
        self._h = h
        self.ctx = ctx
        self._keep = []  # graphs and queries must outlive the batch

    def add(self, graph: Graph, query, mode: int = SGM) -> int:
        q = _as_query(query)
        idx = ctypes.c_uint32()
        _check(lib().beep_batch_add(self._h, graph.handle, q.handle, int(mode), ctypes.byref(idx)))
        self._keep.append((graph, q))
        return int(idx.value)

    def __len__(self) -> int:
        n = ctypes.c_uint32()
        _check(lib().beep_batch_size(self._h, ctypes.byref(n)))
        return int(n.value)

    def run(self, options: int = 0, stats: bool = False):
        n = len(self)
        counts = (ctypes.c_uint64 * max(n, 1))()
        st = Stats()
        _check(lib().beep_batch_run(self._h, int(options), counts, ctypes.byref(st)))
        out = [int(counts[i]) for i in range(n)]
        return (out, st.as_dict()) if stats else out

    TIER_KEYS = ("tiny_max", "small_max", "med_a_max", "med_max", "donate_min_iters")

    def autotune(self, options: int = 0, cache: str | None = None, key: str | None = None) -> dict:
        """Pick the tier limits (bitmap word width and lanes per root by
        domain size, and the large tier's donation threshold) by measurement
        (beep_batch_autotune); returns them with the best counting time in
        ms. With cache (a JSON file) and key (a name for this workload), a
        choice stored there under key is applied without measuring, and a new
        one is stored under key, so a deployment tunes once per workload."""
        if cache is not None and key is not None:
            got = tune_cache_get(cache, key)
            if got is not None:
                self.set_tiers(got)
                return {**got, "cached": True}
        cfg = (ctypes.c_uint32 * 5)()
        ms = ctypes.c_double()
        _check(lib().beep_batch_autotune(self._h, int(options), ctypes.byref(cfg), ctypes.byref(ms)))
        out = {**dict(zip(self.TIER_KEYS, list(cfg))), "count_ms": ms.value}
        if cache is not None and key is not None:
            tune_cache_put(cache, key, out)
        return out

    def set_tiers(self, tiers: dict) -> None:
        vals = [int(tiers[k]) for k in self.TIER_KEYS[:4]] + [int(tiers.get("donate_min_iters", 2))]
        cfg = (ctypes.c_uint32 * 5)(*vals)
        _check(lib().beep_batch_set_tiers(self._h, ctypes.byref(cfg)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().beep_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request server over resident graphs with continuous batching."""

    def __init__(self, ctx: Context, max_batch: int = 0, streams: int = 0, hbm_reserve_bytes: int = 0,
                 count_options: int = 0):
        opt = ServeOptions(max_batch, streams, hbm_reserve_bytes, count_options, 0)
        h = _vp()
        _check(lib().beep_serve_create(ctx.handle, ctypes.byref(opt), ctypes.byref(h)))
        self._h = h
        self.ctx = ctx
        self._keep = []
        self._queries = {}

    def add_graph(self, graph: Graph) -> int:
        gid = ctypes.c_int32()
        _check(lib().beep_serve_add_graph(self._h, graph.handle, ctypes.byref(gid)))
        self._keep.append(graph)
        return int(gid.value)

    def submit(self, graph_id: int, query, mode: int = SGM, k: int = 0) -> int:
        q = query if isinstance(query, Query) else self._queries.setdefault(id(query), Query.from_edges(query))
        rid = ctypes.c_uint64()
        _check(lib().beep_serve_submit(self._h, int(graph_id), q.handle, int(mode), int(k), ctypes.byref(rid)))
        return int(rid.value)

    def wait(self, request_id: int, k: int = 0):
        res = ServeResult()
        buf = None
        if k > 0:
            buf = np.zeros((k, MAX_QUERY), dtype=np.int32)
        st = lib().beep_serve_wait(self._h, int(request_id), ctypes.byref(res), _i32p(buf) if buf is not None else None,
                                   int(k))
        _check(st)
        out = {"count": int(res.count), "latency_ms": res.latency_ms, "queue_ms": res.queue_ms, "K": res.K}
        if buf is not None:
            flat = buf.reshape(-1)[: int(res.n_tuples) * res.K]
            out["tuples"] = flat.reshape(-1, res.K) if res.K else flat.reshape(0, 0)
        return out

    def drain(self) -> None:
        _check(lib().beep_serve_drain(self._h))

    def stats(self) -> dict:
        st = ServeStats()
        _check(lib().beep_serve_stats_get(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in ServeStats._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().beep_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def count_noalloc(device: int, n: int, m: int, d_row_ptr: int, d_col_ind: int, query, mode: int = SGM,
                  cuda_stream: int | None = None) -> int:
    """Count through the allocation-free entry point on a device CSR (sorted,
    simple rows) given by device pointers."""
    q = _as_query(query)
    out = ctypes.c_uint64()
    _check(lib().beep_count_noalloc(int(device), _vp(cuda_stream) if cuda_stream else None, int(n), int(m),
                                    _vp(d_row_ptr), _vp(d_col_ind), q.handle, int(mode), ctypes.byref(out)))
    return int(out.value)


def count_shard(graph: Graph, query, shard: int, nshards: int, mode: int = SGM, options: int = 0,
                ctx: Context | None = None, stats: bool = False):
    """Count of the roots whose input vertex id % nshards == shard. With
    stats=True returns (count, stats dict)."""
    q = _as_query(query)
    st = Stats()
    _check(lib().beep_count_shard(ctx.handle if ctx else None, graph.handle, q.handle, int(mode), int(options),
                                  int(shard), int(nshards), ctypes.byref(st)))
    return (int(st.count), st.as_dict()) if stats else int(st.count)


def enumerate_matches(graph: Graph, query, k: int, ctx: Context | None = None):
    """Up to k matches as an int32 array [n, K] in original query-vertex order,
    plus the exact total count."""
    q = _as_query(query)
    K = q.plan()["K"]
    out = np.zeros((max(int(k), 1), K), dtype=np.int32)
    n_out = ctypes.c_uint64()
    total = ctypes.c_uint64()
    _check(lib().beep_enumerate(ctx.handle if ctx else None, graph.handle, q.handle, int(k), _i32p(out),
                                ctypes.byref(n_out), ctypes.byref(total)))
    return out[: n_out.value], int(total.value)


# ---------------------------------------------------------------------------
# synthetic graphs
# ---------------------------------------------------------------------------
def _gen(fn, *args):
    n = ctypes.c_int64()
    m = ctypes.c_int64()
    _check(fn(*args, ctypes.byref(n), ctypes.byref(m), None, None))
    rp = np.zeros(n.value + 1, dtype=np.int32)
    ci = np.zeros(max(m.value, 1), dtype=np.int32)
    _check(fn(*args, ctypes.byref(n), ctypes.byref(m), _i32p(rp), _i32p(ci)))
    return rp, ci[: m.value]


def gen_erdos_renyi(n: int, p: float, seed: int):
    """G(n, p): each pair independently with probability p. Returns (row_ptr, col)."""
    return _gen(lib().beep_gen_erdos_renyi, int(n), float(p), int(seed))


def gen_rmat(scale: int, edge_factor: int, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 0):
    """R-MAT with 2^scale vertices and edge_factor * 2^scale sampled edges,
    symmetrised, loops and duplicates removed. Returns (row_ptr, col)."""
    return _gen(lib().beep_gen_rmat, int(scale), int(edge_factor), float(a), float(b), float(c), int(seed))


def gen_chung_lu(n: int, avg_degree: float, exponent: float, seed: int):
    """Chung-Lu power-law graph. Returns (row_ptr, col)."""
    return _gen(lib().beep_gen_chung_lu, int(n), float(avg_degree), float(exponent), int(seed))


def write_bel(path: str, row_ptr, col_ind) -> None:
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    ci = np.ascontiguousarray(col_ind, dtype=np.int32)
    _check(lib().beep_write_bel(os.fsencode(path), len(rp) - 1, _i32p(rp), _i32p(ci) if len(ci) else None))


def write_mtx(path: str, edges) -> None:
    with open(path, "w") as f:
        f.write(patterns.to_mtx(list(edges)))


# ---------------------------------------------------------------------------
# reference-shaped entry point
# ---------------------------------------------------------------------------
GRAPH_MATCH = "sgm"
GRAPH_COUNT = "sgc"


class SG_Match:
    """Mirror of graph::SG_Match<uint>(MAINTASK task, ProcessBy by, int dev,
    uint cutoff, int ndev) (subgraph_matching.cuh:113-145). `by` and `cutoff`
    are accepted for signature parity: the cutoff is recomputed from the data
    graph's degrees as the reference's main() does (src/main.cu:132); only one
    device per process is supported (ndev must be 1)."""

    def __init__(self, task: str = GRAPH_MATCH, by: str = "node", dev: int = 0, cutoff: int = 768, ndev: int = 1):
        if task not in (GRAPH_MATCH, GRAPH_COUNT):
            raise ValueError(f"Unrecognized -mt option (Main TASK): {task}")
        if ndev != 1:
            raise ValueError("one device per process (ndev must be 1)")
        self.task = task
        self.dev = dev
        self.ctx = Context(dev)
        self.last_stats: dict | None = None

    def run(self, data_graph, query_graph, verbose: bool = True) -> int:
        """Count matches of query_graph (Query or edge list) in data_graph
        (Graph or (row_ptr, col) host CSR). Prints the reference's result line."""
        g = data_graph if isinstance(data_graph, Graph) else Graph.from_csr(self.ctx, *data_graph)
        c, st = count(g, query_graph, SGC if self.task == GRAPH_COUNT else SGM, OPT_TIMING, ctx=self.ctx,
                      stats=True)
        self.last_stats = st
        if verbose:
            print(f"------------- Counter = {c}")
        return c


# the reference's -m converter tasks (src/main.cu:40-67)
CONVERT_TASKS = {"txt-bel": 0, "mtx-bel": 1, "tsv-bel": 2, "tsv-mtx": 3, "bel-mtx": 4}


def convert(task: str, src_path: str, dst_path: str) -> int:
    """Convert a graph file as the reference's `-m <task> -g src -r dst` does
    (graph::MtB_Writer, include/FIleReader.cuh:456-912). Returns the records
    (or Matrix Market entries) written."""
    if task not in CONVERT_TASKS:
        raise BeepError(ERR_INVALID_ARG, f"unknown converter task {task!r}")
    n = ctypes.c_uint64(0)
    _check(lib().beep_convert(CONVERT_TASKS[task], os.fsencode(src_path), os.fsencode(dst_path), ctypes.byref(n)))
    return int(n.value)
