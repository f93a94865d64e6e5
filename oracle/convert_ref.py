"""Test infrastructure only: a plain-Python restatement of the reference's
graph-file converters (src/main.cu:40-67 over graph::MtB_Writer,
include/FIleReader.cuh:456-912), the checker for beep_convert.

Each function returns the bytes the reference writes for an input file, or
raises ValueError where the reference cannot finish (reads past an empty edge
list, uninitialised sizes) and the library reports an error instead. Integer
parsing follows C's sscanf/fscanf with %llu / %lld as the reference uses them.
"""
from __future__ import annotations

import re
import struct

_U64 = (1 << 64) - 1
_U32 = (1 << 32) - 1


def _scan_ull(tok: str):
    """strtoull-like parse of one %llu token: optional sign, decimal digits;
    a leading '-' wraps modulo 2^64; overflow saturates to 2^64-1."""
    m = re.match(r"[+-]?\d+", tok)
    if not m:
        return None, tok
    s = m.group(0)
    v = int(s)
    if v > _U64 or v < -_U64:
        v = _U64
    elif v < 0:
        v = (v + (1 << 64)) & _U64
    return v, tok[m.end():]


def _scan_ll(tok: str):
    """strtoll-like parse of one %lld token (saturating)."""
    m = re.match(r"[+-]?\d+", tok)
    if not m:
        return None, tok
    v = int(m.group(0))
    v = max(min(v, (1 << 63) - 1), -(1 << 63))
    return v, tok[m.end():]


def _sscanf_ints(line: str, k: int, signed: bool):
    """Leading integers of `line` as sscanf("%lld %lld ...") reads them:
    whitespace skipped before each, stop at the first that fails."""
    out = []
    rest = line
    for _ in range(k):
        rest = rest.lstrip(" \t\n\r\v\f")
        v, rest2 = (_scan_ll if signed else _scan_ull)(rest)
        if v is None:
            break
        out.append(v)
        rest = rest2
    return out


def _sscanf_mtx_entry(line: str, with_value: bool):
    """sscanf(line, "%lld %lld %lf") / ("%lld %lld"): number of conversions."""
    vals = _sscanf_ints(line, 2, signed=True)
    if len(vals) < 2 or not with_value:
        if not vals and not line.strip():
            return -1, vals  # EOF: nothing but whitespace
        return len(vals), vals
    rest = line
    for _ in range(2):  # skip the two integers
        rest = rest.lstrip(" \t\n\r\v\f")
        _, rest = _scan_ll(rest)
    rest = rest.lstrip(" \t\n\r\v\f")
    m = re.match(r"[+-]?((\d+\.?\d*|\.\d+)([eE][+-]?\d+)?|inf|nan)", rest, re.I)
    return (3 if m else 2), vals


def _bel(pairs) -> bytes:
    """Records {u64 dst, u64 src, u64 0} for (src, dst) pairs
    (FIleReader.cuh:627-633)."""
    return b"".join(struct.pack("<QQQ", d, s, 0) for s, d in pairs)


def txt_bel(text: str) -> bytes:
    """write_txt_bel<uint, uint>(makeFull=true, numCol=2, srcIndex=0)
    (main.cu:64-66, FIleReader.cuh:816-907). Empty lines are skipped (the
    reference's fscanf loop cannot move past one)."""
    e = []
    for line in text.split("\n"):
        if line == "" or line[0] == "%":
            continue
        v = _sscanf_ints(line, 2, signed=False)
        if len(v) == 2 and v[0] != v[1]:
            a, b = v[0] & _U32, v[1] & _U32
            e.append((a, b))
            e.append((b, a))
    return _bel(sorted(set(e)))


def mtx_bel(text: str) -> bytes:
    """write_market_bel<uint, int>(makeFull=false) (main.cu:40-43,
    FIleReader.cuh:461-641)."""
    lines = text.split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    it = iter(lines)
    symmetric = array = pattern = False
    size_line = None
    for line in it:
        if line == "" or line[0] != "%":
            size_line = line
            break
        if len(line) >= 2:
            symmetric = "symmetric" in line
            array = "array" in line
            pattern = "pattern" in line
    if size_line is None:
        raise ValueError("invalid problem description")
    hdr = _sscanf_ints(size_line, 3, signed=True)
    if array and len(hdr) == 2:
        nx, nnz = hdr[0], hdr[0] * hdr[1]
    elif not array and len(hdr) == 3:
        if hdr[0] != hdr[1]:
            raise ValueError("not square")
        nx, nnz = hdr[0], hdr[2]
    else:
        raise ValueError("invalid problem description")
    nodes, entries = nx & _U32, nnz & _U32  # both held in 32-bit unsigned variables
    e = []
    for i in range(entries):
        line = next(it, "")
        k, v = _sscanf_mtx_entry(line, with_value=not pattern)
        if array and k == 1:
            c = i // nodes
            r = i - nodes * c
        elif array or (k < 2 if not pattern else k != 2):
            break
        else:
            r, c = v
        e.append((r & _U32, c & _U32))
        if symmetric and c != r:
            e.append((c & _U32, r & _U32))
    return _bel(sorted(e))


def _fscanf_triples(text: str):
    """fscanf(fp, "%llu %llu %llu") repeated until it fails."""
    toks = text.split()
    out = []
    i = 0
    while i + 3 <= len(toks):
        vals = []
        for t in toks[i:i + 3]:
            v, rest = _scan_ull(t)
            if v is None:
                return out
            vals.append(v)
            if rest:  # a token with trailing garbage stops the next conversion
                if len(vals) == 3:
                    out.append(tuple(vals))
                return out
        out.append(tuple(vals))
        i += 3
    return out


def tsv_bel(text: str) -> bytes:
    """write_tsv_bel<uint64, uint64> (main.cu:46-50, FIleReader.cuh:324-381):
    "dst src weight" triples, written in file order."""
    return _bel((s, d) for d, s, _ in _fscanf_triples(text))


def _market(pairs, weights) -> str:
    if not pairs:
        raise ValueError("no edges")
    n = pairs[-1][0]
    out = ["%%MatrixMarket matrix coordinate general", f"{n} {n} {len(pairs)}"]
    out += [f"{s} {d} {w}" for (s, d), w in zip(pairs, weights)]
    return "\n".join(out) + "\n"


def _as_int32(x: int) -> int:
    x &= _U32
    return x - (1 << 32) if x >= (1 << 31) else x


def tsv_mtx(text: str) -> str:
    """write_tsv_market<uint, int> (main.cu:52-56, FIleReader.cuh:706-753)."""
    t = _fscanf_triples(text)
    return _market([(s & _U32, d & _U32) for d, s, _ in t], [_as_int32(w) for _, _, w in t])


def bel_mtx(data: bytes) -> str:
    """write_bel_market<uint, int> (main.cu:58-62, FIleReader.cuh:757-813)."""
    nrec = len(data) // 24
    recs = [struct.unpack_from("<QQQ", data, 24 * i) for i in range(nrec)]
    return _market([(s & _U32, d & _U32) for d, s, _ in recs], [_as_int32(w) for _, _, w in recs])
