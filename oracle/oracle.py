"""ctypes wrapper of the CPU oracle (``oracle/fgss_oracle.c``).

TEST INFRASTRUCTURE ONLY: the checker the CUDA path is compared against.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product path never does.

Functions take and return numpy arrays.  Record arrays are in the reference's
MEMORY order (``src/fgssjoin/data.cu:97-113``: the .bin order reversed, so
descending size) unless a docstring says FILE order.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libfgss_oracle.so")
_lib = None


class _Pair(ctypes.Structure):
    _fields_ = [("q", ctypes.c_uint32), ("s", ctypes.c_uint32),
                ("overlap", ctypes.c_uint32), ("sim", ctypes.c_float)]


class _Stats(ctypes.Structure):
    _fields_ = [("candidates", ctypes.c_uint64), ("intersections", ctypes.c_uint64),
                ("results", ctypes.c_uint64), ("index_entries", ctypes.c_uint64),
                ("probe_entries", ctypes.c_uint64)]


def build():
    """Compile the oracle with its Makefile (gcc, strict IEEE float)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        u32p = P(ctypes.c_uint32)
        L.orc_tokenize.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   P(ctypes.c_uint32), P(ctypes.c_uint64), P(ctypes.c_uint32),
                                   P(u32p), P(u32p), P(u32p), P(u32p)]
        L.orc_tokenize.restype = ctypes.c_int
        L.orc_join.argtypes = [u32p, u32p, u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                               ctypes.c_uint32, ctypes.c_int, P(P(_Pair)), P(_Stats), ctypes.c_int,
                               P(u32p), P(ctypes.c_uint64), ctypes.c_uint32, ctypes.c_uint32,
                               P(ctypes.c_uint8), ctypes.c_uint32, ctypes.c_uint32]
        L.orc_join.restype = ctypes.c_int64
        L.orc_brute.argtypes = [u32p, u32p, u32p, ctypes.c_uint32, ctypes.c_float, P(P(_Pair))]
        L.orc_brute.restype = ctypes.c_int64
        L.orc_free.argtypes = [ctypes.c_void_p]
        for name in ("orc_max_prefix", "orc_mid_prefix", "orc_min_size", "orc_max_size"):
            f = getattr(L, name)
            f.argtypes = [ctypes.c_float, ctypes.c_uint32]
            f.restype = ctypes.c_uint32
        L.orc_min_overlap.argtypes = [ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_min_overlap.restype = ctypes.c_float
        L.orc_similarity.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_similarity.restype = ctypes.c_float
        L.orc_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def _take(ptr, n, dtype=np.uint32):
    if n == 0:
        out = np.zeros(0, dtype=dtype)
    else:
        out = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)
    lib().orc_free(ptr)
    return out


def tokenize(text, q=3, mode="qgram", pad=False, pad_char=1, suffix=True, lower=True):
    """Text -> (ids, lens, tokens, locs, n_terms) in FILE order (ascending size).

    mode "qgram": q-grams of each non-empty line; ``pad`` adds q-1 copies of
    ``pad_char`` on both sides; ``suffix`` numbers repeated grams as distinct
    tokens (qgram.cpp:27-44) instead of keeping only the first.
    mode "kmer": canonical k-mers (k = q) of ACGT lines, distinct per line.
    """
    if isinstance(text, str):
        text = text.encode("latin-1")
    L = lib()
    ns = ctypes.c_uint32(); nt = ctypes.c_uint64(); nterm = ctypes.c_uint32()
    pi = ctypes.POINTER(ctypes.c_uint32)()
    pl = ctypes.POINTER(ctypes.c_uint32)()
    pt = ctypes.POINTER(ctypes.c_uint32)()
    po = ctypes.POINTER(ctypes.c_uint32)()
    rc = L.orc_tokenize(text, len(text), q, 1 if mode == "kmer" else 0, int(pad), pad_char,
                        int(suffix), int(lower), ctypes.byref(ns), ctypes.byref(nt), ctypes.byref(nterm),
                        ctypes.byref(pi), ctypes.byref(pl), ctypes.byref(pt), ctypes.byref(po))
    if rc != 0:
        raise ValueError("orc_tokenize failed: %d" % rc)
    return (_take(pi, ns.value), _take(pl, ns.value), _take(pt, nt.value), _take(po, nt.value),
            nterm.value)


def file_to_memory(ids, lens, tokens):
    """FILE order -> MEMORY order (data.cu:97-113): records reversed; returns id, pos, len, tokens."""
    ids = np.asarray(ids, dtype=np.uint32)
    lens = np.asarray(lens, dtype=np.uint32)
    tokens = np.asarray(tokens, dtype=np.uint32)
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    order = np.arange(len(lens))[::-1]
    mid = ids[order].copy()
    mlen = lens[order].copy()
    if len(tokens):
        idx = np.concatenate([np.arange(off[i], off[i + 1]) for i in order]) if len(order) else np.zeros(0, np.int64)
        mtok = tokens[idx].copy()
    else:
        mtok = tokens.copy()
    mpos = np.zeros(len(mlen), dtype=np.uint32)
    if len(mlen) > 1:
        mpos[1:] = np.cumsum(mlen[:-1])
    return mid, mpos, mlen, mtok


def decode_bin(raw):
    """ppjoin .bin bytes -> (ids, lens, tokens) in FILE order (data.cu:53-89)."""
    a = np.frombuffer(raw, dtype="<i4")
    ids, lens, toks = [], [], []
    i = 0
    while i < len(a):
        ids.append(a[i]); n = int(a[i + 1]); lens.append(n)
        toks.append(a[i + 2:i + 2 + n]); i += 2 + n
    tok = np.concatenate(toks).astype(np.uint32) if toks else np.zeros(0, np.uint32)
    return np.array(ids, dtype=np.uint32), np.array(lens, dtype=np.uint32), tok


def encode_bin(ids, lens, tokens):
    """(ids, lens, tokens) in FILE order -> ppjoin .bin bytes."""
    out = []
    off = 0
    for i, n in zip(ids, lens):
        out.append(np.array([i, n], dtype="<i4"))
        out.append(np.asarray(tokens[off:off + n], dtype="<i4"))
        off += int(n)
    return np.concatenate(out).tobytes() if out else b""


def join(pos, lens, tokens, n_terms, t, block_size=0, threads=0, want_candidates=False, query_range=None,
         side=None, query_step=1, query_phase=0):
    """Reference-semantics self-join on MEMORY-order records.
    ``query_step`` > 1 restricts the queries to every query_step-th one (from
    ``query_phase``): a strided sample for bounded CPU timing.

    Returns (pairs, stats[, candidates]) where pairs is a structured array
    (q, s, overlap, sim) sorted by (q, s) in memory indices and stats a dict
    with the reference's counters.  ``candidates`` is an (n, 3) array of
    (q, s, partial score) for every cell with score > 0 after filtering.
    """
    L = lib()
    pos_a, pp = _u32(pos)
    len_a, lp = _u32(lens)
    tok_a, tp = _u32(tokens if len(tokens) else np.zeros(1, np.uint32))
    out = ctypes.POINTER(_Pair)()
    st = _Stats()
    cptr = ctypes.POINTER(ctypes.c_uint32)()
    ncand = ctypes.c_uint64()
    nthreads = threads if threads > 0 else L.orc_num_threads()
    qb, qe = query_range if query_range else (0, 0)
    side_p = None
    if side is not None:
        side_a = np.ascontiguousarray(side, dtype=np.uint8)
        side_p = side_a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    n = L.orc_join(pp, lp, tp, len(len_a), int(n_terms), ctypes.c_float(t), block_size, nthreads,
                   ctypes.byref(out), ctypes.byref(st), int(want_candidates), ctypes.byref(cptr),
                   ctypes.byref(ncand), int(qb), int(qe), side_p, int(query_step), int(query_phase))
    if n < 0:
        raise ValueError("orc_join failed: %d" % n)
    pairs = _pairs(out, n)
    stats = {k: int(getattr(st, k)) for k, _ in _Stats._fields_}
    if want_candidates:
        c = _take(cptr, 3 * ncand.value).reshape(-1, 3) if ncand.value else np.zeros((0, 3), np.uint32)
        if not ncand.value and cptr:
            L.orc_free(cptr)
        return pairs, stats, c
    return pairs, stats


PAIR_DTYPE = np.dtype([("q", "<u4"), ("s", "<u4"), ("overlap", "<u4"), ("sim", "<f4")])


def _pairs(ptr, n):
    if n == 0:
        if ptr:
            lib().orc_free(ptr)
        return np.zeros(0, dtype=PAIR_DTYPE)
    buf = ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint8 * (16 * n))).contents
    arr = np.frombuffer(bytes(buf), dtype=PAIR_DTYPE).copy()
    lib().orc_free(ptr)
    return arr


def brute(pos, lens, tokens, t):
    """All-pairs checker without filters (same final tests as the reference)."""
    L = lib()
    pos_a, pp = _u32(pos)
    len_a, lp = _u32(lens)
    tok_a, tp = _u32(tokens if len(tokens) else np.zeros(1, np.uint32))
    out = ctypes.POINTER(_Pair)()
    n = L.orc_brute(pp, lp, tp, len(len_a), ctypes.c_float(t), ctypes.byref(out))
    return _pairs(out, n)


def bounds_table(t, maxlen):
    """Per-length float32 bounds of similarity.cuh: (max_prefix, mid_prefix, min_size, max_size)."""
    L = lib()
    ft = ctypes.c_float(t)
    n = np.arange(maxlen + 1)
    return (np.array([L.orc_max_prefix(ft, int(i)) for i in n], np.uint32),
            np.array([L.orc_mid_prefix(ft, int(i)) for i in n], np.uint32),
            np.array([L.orc_min_size(ft, int(i)) for i in n], np.uint32),
            np.array([L.orc_max_size(ft, int(i)) for i in n], np.uint32))


def tokenize_dual(text_r, text_s, **tok):
    """Oracle tokenization of R's text then S's text as one input (one shared
    vocabulary), split into the two sides the way fgss_tokenize_dual splits
    them: ((id, pos, len, tokens) of R, the same of S, n_terms), MEMORY order,
    ids counting the non-empty lines of each side's own text."""
    if text_r and not text_r.endswith(b"\n"):
        text_r = text_r + b"\n"
    nr = sum(1 for x in text_r.split(b"\n") if x)
    ids, lens, tok_, loc, nt = tokenize(text_r + text_s, **tok)
    mid, mpos, mlen, mtok = file_to_memory(ids, lens, tok_)

    def side(mask, shift):
        ln = mlen[mask]
        t = np.concatenate([mtok[p:p + n] for p, n in zip(mpos[mask], ln)]) if len(ln) else np.zeros(0, np.uint32)
        p = np.concatenate([[0], np.cumsum(ln[:-1])]).astype(np.uint32) if len(ln) else np.zeros(0, np.uint32)
        return mid[mask] - shift, p, ln, t.astype(np.uint32)
    return side(mid <= nr, 0), side(mid > nr, nr), nt


def rs_union(r_len, s_len):
    """Memory order of the union of two record sets (each in memory order):
    descending size, then R before S, then the index within its side.
    Returns (side u8, index within side u32) per union record."""
    r_len = np.asarray(r_len, dtype=np.int64)
    s_len = np.asarray(s_len, dtype=np.int64)
    ln = np.concatenate([r_len, s_len])
    side = np.concatenate([np.zeros(len(r_len), np.uint8), np.ones(len(s_len), np.uint8)])
    idx = np.concatenate([np.arange(len(r_len)), np.arange(len(s_len))]).astype(np.int64)
    order = np.lexsort((idx, side, -ln))
    return side[order], idx[order].astype(np.uint32)


RS_PAIR_DTYPE = np.dtype([("r", "<u4"), ("s", "<u4"), ("overlap", "<u4"), ("sim", "<f4")])


def rsjoin(r, s, n_terms, t, threads=0):
    """R-S join as defined by the library: the self-join of R and S together (union
    in rs_union order) restricted to pairs with one record from each side, each
    reported as (index in R, index in S) and sorted by (r, s).  ``r`` and ``s`` are
    (pos, len, tokens) in memory order over one vocabulary.  Returns (pairs, stats)."""
    (rp, rl, rt), (sp, sl, stk) = r, s
    rp, rl, rt = (np.asarray(x, dtype=np.uint32) for x in (rp, rl, rt))
    sp, sl, stk = (np.asarray(x, dtype=np.uint32) for x in (sp, sl, stk))
    side, idx = rs_union(rl, sl)
    m = side == 0
    ulen = np.empty(len(side), np.uint32)
    upos = np.empty(len(side), np.uint32)
    ulen[m], upos[m] = rl[idx[m]], rp[idx[m]]
    ulen[~m], upos[~m] = sl[idx[~m]], sp[idx[~m]] + len(rt)
    utok = np.concatenate([rt, stk]).astype(np.uint32)
    pairs, st = join(upos, ulen, utok, n_terms, t, threads=threads, side=side)
    out = np.zeros(len(pairs), dtype=RS_PAIR_DTYPE)
    if len(pairs):
        q, v = pairs["q"], pairs["s"]
        q_is_r = side[q] == 0
        out["r"] = np.where(q_is_r, idx[q], idx[v])
        out["s"] = np.where(q_is_r, idx[v], idx[q])
        out["overlap"] = pairs["overlap"]
        out["sim"] = pairs["sim"]
        out = out[np.lexsort((out["s"], out["r"]))]
    return out, st


def rs_brute(r, s, t):
    """All R x S pairs with float(o) / float(|r| + |s| - o) >= t and o > 0 (the
    reference's final test, block.cu:190-193), sorted by (r, s); small inputs only."""
    (rp, rl, rt), (sp, sl, stk) = r, s
    res = []
    rsets = [np.asarray(rt[int(p):int(p) + int(n)]) for p, n in zip(rp, rl)]
    ssets = [np.asarray(stk[int(p):int(p) + int(n)]) for p, n in zip(sp, sl)]
    for i, a in enumerate(rsets):
        for j, b in enumerate(ssets):
            o = len(np.intersect1d(a, b, assume_unique=True))
            if o == 0:
                continue
            sim = np.float32(o) / np.float32(len(a) + len(b) - o)
            if sim >= np.float32(t):
                res.append((i, j, o, sim))
    return np.array(res, dtype=RS_PAIR_DTYPE)
