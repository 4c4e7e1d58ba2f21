"""ctypes binding of libfgss.so (C ABI: include/fgss.h)."""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_lib", "libfgss.so")

METHOD_PLAIN, METHOD_BATCHED = 0, 1
BOUNDS_REFERENCE, BOUNDS_EXACT = 0, 1
# filter strategies of the batched method (fgss_join_opts.filter)
FILTERS = {"auto": 0, "warp": 1, "cta": 2, "global": 3}
FILTER_NAMES = {v: k for k, v in FILTERS.items()}
TOK_QGRAM, TOK_KMER = 0, 1

# every entry point include/fgss.h declares
EXPORTED_SYMBOLS = [
    "fgss_options_default", "fgss_create", "fgss_destroy", "fgss_strerror", "fgss_last_error", "fgss_version",
    "fgss_load_bin", "fgss_write_bin", "fgss_sets_free", "fgss_sets_view_of",
    "fgss_tok_opts_default", "fgss_tokenize", "fgss_tokenize_dual",
    "fgss_join_opts_default", "fgss_selfjoin", "fgss_selfjoin_batch", "fgss_rsjoin", "fgss_pairs_free",
    "fgss_pairs_print", "fgss_selfjoin_to_file",
    "fgss_model_train", "fgss_model_save", "fgss_model_load", "fgss_model_grad", "fgss_model_num_params",
    "fgss_autotune", "fgss_bounds_table", "fgss_overlap_table", "fgss_query_costs", "fgss_dev_exclusive_scan_u32", "fgss_dev_sort_pairs_u64",
    "fgss_dev_exclusive_scan_u32_noalloc",
]

_u32p = ctypes.POINTER(ctypes.c_uint32)


class _Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("stream", ctypes.c_void_p), ("verbose", ctypes.c_int),
                ("tune_cache_path", ctypes.c_char_p)]


class _Sets(ctypes.Structure):
    _fields_ = [("id", _u32p), ("pos", _u32p), ("len", _u32p), ("tokens", _u32p), ("loc", _u32p),
                ("n_sets", ctypes.c_uint64), ("n_tokens", ctypes.c_uint64), ("n_terms", ctypes.c_uint32),
                ("max_len", ctypes.c_uint32)]


class _View(ctypes.Structure):
    _fields_ = [("id", ctypes.c_void_p), ("pos", ctypes.c_void_p), ("len", ctypes.c_void_p),
                ("tokens", ctypes.c_void_p), ("n_sets", ctypes.c_uint64), ("n_tokens", ctypes.c_uint64),
                ("n_terms", ctypes.c_uint32), ("on_device", ctypes.c_int)]


class _TokOpts(ctypes.Structure):
    _fields_ = [("q", ctypes.c_int), ("mode", ctypes.c_int), ("pad", ctypes.c_int), ("pad_char", ctypes.c_int),
                ("suffix", ctypes.c_int), ("lower", ctypes.c_int)]


class _JoinOpts(ctypes.Structure):
    _fields_ = [("threshold", ctypes.c_float), ("bounds", ctypes.c_int), ("method", ctypes.c_int),
                ("out_on_device", ctypes.c_int), ("want_candidates", ctypes.c_int), ("use_model", ctypes.c_int),
                ("result_capacity", ctypes.c_uint64), ("query_begin", ctypes.c_uint64),
                ("query_end", ctypes.c_uint64), ("no_graph", ctypes.c_int), ("filter", ctypes.c_int)]


class _Stats(ctypes.Structure):
    _fields_ = [("candidates", ctypes.c_uint64), ("intersections", ctypes.c_uint64), ("results", ctypes.c_uint64),
                ("index_entries", ctypes.c_uint64), ("probe_tokens", ctypes.c_uint64),
                ("window_entries", ctypes.c_uint64), ("verified", ctypes.c_uint64),
                ("heavy_queries", ctypes.c_uint64), ("overflow_retries", ctypes.c_uint32),
                ("ms_total", ctypes.c_float), ("ms_index", ctypes.c_float), ("ms_filter", ctypes.c_float),
                ("ms_verify", ctypes.c_float), ("ms_output", ctypes.c_float), ("ms_probe", ctypes.c_float),
                ("merged_tokens", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("predicted_candidates", ctypes.c_uint64), ("predicted_results", ctypes.c_uint64),
                ("query_tokens", ctypes.c_uint64), ("ms_heavy", ctypes.c_float), ("ms_reserved", ctypes.c_float)]


class _Pairs(ctypes.Structure):
    _fields_ = [("q", _u32p), ("s", _u32p), ("id_q", _u32p), ("id_s", _u32p), ("overlap", _u32p),
                ("sim", ctypes.POINTER(ctypes.c_float)), ("n", ctypes.c_uint64), ("on_device", ctypes.c_int),
                ("cand", _u32p), ("n_cand", ctypes.c_uint64), ("priv", ctypes.c_void_p)]


class _TuneResult(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_int), ("hash_log2", ctypes.c_int), ("regs_rt", ctypes.c_int),
                ("ctas_per_sm", ctypes.c_int),
                ("ms", ctypes.c_float), ("key", ctypes.c_char * 64), ("filter", ctypes.c_int)]


class FgssError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (status %d)" % (msg, status))
        self.status = status


_lib = None


def lib_path():
    return _LIB


def load_library():
    """Loads libfgss.so (built by ``__graft_entry__.build()``); raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB):
        raise FgssError(-1, "libfgss.so is not built (%s); run __graft_entry__.build()" % _LIB)
    L = ctypes.CDLL(_LIB)
    P = ctypes.POINTER
    L.fgss_create.argtypes = [P(ctypes.c_void_p), P(_Options)]
    L.fgss_destroy.argtypes = [ctypes.c_void_p]
    L.fgss_strerror.restype = ctypes.c_char_p
    L.fgss_strerror.argtypes = [ctypes.c_int]
    L.fgss_last_error.restype = ctypes.c_char_p
    L.fgss_last_error.argtypes = [ctypes.c_void_p]
    L.fgss_load_bin.argtypes = [ctypes.c_char_p, P(_Sets)]
    L.fgss_write_bin.argtypes = [ctypes.c_char_p, ctypes.c_char_p, P(_Sets)]
    L.fgss_sets_free.argtypes = [P(_Sets)]
    L.fgss_tokenize.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint64, P(_TokOpts), P(_Sets)]
    L.fgss_selfjoin.argtypes = [ctypes.c_void_p, P(_View), P(_JoinOpts), P(_Pairs), P(_Stats)]
    L.fgss_selfjoin_batch.argtypes = [ctypes.c_void_p, P(_View), P(_JoinOpts), ctypes.c_int, P(_Pairs), P(_Stats)]
    L.fgss_tokenize_dual.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint64, ctypes.c_char_p,
                                     ctypes.c_uint64, P(_TokOpts), P(_Sets), P(_Sets)]
    L.fgss_rsjoin.argtypes = [ctypes.c_void_p, P(_View), P(_View), P(_JoinOpts), P(_Pairs), P(_Stats)]
    L.fgss_selfjoin_to_file.argtypes = [ctypes.c_void_p, P(_View), P(_JoinOpts), ctypes.c_char_p, ctypes.c_int,
                                        ctypes.c_int, P(_Stats)]
    L.fgss_pairs_free.argtypes = [P(_Pairs)]
    L.fgss_query_costs.argtypes = [ctypes.c_void_p, P(_View), P(_JoinOpts), ctypes.c_void_p]
    L.fgss_model_train.argtypes = [ctypes.c_void_p, P(_View), P(ctypes.c_float), ctypes.c_int, ctypes.c_int,
                                   ctypes.c_float, ctypes.c_uint64, P(ctypes.c_float)]
    L.fgss_model_save.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    L.fgss_model_load.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    L.fgss_model_grad.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                  ctypes.c_void_p, P(ctypes.c_float)]
    L.fgss_dev_exclusive_scan_u32.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
    L.fgss_dev_sort_pairs_u64.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.c_int, ctypes.c_int]
    L.fgss_dev_exclusive_scan_u32_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                                      ctypes.c_void_p]
    L.fgss_autotune.argtypes = [ctypes.c_void_p, P(_View), P(_JoinOpts), ctypes.c_int, P(_TuneResult)]
    L.fgss_bounds_table.argtypes = [ctypes.c_float, ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.fgss_overlap_table.argtypes = [ctypes.c_float, ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    _lib = L
    return L


def bounds_table(threshold, max_len, bounds="reference"):
    """Host-side bound tables (no GPU): probe, index, min_size, max_size per
    length and the smallest accepted overlap per length sum."""
    L = load_library()
    mode = {"reference": BOUNDS_REFERENCE, "exact": BOUNDS_EXACT}.get(bounds, bounds)
    probe = np.zeros(max_len + 1, np.uint16)
    index = np.zeros(max_len + 1, np.uint16)
    mins = np.zeros(max_len + 1, np.uint32)
    maxs = np.zeros(max_len + 1, np.uint32)
    need = np.zeros(2 * max_len + 1, np.uint32)
    st = L.fgss_bounds_table(ctypes.c_float(threshold), mode, max_len, probe.ctypes.data, index.ctypes.data,
                             mins.ctypes.data, maxs.ctypes.data, need.ctypes.data)
    if st != 0:
        raise FgssError(st, "fgss_bounds_table failed")
    return probe, index, mins, maxs, need


def overlap_table(threshold, max_sum, bounds="reference"):
    """Host-side overlap tables (no GPU) per length sum: the smallest count the
    positional filter keeps (cand_min) and floor(min overlap) (inter_min)."""
    L = load_library()
    mode = {"reference": BOUNDS_REFERENCE, "exact": BOUNDS_EXACT}.get(bounds, bounds)
    cand = np.zeros(max_sum + 1, np.uint32)
    inter = np.zeros(max_sum + 1, np.uint32)
    st = L.fgss_overlap_table(ctypes.c_float(threshold), mode, max_sum, cand.ctypes.data, inter.ctypes.data)
    if st != 0:
        raise FgssError(st, "fgss_overlap_table failed")
    return cand, inter


def _check(L, ctx, st):
    if st != 0:
        msg = L.fgss_last_error(ctx).decode(errors="replace") or L.fgss_strerror(st).decode()
        raise FgssError(st, msg)


def _arr(a, dtype=np.uint32):
    return np.ascontiguousarray(a, dtype=dtype)


class Sets:
    """Token sets in the reference's MEMORY order (src/fgssjoin/data.cu:97-113).

    Arrays: id, pos, len, tokens (uint32) and optionally loc (q-gram position of
    each token).  ``n_terms`` = max token + 1 (data.cu:77-78).
    """

    def __init__(self, id, pos, len, tokens, n_terms=None, loc=None):
        self.id = _arr(id)
        self.pos = _arr(pos)
        self.len = _arr(len)
        self.tokens = _arr(tokens)
        self.loc = None if loc is None else _arr(loc)
        if n_terms is None:
            n_terms = int(self.tokens.max()) + 1 if self.tokens.size else 0
        self.n_terms = int(n_terms)

    @property
    def n_sets(self):
        return int(self.len.size)

    @property
    def n_tokens(self):
        return int(self.tokens.size)

    @classmethod
    def _from_c(cls, s):
        n, T = s.n_sets, s.n_tokens

        def take(p, k):
            return np.ctypeslib.as_array(p, shape=(k,)).copy() if k else np.zeros(0, np.uint32)
        loc = take(s.loc, T) if s.loc else None
        return cls(take(s.id, n), take(s.pos, n), take(s.len, n), take(s.tokens, T), s.n_terms, loc)

    @classmethod
    def from_bin(cls, path):
        L = load_library()
        s = _Sets()
        st = L.fgss_load_bin(os.fsencode(path), ctypes.byref(s))
        if st != 0:
            raise FgssError(st, "cannot load %s: %s" % (path, L.fgss_strerror(st).decode()))
        try:
            return cls._from_c(s)
        finally:
            L.fgss_sets_free(ctypes.byref(s))

    def _as_c(self):
        s = _Sets()
        s.id = self.id.ctypes.data_as(_u32p)
        s.pos = self.pos.ctypes.data_as(_u32p)
        s.len = self.len.ctypes.data_as(_u32p)
        s.tokens = self.tokens.ctypes.data_as(_u32p)
        s.loc = self.loc.ctypes.data_as(_u32p) if self.loc is not None else None
        s.n_sets, s.n_tokens, s.n_terms = self.n_sets, self.n_tokens, self.n_terms
        return s

    def to_bin(self, path, loc_path=None):
        """Writes the .bin (FILE order, ascending size) and optionally the .loc."""
        L = load_library()
        s = self._as_c()
        st = L.fgss_write_bin(os.fsencode(path), os.fsencode(loc_path) if loc_path else None, ctypes.byref(s))
        if st != 0:
            raise FgssError(st, "cannot write %s" % path)

    def view(self):
        v = _View()
        v.id = self.id.ctypes.data
        v.pos = self.pos.ctypes.data
        v.len = self.len.ctypes.data
        v.tokens = self.tokens.ctypes.data if self.tokens.size else None
        v.n_sets, v.n_tokens, v.n_terms, v.on_device = self.n_sets, self.n_tokens, self.n_terms, 0
        return v


def ppjoin_format(path):
    """Mirror of the reference loader ``ppjoin_format`` (data.cu:31-126)."""
    return Sets.from_bin(path)


class _PairsOwner:
    """Owns one fgss_pairs result (a copy of the struct) and frees it once."""

    def __init__(self, lib, p):
        self._lib = lib
        self._p = _Pairs()
        ctypes.memmove(ctypes.byref(self._p), ctypes.byref(p), ctypes.sizeof(_Pairs))

    def __del__(self):
        try:
            self._lib.fgss_pairs_free(ctypes.byref(self._p))
        except Exception:  # interpreter shutdown
            pass


class Pairs:
    """Join result, sorted by (q, s): memory indices q < s, ids, overlap, sim."""

    def __init__(self, q, s, id_q, id_s, overlap, sim, stats, candidates=None):
        self.q, self.s, self.id_q, self.id_s, self.overlap, self.sim = q, s, id_q, id_s, overlap, sim
        self.stats = stats
        self.candidates = candidates

    def __len__(self):
        return int(self.q.shape[0])

    def lines(self):
        """The reference's stdout lines, "%d %d %f" (block.cu:193)."""
        return ["%d %d %f" % (int(a), int(b), float(c)) for a, b, c in zip(self.id_q, self.id_s, self.sim)]


def _stats_dict(st):
    return {k: (float(getattr(st, k)) if k.startswith("ms_") else int(getattr(st, k))) for k, _ in _Stats._fields_}


class Context:
    """A libfgss context bound to one CUDA device and stream."""

    def __init__(self, device=0, stream=None, verbose=False, tune_cache_path=None):
        self._L = load_library()
        o = _Options()
        o.device = device
        o.stream = stream
        o.verbose = int(verbose)
        self._tune_path = os.fsencode(tune_cache_path) if tune_cache_path else None
        o.tune_cache_path = self._tune_path
        self._ctx = ctypes.c_void_p()
        st = self._L.fgss_create(ctypes.byref(self._ctx), ctypes.byref(o))
        if st != 0:
            raise FgssError(st, self._L.fgss_last_error(None).decode(errors="replace") or "fgss_create failed")

    def close(self):
        if self._ctx:
            self._L.fgss_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._ctx

    # ------------------------------------------------------------ tokenizer
    def tokenize(self, text, q=3, mode="qgram", pad=False, pad_char=1, suffix=True, lower=True):
        """Text -> Sets on the GPU (see fgss_tokenize in include/fgss.h)."""
        if isinstance(text, str):
            text = text.encode("latin-1")
        o = _TokOpts(q, TOK_KMER if mode == "kmer" else TOK_QGRAM, int(pad), pad_char, int(suffix), int(lower))
        s = _Sets()
        st = self._L.fgss_tokenize(self._ctx, text, len(text), ctypes.byref(o), ctypes.byref(s))
        _check(self._L, self._ctx, st)
        try:
            return Sets._from_c(s)
        finally:
            self._L.fgss_sets_free(ctypes.byref(s))

    def tokenize_dual(self, text_r, text_s, q=3, mode="qgram", pad=False, pad_char=1, suffix=True, lower=True):
        """Two texts over one vocabulary -> (Sets of R, Sets of S) (fgss_tokenize_dual)."""
        text_r = text_r.encode("latin-1") if isinstance(text_r, str) else text_r
        text_s = text_s.encode("latin-1") if isinstance(text_s, str) else text_s
        o = _TokOpts(q, TOK_KMER if mode == "kmer" else TOK_QGRAM, int(pad), pad_char, int(suffix), int(lower))
        a, b = _Sets(), _Sets()
        st = self._L.fgss_tokenize_dual(self._ctx, text_r, len(text_r), text_s, len(text_s), ctypes.byref(o),
                                        ctypes.byref(a), ctypes.byref(b))
        _check(self._L, self._ctx, st)
        try:
            return Sets._from_c(a), Sets._from_c(b)
        finally:
            self._L.fgss_sets_free(ctypes.byref(a))
            self._L.fgss_sets_free(ctypes.byref(b))

    # ----------------------------------------------------------------- join
    @staticmethod
    def _opts(threshold, method, bounds, want_candidates, use_model, out_on_device=False, result_capacity=0,
              query_range=None, filter="auto"):
        o = _JoinOpts()
        o.filter = FILTERS[filter] if isinstance(filter, str) else int(filter)
        o.threshold = float(threshold)
        o.method = {"plain": METHOD_PLAIN, "batched": METHOD_BATCHED}.get(method, method)
        o.bounds = {"reference": BOUNDS_REFERENCE, "exact": BOUNDS_EXACT}.get(bounds, bounds)
        o.want_candidates = int(want_candidates)
        o.use_model = int(use_model)
        o.out_on_device = int(out_on_device)
        o.result_capacity = int(result_capacity)
        if query_range is not None:
            o.query_begin, o.query_end = int(query_range[0]), int(query_range[1])
        return o

    def _collect(self, p, st, want_candidates):
        """Pairs over the library's host columns without copying them: the
        columns are released (fgss_pairs_free) when the last array over them
        is garbage-collected."""
        L = self._L
        n = p.n
        owner = _PairsOwner(L, p)

        def take(ptr, ctype=ctypes.c_uint32, dtype=np.uint32):
            if not n:
                return np.zeros(0, dtype)
            buf = (ctype * n).from_address(ctypes.cast(ptr, ctypes.c_void_p).value)
            buf._owner = owner  # the arrays keep the columns alive
            return np.frombuffer(buf, dtype)
        cands = None
        if want_candidates:
            nc = p.n_cand
            cands = (np.ctypeslib.as_array(p.cand, shape=(3 * nc,)).reshape(-1, 3).copy()
                     if nc else np.zeros((0, 3), np.uint32))
        return Pairs(take(p.q), take(p.s), take(p.id_q), take(p.id_s), take(p.overlap),
                     take(p.sim, ctypes.c_float, np.float32), _stats_dict(st), cands)

    def query_costs(self, sets, threshold, bounds="reference", use_model=True):
        """Per-query work estimates of the join (fgss_query_costs): window entries
        + 4 x the learned model's predicted candidates + size, memory order."""
        v = sets.view() if isinstance(sets, Sets) else sets
        o = self._opts(threshold, "batched", bounds, False, use_model)
        out = np.zeros(max(int(v.n_sets), 1), np.uint64)
        rc = self._L.fgss_query_costs(self._ctx, ctypes.byref(v), ctypes.byref(o), out.ctypes.data)
        _check(self._L, self._ctx, rc)
        return out[:int(v.n_sets)]

    def selfjoin(self, sets, threshold, method="plain", bounds="reference", want_candidates=False,
                 use_model=False, result_capacity=0, query_range=None, filter="auto"):
        """Self-join of ``sets`` (host Sets or a device view) at ``threshold``.

        ``query_range`` = (begin, end) processes only the pairs whose first
        record (memory index) lies in [begin, end): one shard of the join."""
        v = sets.view() if isinstance(sets, Sets) else sets
        o = self._opts(threshold, method, bounds, want_candidates, use_model, result_capacity=result_capacity,
                       query_range=query_range, filter=filter)
        p = _Pairs()
        st = _Stats()
        rc = self._L.fgss_selfjoin(self._ctx, ctypes.byref(v), ctypes.byref(o), ctypes.byref(p), ctypes.byref(st))
        _check(self._L, self._ctx, rc)
        return self._collect(p, st, want_candidates)

    def rsjoin(self, r, s, threshold, method="batched", bounds="reference", use_model=False, result_capacity=0):
        """R-S join (fgss_rsjoin): pairs (index in R, index in S) with Jaccard >= threshold,
        returned with ``q`` = the R index and ``s`` = the S index, sorted by (q, s)."""
        vr = r.view() if isinstance(r, Sets) else r
        vs = s.view() if isinstance(s, Sets) else s
        o = self._opts(threshold, method, bounds, False, use_model, result_capacity=result_capacity)
        p = _Pairs()
        st = _Stats()
        rc = self._L.fgss_rsjoin(self._ctx, ctypes.byref(vr), ctypes.byref(vs), ctypes.byref(o), ctypes.byref(p),
                                 ctypes.byref(st))
        _check(self._L, self._ctx, rc)
        return self._collect(p, st, False)

    def selfjoin_to_file(self, sets, threshold, path, fmt="text", shards=4, method="batched", bounds="reference",
                         use_model=False):
        """Streaming self-join (fgss_selfjoin_to_file): the pairs go to ``path`` as the
        reference's text lines (fmt "text") or 12-byte binary records (fmt "binary")
        while the GPU joins the next of ``shards`` query ranges; returns the stats."""
        v = sets.view() if isinstance(sets, Sets) else sets
        o = self._opts(threshold, method, bounds, False, use_model)
        st = _Stats()
        rc = self._L.fgss_selfjoin_to_file(self._ctx, ctypes.byref(v), ctypes.byref(o), os.fsencode(path),
                                           {"text": 0, "binary": 1}[fmt], int(shards), ctypes.byref(st))
        _check(self._L, self._ctx, rc)
        return _stats_dict(st)

    def selfjoin_batch(self, sets_list, thresholds, method="batched", bounds="reference", use_model=False,
                       result_capacity=0, filter="auto"):
        """Many independent self-joins in one call (one persistent launch per stage)."""
        n = len(sets_list)
        views = (_View * n)(*[s.view() if isinstance(s, Sets) else s for s in sets_list])
        opts = (_JoinOpts * n)(*[self._opts(t, method, bounds, False, use_model, result_capacity=result_capacity,
                                            filter=filter)
                                 for t in thresholds])
        outs = (_Pairs * n)()
        sts = (_Stats * n)()
        rc = self._L.fgss_selfjoin_batch(self._ctx, views, opts, n, outs, sts)
        _check(self._L, self._ctx, rc)
        return [self._collect(outs[i], sts[i], False) for i in range(n)]

    def autotune(self, sets, threshold, reps=2, bounds="reference"):
        """Times every fused-kernel launch shape on this join; caches the best."""
        v = sets.view() if isinstance(sets, Sets) else sets
        o = self._opts(threshold, "batched", bounds, False, False)
        r = _TuneResult()
        _check(self._L, self._ctx, self._L.fgss_autotune(self._ctx, ctypes.byref(v), ctypes.byref(o), reps,
                                                         ctypes.byref(r)))
        return {"threads": r.threads, "hash_log2": r.hash_log2, "regs_rt": r.regs_rt, "ctas_per_sm": r.ctas_per_sm,
                "ms": r.ms, "key": r.key.decode(), "filter": FILTER_NAMES[r.filter]}

    # --------------------------------------------------------------- model
    def model_train(self, sets_list, thresholds, epochs=300, lr=0.01, seed=0):
        n = len(sets_list)
        views = (_View * n)(*[s.view() if isinstance(s, Sets) else s for s in sets_list])
        ts = (ctypes.c_float * n)(*thresholds)
        loss = ctypes.c_float()
        rc = self._L.fgss_model_train(self._ctx, views, ts, n, epochs, lr, seed, ctypes.byref(loss))
        _check(self._L, self._ctx, rc)
        return float(loss.value)

    def model_grad(self, feat, target, params):
        """One GPU forward/backward of the cost-model MLP: returns (grads, loss)."""
        feat = np.ascontiguousarray(feat, np.float32)
        target = np.ascontiguousarray(target, np.float32)
        params = np.ascontiguousarray(params, np.float32)
        grads = np.zeros_like(params)
        loss = ctypes.c_float()
        rc = self._L.fgss_model_grad(self._ctx, feat.ctypes.data, target.ctypes.data, feat.shape[0],
                                     params.ctypes.data, grads.ctypes.data, ctypes.byref(loss))
        _check(self._L, self._ctx, rc)
        return grads, float(loss.value)

    def model_save(self, path):
        _check(self._L, self._ctx, self._L.fgss_model_save(self._ctx, os.fsencode(path)))

    def model_load(self, path):
        _check(self._L, self._ctx, self._L.fgss_model_load(self._ctx, os.fsencode(path)))

    # ---------------------------------------------------- device primitives
    def dev_exclusive_scan_u32(self, d_in, d_out, n):
        _check(self._L, self._ctx, self._L.fgss_dev_exclusive_scan_u32(self._ctx, d_in, d_out, n))

    def dev_sort_pairs_u64(self, d_keys, d_vals, n, begin_bit=0, end_bit=64):
        _check(self._L, self._ctx, self._L.fgss_dev_sort_pairs_u64(self._ctx, d_keys, d_vals, n, begin_bit, end_bit))
