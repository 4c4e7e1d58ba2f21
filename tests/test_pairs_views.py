"""Host logic of the binding's result views (CPU only): a join's pairs are numpy
views over the library's host columns, released by one fgss_pairs_free call
once the last array over them is gone."""
import ctypes
import gc

import numpy as np

from new_fgssjoin_b200 import binding as B


class _FakeLib:
    """Stands in for libfgss: records the fgss_pairs_free calls."""

    def __init__(self):
        self.freed = []

    def fgss_pairs_free(self, pref):
        p = pref._obj
        self.freed.append(ctypes.cast(p.q, ctypes.c_void_p).value)


class _Host:
    _L = None


def _pairs_over(cols):
    p = B._Pairs()
    p.q, p.s, p.id_q, p.id_s, p.overlap = [c.ctypes.data_as(B._u32p) for c in cols[:5]]
    p.sim = cols[5].ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    p.n = cols[0].size
    return p


def test_views_see_the_columns_and_free_them_once_after_the_last_array():
    n = 1000
    rng = np.random.default_rng(1)
    cols = [rng.integers(0, 1 << 30, n).astype(np.uint32) for _ in range(5)] + [rng.random(n).astype(np.float32)]
    host = _Host()
    host._L = _FakeLib()
    out = B.Context._collect(host, _pairs_over(cols), B._Stats(), False)
    for got, want in zip((out.q, out.s, out.id_q, out.id_s, out.overlap, out.sim), cols):
        assert got.dtype == want.dtype and np.array_equal(got, want)
        assert got.ctypes.data == want.ctypes.data  # a view, not a copy
    assert len(out) == n
    del got, want
    keep = out.sim
    del out
    gc.collect()
    assert host._L.freed == []  # one array still refers to the columns
    assert float(keep[3]) == float(cols[5][3])
    del keep
    gc.collect()
    assert host._L.freed == [cols[0].ctypes.data]


def test_empty_result_frees_its_struct():
    host = _Host()
    host._L = _FakeLib()
    p = B._Pairs()
    out = B.Context._collect(host, p, B._Stats(), False)
    assert len(out) == 0 and out.sim.dtype == np.float32
    del out
    gc.collect()
    assert host._L.freed == [None]
