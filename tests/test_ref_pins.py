"""CPU: the library's bound tables and .bin loader pinned against the
reference project's own code, compiled here from its sources by
oracle/ref_build.sh (oracle/_ref/ref_bounds over include/fgssjoin/similarity.cuh,
oracle/_ref/ref_load over src/fgssjoin/data.cu's ppjoin_format).  Skipped where
those binaries were not built (no reference checkout)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
import new_fgssjoin_b200 as F
from new_fgssjoin_b200 import datagen
from oracle import oracle as O

REF_BOUNDS = os.path.join(ROOT, "oracle", "_ref", "ref_bounds")
REF_LOAD = os.path.join(ROOT, "oracle", "_ref", "ref_load")
MAXLEN = 65535


def _ref_tables(t, L):
    raw = subprocess.run([REF_BOUNDS, repr(t), str(L)], capture_output=True, check=True, timeout=120).stdout
    a = np.frombuffer(raw, dtype="<u4")
    n1, s1 = L + 1, 2 * L + 1
    assert len(a) == 4 * n1 + 3 * s1
    cut = np.cumsum([0, n1, n1, n1, n1, s1, s1, s1])
    return [a[cut[i]:cut[i + 1]] for i in range(7)]


@pytest.mark.skipif(not os.path.exists(REF_BOUNDS), reason="reference bound harness not built")
@pytest.mark.parametrize("t", [0.5, 0.6, 0.7, 0.75, 0.8, 0.9, 0.95])
def test_bound_tables_equal_reference_similarity_header(t):
    """Every length n <= 65535 and length sum S <= 131070: the library's tables
    equal the reference's similarity.cuh functions evaluated as its kernels
    use them."""
    probe, index, mins, maxs, cand, inter, need = _ref_tables(t, MAXLEN)
    g_probe, g_index, g_mins, g_maxs, g_need = F.bounds_table(t, MAXLEN)
    g_cand, g_inter = F.overlap_table(t, 2 * MAXLEN)
    # n = 0: the reference's prefix of 1 would read a neighbour's token; an
    # empty record has no prefix here (it joins nothing)
    assert g_probe[0] == 0 and g_index[0] == 0
    assert np.array_equal(g_probe[1:].astype(np.uint32), probe[1:])
    assert np.array_equal(g_index[1:].astype(np.uint32), index[1:])
    assert np.array_equal(g_mins, mins) and np.array_equal(g_maxs, maxs)
    assert np.array_equal(g_cand, cand) and np.array_equal(g_inter, inter)
    # need[S] for S >= 2 (a pair of non-empty records)
    assert np.array_equal(g_need[2:], need[2:])


@pytest.mark.skipif(not os.path.exists(REF_BOUNDS), reason="reference bound harness not built")
def test_genomic_read_prefix_is_the_reference_float32_one():
    """A 135-token read at t = 0.8: the reference's float32 index prefix is 15,
    one shorter than the exact bound's 16."""
    _, index, *_ = _ref_tables(0.8, 200)
    assert index[135] == 15 and F.bounds_table(0.8, 200)[1][135] == 15
    assert F.bounds_table(0.8, 200, bounds="exact")[1][135] == 16


def _ref_load(path):
    raw = subprocess.run([REF_LOAD, path], capture_output=True, check=True, timeout=120).stdout
    a = np.frombuffer(raw, dtype="<u4")
    n, T, nt = (int(x) for x in a[:3])
    o = 3
    ids, pos, lens = a[o:o + n], a[o + n:o + 2 * n], a[o + 2 * n:o + 3 * n]
    return ids, pos, lens, a[o + 3 * n:o + 3 * n + T], nt


def _same(path):
    ids, pos, lens, tok, nt = _ref_load(path)
    s = F.ppjoin_format(path)
    assert np.array_equal(s.id, ids) and np.array_equal(s.pos, pos) and np.array_equal(s.len, lens)
    assert np.array_equal(s.tokens, tok) and s.n_terms == nt


@pytest.mark.skipif(not os.path.exists(REF_LOAD), reason="reference loader harness not built")
def test_loader_equals_reference_ppjoin_format_on_the_fixture():
    _same(os.path.join(GOLDEN, "small.txt.3gram.bin"))


@pytest.mark.skipif(not os.path.exists(REF_LOAD), reason="reference loader harness not built")
def test_loader_equals_reference_ppjoin_format_on_written_titles(tmp_path):
    """A .bin written by the library from 5,000 tokenized titles loads into the
    same memory-order arrays with the reference's loader and with ours."""
    ids, lens, tok, loc, nt = O.tokenize(datagen.titles(5000, seed=11), **datagen.TITLE_TOK)
    _, mpos, mlen, mtok = O.file_to_memory(ids, lens, tok)
    sets = F.Sets(np.ascontiguousarray(ids[::-1], dtype=np.uint32), mpos, mlen, mtok, n_terms=nt)
    p = str(tmp_path / "titles.bin")
    sets.to_bin(p)
    _same(p)
