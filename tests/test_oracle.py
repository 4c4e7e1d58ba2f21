"""CPU: the oracle pinned against the reference's fixtures and golden pairs."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as O


def _fixture():
    raw = open(os.path.join(GOLDEN, "small.txt.3gram.bin"), "rb").read()
    return raw, O.decode_bin(raw)


def test_fixture_decode_ascending_sizes():
    raw, (ids, lens, tok) = _fixture()
    assert list(ids) == [5, 1, 3, 2, 4]
    assert list(lens) == [11, 16, 18, 19, 24]
    assert len(tok) == 88 and tok.max() + 1 == 42


def test_tokenizer_reproduces_fixture_bytes():
    """Unpadded 3-grams with occurrence suffix, ids by (df, first occurrence)."""
    text = open(os.path.join(GOLDEN, "small.txt"), "rb").read()
    ids, lens, tok, loc, nterm = O.tokenize(text, q=3, pad=False, suffix=True, lower=True)
    raw, _ = _fixture()
    assert O.encode_bin(ids, lens, tok) == raw
    assert loc.astype("<i4").tobytes() == open(os.path.join(GOLDEN, "small.txt.3gram.bin.loc"), "rb").read()
    assert nterm == 42


@pytest.mark.parametrize("t", ["0.5", "0.59", "0.6", "0.7", "0.75", "0.8", "0.9"])
def test_join_golden_pairs(t):
    raw, (ids, lens, tok) = _fixture()
    mid, mpos, mlen, mtok = O.file_to_memory(ids, lens, tok)
    pairs, st = O.join(mpos, mlen, mtok, 42, float(t))
    got = sorted("%d %d %f" % (mid[p["q"]], mid[p["s"]], p["sim"]) for p in pairs)
    gold = json.load(open(os.path.join(GOLDEN, "small_pairs.json")))[t]
    assert got == gold
    assert st["results"] == len(gold)


def _rand_sets(rng, n, vocab, lo, hi):
    lens = np.sort(rng.integers(lo, hi + 1, n))[::-1]
    toks = [np.sort(rng.choice(vocab, size=int(l), replace=False)) for l in lens]
    pos = np.zeros(n, np.uint32)
    pos[1:] = np.cumsum(lens[:-1])
    return pos, lens.astype(np.uint32), np.concatenate(toks).astype(np.uint32)


@pytest.mark.parametrize("t", [0.5, 0.6, 0.7, 0.8, 0.9, 0.95])
def test_join_subset_of_brute_force(t):
    """Filters only remove pairs: reference semantics is a subset of the all-pairs check."""
    rng = np.random.default_rng(int(t * 100))
    pos, lens, tok = _rand_sets(rng, 300, 40, 1, 12)
    ref, _ = O.join(pos, lens, tok, 40, t)
    bf = O.brute(pos, lens, tok, t)
    a = set(zip(ref["q"], ref["s"]))
    b = set(zip(bf["q"], bf["s"]))
    assert a <= b
    if t in (0.5, 0.7, 0.9, 0.95):
        assert a == b  # no float32 bound differs from the exact one at these thresholds


def test_join_block_size_invariant_for_sorted_input():
    """block.cu:121-130 skips only block pairs that the size filter empties."""
    rng = np.random.default_rng(3)
    pos, lens, tok = _rand_sets(rng, 200, 30, 1, 10)
    a, sa = O.join(pos, lens, tok, 30, 0.6)
    for bs in (7, 50, 199):
        b, sb = O.join(pos, lens, tok, 30, 0.6, block_size=bs)
        assert np.array_equal(a, b)
        for k in ("candidates", "intersections", "results", "index_entries"):
            assert sa[k] == sb[k]  # only the list-scan count grows with more tiles


def test_float32_bounds_differ_from_exact_where_expected():
    """At t = 0.8 a 135-token read gets an index prefix of 15 (16 exactly)."""
    assert O.lib().orc_mid_prefix(np.float32(0.8), 135) == 15
    assert O.lib().orc_mid_prefix(np.float32(0.7), 135) == 135 - int(np.ceil(2 * 0.7 / 1.7 * 135)) + 1


def test_rs_union_order():
    side, idx = O.rs_union([5, 3, 3, 1], [4, 3, 2])
    # descending size, R before S at equal size, then index within the side
    assert side.tolist() == [0, 1, 0, 0, 1, 1, 0]
    assert idx.tolist() == [0, 0, 1, 2, 1, 2, 3]


@pytest.mark.parametrize("t", [0.5, 0.7, 0.8, 0.9])
def test_rsjoin_equals_brute_force(t):
    """The R-S join (self-join of the union restricted to pairs across) against
    all R x S pairs; equal wherever the float32 bounds lose no pair (t = 0.8 is
    checked as a subset, as for the self-join)."""
    from rs_util import split_titles, oracle_dual
    tr, ts = split_titles(2400, 7)
    (rid, rp, rl, rt), (sid, sp, sl, stk), nt = oracle_dual(tr, ts, q=3, pad=True, suffix=False)
    got, st = O.rsjoin((rp, rl, rt), (sp, sl, stk), nt, t)
    ref = O.rs_brute((rp, rl, rt), (sp, sl, stk), t)
    assert st["results"] == len(got) and len(ref) > 0
    key = lambda a: set(zip(a["r"].tolist(), a["s"].tolist()))
    assert key(got) <= key(ref)
    if t != 0.8:
        assert key(got) == key(ref)
    m = {(r, s): (o, x) for r, s, o, x in ref.tolist()}
    for r, s, o, x in got.tolist():
        assert m[(r, s)] == (o, x)
