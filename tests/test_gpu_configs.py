"""GPU parity at the benchmark configurations' full sizes: the CUDA path
(GPU tokenizer, then the join by both methods through the C ABI) against the
CPU oracle on the same seeded inputs.

  C1  18,000 titles, t = 0.9 (the output pair set must equal the reference's)
  C2  100,000 titles at t = 0.5 and 0.8 (0.8: float32 bounds drop pairs with J = t)
  C3  heavy-tailed records at 300,000 (the 1,000,000-record join is checked
      against the oracle by every bench run: "pairs_equal_oracle")
  C4  500,000 reads of 150 bases, canonical 16-mers, t = 0.8
  C5  24 joins of the 256-join batch draw, one batched call
"""
import numpy as np
import pytest

from new_fgssjoin_b200 import datagen
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _same(got, ref, st):
    assert len(got) == len(ref)
    assert np.array_equal(got.q, ref["q"]) and np.array_equal(got.s, ref["s"])
    assert np.array_equal(got.overlap, ref["overlap"])
    assert np.array_equal(got.sim, ref["sim"])  # float32 division, bit-exact
    for k in ("candidates", "intersections", "results", "index_entries"):
        assert got.stats[k] == st[k], (k, got.stats[k], st[k])


def _tokenized_equal_oracle(sets, text, tok):
    ids, lens, toks, loc, nt = O.tokenize(text, **tok)
    mid, mpos, mlen, mtok = O.file_to_memory(ids, lens, toks)
    assert sets.n_terms == nt
    assert np.array_equal(sets.id, mid) and np.array_equal(sets.len, mlen)
    assert np.array_equal(sets.pos, mpos) and np.array_equal(sets.tokens, mtok)


def test_c1_titles18k_full_size(ctx):
    text = datagen.titles(18_000, seed=1)
    sets = ctx.tokenize(text, **datagen.TITLE_TOK)
    _tokenized_equal_oracle(sets, text, datagen.TITLE_TOK)
    ref, st = O.join(sets.pos, sets.len, sets.tokens, sets.n_terms, 0.9)
    assert st["results"] > 0
    for method in ("plain", "batched"):
        _same(ctx.selfjoin(sets, 0.9, method=method), ref, st)


@pytest.fixture(scope="module")
def titles100k(ctx):
    return ctx.tokenize(datagen.titles(100_000, seed=2), **datagen.TITLE_TOK)


@pytest.mark.parametrize("t", [0.5, 0.8])
def test_c2_titles100k_full_size(ctx, titles100k, t):
    s = titles100k
    ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
    for method in ("plain", "batched"):
        _same(ctx.selfjoin(s, t, method=method, use_model=method == "batched"), ref, st)


def test_c3_heavy_tailed_300k(ctx):
    s = ctx.tokenize(datagen.heavy(300_000, seed=4), **datagen.TITLE_TOK)
    ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, 0.7)
    assert st["results"] > 0
    _same(ctx.selfjoin(s, 0.7, method="batched"), ref, st)


def test_c4_reads500k_full_size(ctx):
    text = datagen.reads(500_000, seed=5)
    s = ctx.tokenize(text, **datagen.READ_TOK)
    assert int(s.len.max()) <= 135
    ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, 0.8)
    assert st["results"] > 0
    for method in ("plain", "batched"):
        _same(ctx.selfjoin(s, 0.8, method=method), ref, st)


def test_c5_batch_of_joins(ctx):
    sizes, ts = datagen.batch_sizes(256, 1000, 200_000, seed=6)
    k = 24
    sets = [ctx.tokenize(datagen.titles(int(sizes[i]), seed=600_018 + i), **datagen.TITLE_TOK) for i in range(k)]
    got = ctx.selfjoin_batch(sets, [float(t) for t in ts[:k]], method="batched")
    for i in range(k):
        ref, st = O.join(sets[i].pos, sets[i].len, sets[i].tokens, sets[i].n_terms, float(ts[i]))
        _same(got[i], ref, st)
