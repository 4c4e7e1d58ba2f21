"""GPU tokenizer against the oracle and the reference's fixture."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from new_fgssjoin_b200 import datagen
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mem(ids, lens, tok, loc):
    mid, mpos, mlen, mtok = O.file_to_memory(ids, lens, tok)
    _, _, _, mloc = O.file_to_memory(ids, lens, loc)
    return mid, mpos, mlen, mtok, mloc


def test_fixture_bytes(ctx, tmp_path):
    text = open(os.path.join(GOLDEN, "small.txt"), "rb").read()
    s = ctx.tokenize(text, q=3, pad=False, suffix=True, lower=True)
    out = tmp_path / "small.bin"
    s.to_bin(str(out), str(out) + ".loc")
    assert out.read_bytes() == open(os.path.join(GOLDEN, "small.txt.3gram.bin"), "rb").read()
    assert (tmp_path / "small.bin.loc").read_bytes() == \
        open(os.path.join(GOLDEN, "small.txt.3gram.bin.loc"), "rb").read()
    assert s.n_terms == 42


@pytest.mark.parametrize("opts", [
    dict(q=3, pad=True, suffix=False),
    dict(q=3, pad=False, suffix=True),
    dict(q=2, pad=True, suffix=True),
    dict(q=5, pad=False, suffix=False),
    dict(q=11, pad=True, suffix=False),   # hashed grams
])
def test_titles_vs_oracle(ctx, opts):
    text = datagen.titles(3000, seed=21) + b"\n\nAB\nAbc abc ABC\n"
    s = ctx.tokenize(text, lower=True, **opts)
    ids, lens, tok, loc, nt = O.tokenize(text, lower=True, **opts)
    mid, mpos, mlen, mtok, mloc = _mem(ids, lens, tok, loc)
    assert s.n_terms == nt
    assert np.array_equal(s.id, mid) and np.array_equal(s.len, mlen) and np.array_equal(s.pos, mpos)
    assert np.array_equal(s.tokens, mtok) and np.array_equal(s.loc, mloc)


def test_kmers_vs_oracle(ctx):
    text = datagen.reads(2000, seed=5, genome_len=50000) + b"ACGTNACGTACGTACGTACGTAC\n"
    s = ctx.tokenize(text, **datagen.READ_TOK)
    ids, lens, tok, loc, nt = O.tokenize(text, q=16, mode="kmer", pad=False, suffix=False)
    mid, mpos, mlen, mtok, mloc = _mem(ids, lens, tok, loc)
    assert s.n_terms == nt
    assert np.array_equal(s.id, mid) and np.array_equal(s.len, mlen)
    assert np.array_equal(s.tokens, mtok) and np.array_equal(s.loc, mloc)


def test_empty_text(ctx):
    s = ctx.tokenize(b"", q=3)
    assert s.n_sets == 0 and s.n_tokens == 0
    s = ctx.tokenize(b"\n\nab\n", q=3, pad=False)  # no line yields a 3-gram
    assert s.n_sets == 0
