"""GPU R-S join and two-text tokenization against the oracle."""
import numpy as np
import pytest

import new_fgssjoin_b200 as F
from new_fgssjoin_b200 import datagen
from oracle import oracle as O
from rs_util import split_titles, oracle_dual

pytestmark = pytest.mark.gpu


def _check_rs(got, ref, st=None):
    assert len(got) == len(ref)
    assert np.array_equal(got.q, ref["r"])
    assert np.array_equal(got.s, ref["s"])
    assert np.array_equal(got.overlap, ref["overlap"])
    assert np.array_equal(got.sim, ref["sim"])
    if st is not None:
        for k in ("candidates", "intersections", "results", "index_entries"):
            assert got.stats[k] == st[k], (k, got.stats, st)


@pytest.fixture(scope="module")
def titles_rs(ctx):
    tr, ts = split_titles(6000, 11)
    return tr, ts, ctx.tokenize_dual(tr, ts, **datagen.TITLE_TOK)


def test_tokenize_dual_matches_oracle(titles_rs):
    tr, ts, (r, s) = titles_rs
    (rid, rp, rl, rt), (sid, sp, sl, stk), nt = oracle_dual(tr, ts, q=3, pad=True, suffix=False)
    assert r.n_terms == s.n_terms == nt
    for got, (i, p, ln, t) in ((r, (rid, rp, rl, rt)), (s, (sid, sp, sl, stk))):
        assert np.array_equal(got.id, i) and np.array_equal(got.pos, p)
        assert np.array_equal(got.len, ln) and np.array_equal(got.tokens, t)


@pytest.mark.parametrize("method", ["plain", "batched"])
@pytest.mark.parametrize("t", [0.5, 0.7, 0.8, 0.9])
def test_rsjoin_titles_vs_oracle(ctx, titles_rs, method, t):
    _, _, (r, s) = titles_rs
    ref, st = O.rsjoin((r.pos, r.len, r.tokens), (s.pos, s.len, s.tokens), r.n_terms, t)
    assert len(ref) > 0
    got = ctx.rsjoin(r, s, t, method=method)
    _check_rs(got, ref, st)
    assert np.array_equal(got.id_q, r.id[got.q]) and np.array_equal(got.id_s, s.id[got.s])


def test_rsjoin_exact_bounds_equal_brute_force(ctx):
    tr, ts = split_titles(1600, 12)
    r, s = ctx.tokenize_dual(tr, ts, **datagen.TITLE_TOK)
    for t in (0.6, 0.8):
        ref = O.rs_brute((r.pos, r.len, r.tokens), (s.pos, s.len, s.tokens), t)
        got = ctx.rsjoin(r, s, t, bounds="exact")
        assert np.array_equal(got.q, ref["r"]) and np.array_equal(got.s, ref["s"])
        assert np.array_equal(got.overlap, ref["overlap"])


def test_rsjoin_reads_unbalanced_vs_oracle(ctx):
    """k-mer reads (vocabulary above 32k terms); R much smaller than S."""
    text = datagen.reads(6000, seed=13, genome_len=80000)
    lines = text.split(b"\n")[:-1]
    tr = b"\n".join(lines[:500]) + b"\n"
    ts = b"\n".join(lines[500:]) + b"\n"
    r, s = ctx.tokenize_dual(tr, ts, **datagen.READ_TOK)
    ref, st = O.rsjoin((r.pos, r.len, r.tokens), (s.pos, s.len, s.tokens), r.n_terms, 0.8)
    assert len(ref) > 0
    for method in ("plain", "batched"):
        _check_rs(ctx.rsjoin(r, s, 0.8, method=method), ref, st)
    # with exact bounds the roles swapped give the same pairs, swapped
    a = ctx.rsjoin(r, s, 0.8, bounds="exact")
    got = ctx.rsjoin(s, r, 0.8, bounds="exact")
    order = np.lexsort((got.q, got.s))
    assert np.array_equal(got.s[order], a.q) and np.array_equal(got.q[order], a.s)


def test_rsjoin_of_a_set_with_itself(ctx, titles_rs):
    """R joined with a copy of itself: every non-empty record pairs with its own
    copy (J = 1), plus the cross pairs of the self-join in both orientations."""
    _, _, (r, _) = titles_rs
    got = ctx.rsjoin(r, r, 0.9)
    ref, st = O.rsjoin((r.pos, r.len, r.tokens), (r.pos, r.len, r.tokens), r.n_terms, 0.9)
    _check_rs(got, ref, st)
    diag = got.q == got.s
    assert diag.sum() == r.n_sets


def test_rsjoin_empty_side_and_device_views(ctx, titles_rs):
    import torch
    _, _, (r, s) = titles_rs
    empty = F.Sets(np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32),
                   r.n_terms)
    assert len(ctx.rsjoin(r, empty, 0.7)) == 0 and len(ctx.rsjoin(empty, s, 0.7, method="plain")) == 0

    def dev(x):
        from new_fgssjoin_b200.binding import _View
        arrs = [torch.from_numpy(a.view(np.int32)).cuda() for a in (x.id, x.pos, x.len, x.tokens)]
        v = _View()
        v.id, v.pos, v.len, v.tokens = [a.data_ptr() for a in arrs]
        v.n_sets, v.n_tokens, v.n_terms, v.on_device = x.n_sets, x.n_tokens, x.n_terms, 1
        return v, arrs
    (vr, ar), (vs, as_) = dev(r), dev(s)
    ref, st = O.rsjoin((r.pos, r.len, r.tokens), (s.pos, s.len, s.tokens), r.n_terms, 0.7)
    _check_rs(ctx.rsjoin(vr, vs, 0.7), ref, st)


def test_rsjoin_rejects_bad_input(ctx, titles_rs):
    _, _, (r, s) = titles_rs
    bad = F.Sets(s.id, s.pos, s.len + 1, s.tokens, s.n_terms)  # last record runs past the tokens
    with pytest.raises(F.FgssError):
        ctx.rsjoin(r, bad, 0.7)
    got = ctx.rsjoin(r, s, 0.7)  # the context stays usable
    assert len(got) > 0
