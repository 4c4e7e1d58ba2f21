"""GPU parity: the CUDA join through the C ABI against the CPU oracle."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
import new_fgssjoin_b200 as F
from new_fgssjoin_b200 import datagen
from oracle import oracle as O

pytestmark = pytest.mark.gpu

THRESHOLDS = [0.5, 0.6, 0.7, 0.8, 0.9, 0.95]


def _check_same(got, ref, st=None):
    assert len(got) == len(ref)
    assert np.array_equal(got.q, ref["q"])
    assert np.array_equal(got.s, ref["s"])
    assert np.array_equal(got.overlap, ref["overlap"])
    assert np.array_equal(got.sim, ref["sim"])  # float32 division, bit-exact
    if st is not None:
        for k in ("candidates", "intersections", "results"):
            assert got.stats[k] == st[k], (k, got.stats, st)
        assert got.stats["index_entries"] == st["index_entries"]


@pytest.mark.parametrize("method", ["plain", "batched"])
@pytest.mark.parametrize("t", ["0.5", "0.59", "0.6", "0.7", "0.75", "0.8", "0.9"])
def test_golden_fixture_pairs(ctx, method, t):
    s = F.ppjoin_format(os.path.join(GOLDEN, "small.txt.3gram.bin"))
    got = ctx.selfjoin(s, float(t), method=method)
    gold = json.load(open(os.path.join(GOLDEN, "small_pairs.json")))[t]
    assert sorted(got.lines()) == gold


def _titles(n, seed):
    return datagen.titles(n, seed=seed)


@pytest.fixture(scope="module")
def titles_sets(ctx):
    return ctx.tokenize(_titles(6000, 11), **datagen.TITLE_TOK)


@pytest.mark.parametrize("method", ["plain", "batched"])
@pytest.mark.parametrize("t", THRESHOLDS)
def test_titles_vs_oracle(ctx, titles_sets, method, t):
    s = titles_sets
    got = ctx.selfjoin(s, t, method=method)
    ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
    _check_same(got, ref, st)


@pytest.mark.parametrize("t", [0.5, 0.6, 0.8])
def test_candidates_match_oracle(ctx, titles_sets, t):
    """The plain method's candidate list (q, s, partial score) equals the reference filter's cells > 0,
    restricted to the candidates a merge can still bring to floor(min overlap)."""
    s = titles_sets
    got = ctx.selfjoin(s, t, method="plain", want_candidates=True)
    ref, st, cands = O.join(s.pos, s.len, s.tokens, s.n_terms, t, want_candidates=True)
    assert got.stats["candidates"] == st["candidates"] == len(cands)
    gc = {(int(a), int(b)): int(c) for a, b, c in got.candidates}
    rc = {(int(a), int(b)): int(c) for a, b, c in cands}
    assert set(gc) <= set(rc)
    for k, v in gc.items():
        assert rc[k] == v  # same partial score
    # every pair the reference verifies to an intersection is among ours
    verified = set(zip(ref["q"].tolist(), ref["s"].tolist()))
    assert verified <= set(gc)


def _random_sets(rng, n, vocab, lo, hi, sort=True):
    lens = rng.integers(lo, hi + 1, n)
    if sort:
        lens = np.sort(lens)[::-1]
    toks = [np.sort(rng.choice(vocab, size=int(l), replace=False)) for l in lens]
    pos = np.zeros(n, np.uint32)
    if n > 1:
        pos[1:] = np.cumsum(lens[:-1])
    tok = np.concatenate(toks).astype(np.uint32) if n else np.zeros(0, np.uint32)
    return F.Sets(np.arange(1, n + 1), pos, lens, tok, vocab)


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("t", THRESHOLDS)
def test_random_small_vocab(ctx, seed, t):
    """Dense overlaps, equal sizes, lengths n = 0 (mod 9) and 0.6 n integral (float32 bound edges)."""
    rng = np.random.default_rng(seed * 131 + int(t * 1000))
    s = _random_sets(rng, 700, 60, 1, 45)
    for method in ("plain", "batched"):
        got = ctx.selfjoin(s, t, method=method)
        ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
        _check_same(got, ref, st)


@pytest.mark.parametrize("t", [0.6, 0.8])
def test_unsorted_input_matches_reference_semantics(ctx, t):
    """Records not in descending size: per-entry size filter and the one-tile skip test."""
    rng = np.random.default_rng(5)
    s = _random_sets(rng, 400, 50, 1, 30, sort=False)
    for method in ("plain", "batched"):
        got = ctx.selfjoin(s, t, method=method)
        ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
        _check_same(got, ref, st)


def test_empty_and_singleton_inputs(ctx):
    empty = F.Sets(np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), 0)
    one = F.Sets([7], [0], [3], [1, 2, 3], 4)
    for method in ("plain", "batched"):
        assert len(ctx.selfjoin(empty, 0.5, method=method)) == 0
        assert len(ctx.selfjoin(one, 0.5, method=method)) == 0


def test_empty_records_take_part_in_no_pair(ctx):
    s = F.Sets([1, 2, 3, 4], [0, 3, 6, 6], [3, 3, 0, 0], [1, 2, 3, 1, 2, 3], 4)
    got = ctx.selfjoin(s, 0.5)
    assert got.lines() == ["1 2 1.000000"]


def test_identical_records(ctx):
    n = 50
    tok = np.tile(np.arange(10, dtype=np.uint32), n)
    s = F.Sets(np.arange(1, n + 1), np.arange(n) * 10, np.full(n, 10), tok, 10)
    got = ctx.selfjoin(s, 0.9, method="batched")
    assert len(got) == n * (n - 1) // 2
    assert np.all(got.overlap == 10) and np.all(got.sim == 1.0)


def test_unsorted_tokens_rejected(ctx):
    s = F.Sets([1, 2], [0, 3], [3, 3], [3, 2, 1, 1, 2, 3], 4)
    with pytest.raises(F.FgssError) as e:
        ctx.selfjoin(s, 0.5)
    assert e.value.status == 4


def test_threshold_range(ctx, titles_sets):
    for t in (0.0, 1.0, -0.5, 1.5):
        with pytest.raises(F.FgssError) as e:
            ctx.selfjoin(titles_sets, t)
        assert e.value.status == 1


def test_exact_bounds_equal_rational_brute_force(ctx):
    rng = np.random.default_rng(9)
    s = _random_sets(rng, 300, 40, 1, 40)
    for t, (p, qd) in ((0.8, (4, 5)), (0.6, (3, 5))):
        got = ctx.selfjoin(s, t, bounds="exact")
        want = []
        for qi in range(s.n_sets):
            x = set(s.tokens[s.pos[qi]:s.pos[qi] + s.len[qi]].tolist())
            for si in range(qi + 1, s.n_sets):
                y = set(s.tokens[s.pos[si]:s.pos[si] + s.len[si]].tolist())
                o = len(x & y)
                if o and o * qd >= p * (len(x) + len(y) - o):
                    want.append((qi, si))
        assert list(zip(got.q.tolist(), got.s.tolist())) == want


def test_batch_of_joins_equals_single_joins(ctx):
    sets = [ctx.tokenize(_titles(n, 100 + n), **datagen.TITLE_TOK) for n in (500, 2500, 1200, 4000)]
    ts = [0.6, 0.7, 0.9, 0.8]
    outs = ctx.selfjoin_batch(sets, ts)
    for s, t, got in zip(sets, ts, outs):
        ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
        _check_same(got, ref, st)


def _long_and_short_records(seed):
    """A few records longer than the fused kernel's probe cap among short ones."""
    rng = np.random.default_rng(seed)
    base = rng.choice(8000, size=3000, replace=False)
    recs = [np.sort(np.delete(base, rng.choice(3000, size=int(rng.integers(0, 300)), replace=False)))
            for _ in range(12)]
    recs += [np.sort(rng.choice(8000, size=int(rng.integers(5, 60)), replace=False)) for _ in range(150)]
    return _sets_of(recs, 8000)


def test_batch_stage_launches_cover_every_join_kind(ctx):
    """One batched call whose per-stage launches span joins of every kind at once: empty,
    a single record, records without any pair, long records for the global accumulator,
    and title joins of several sizes and thresholds; every join equals its own oracle join
    and the launches do not grow with the number of joins."""
    empty = F.Sets(np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), 0)
    one = F.Sets([7], [0], [3], [1, 2, 3], 4)
    disjoint = F.Sets([1, 2, 3], [0, 3, 6], [3, 3, 3], [0, 1, 2, 3, 4, 5, 6, 7, 8], 9)
    titles = [ctx.tokenize(_titles(n, 300 + n), **datagen.TITLE_TOK) for n in (700, 2200, 1300)]
    sets = [titles[0], empty, _long_and_short_records(8), one, titles[1], disjoint, titles[2]]
    ts = [0.6, 0.7, 0.7, 0.5, 0.9, 0.5, 0.8]
    outs = ctx.selfjoin_batch(sets, ts, method="batched")
    for s, t, got in zip(sets, ts, outs):
        ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
        _check_same(got, ref, st)
    assert outs[2].stats["heavy_queries"] > 0
    few = ctx.selfjoin_batch(sets[:2], ts[:2], method="batched")[0].stats["launches"]
    # the same stages whatever the number of joins: only sort passes (wider keys) and the
    # global accumulator's launch come on top, where per-join stages would add about 75
    assert outs[0].stats["launches"] <= few + 30


def test_batch_of_many_small_joins(ctx):
    """Sixty joins in one call: the tile maps over many joins, with a shared host input."""
    base = ctx.tokenize(_titles(400, 77), **datagen.TITLE_TOK)
    small = [ctx.tokenize(_titles(int(n), 500 + i), **datagen.TITLE_TOK)
             for i, n in enumerate(np.linspace(20, 600, 30))]
    sets = [x for pair in zip(small, [base] * 30) for x in pair]
    ts = [0.5 + 0.45 * (i % 7) / 6 for i in range(len(sets))]
    outs = ctx.selfjoin_batch(sets, ts, method="batched")
    for s, t, got in zip(sets, ts, outs):
        ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
        _check_same(got, ref, st)


def test_batch_sharing_host_arrays(ctx, titles_sets):
    """Joins of one batched call on the same host arrays (copied to the device once)."""
    s = titles_sets
    ts = [0.6, 0.9, 0.75]
    for method in ("batched", "plain"):
        outs = ctx.selfjoin_batch([s, s, s], ts, method=method)
        for t, got in zip(ts, outs):
            ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
            _check_same(got, ref, st)


def test_long_records_take_the_heavy_path(ctx):
    """Records longer than the shared-memory caps go through the global accumulator."""
    rng = np.random.default_rng(4)
    base = rng.choice(8000, size=3000, replace=False)
    recs = []
    for i in range(30):
        r = base.copy()
        drop = rng.choice(len(r), size=int(rng.integers(0, 300)), replace=False)
        r = np.delete(r, drop)
        recs.append(np.sort(r))
    for i in range(200):
        recs.append(np.sort(rng.choice(8000, size=int(rng.integers(5, 60)), replace=False)))
    recs.sort(key=len, reverse=True)
    lens = np.array([len(r) for r in recs])
    pos = np.concatenate([[0], np.cumsum(lens[:-1])])
    s = F.Sets(np.arange(1, len(recs) + 1), pos, lens, np.concatenate(recs), 8000)
    for method in ("plain", "batched"):
        got = ctx.selfjoin(s, 0.7, method=method)
        ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, 0.7)
        _check_same(got, ref, st)
        assert got.stats["heavy_queries"] > 0


def _sets_of(recs, n_terms):
    recs = sorted(recs, key=len, reverse=True)  # memory order: descending size
    lens = np.array([len(r) for r in recs])
    pos = np.concatenate([[0], np.cumsum(lens[:-1])])
    return F.Sets(np.arange(1, len(recs) + 1), pos, lens, np.concatenate(recs).astype(np.uint32), n_terms)


def test_large_vocabulary_long_records_vs_oracle(ctx):
    """Vocabulary above 32,768 terms: queries of up to 512 tokens use the hashed
    query set, longer ones the hashed bitmap confirmed by binary search; near
    copies make long merges (the warp-cooperative path)."""
    rng = np.random.default_rng(21)
    V = 200000
    recs = []
    for _ in range(40):
        b = np.sort(rng.choice(V, int(rng.integers(300, 1100)), replace=False))
        recs.append(b)
        for _ in range(3):
            keep = b[rng.random(len(b)) > 0.04]
            recs.append(np.unique(np.concatenate([keep, rng.choice(V, 8, replace=False)])))
    for _ in range(300):
        recs.append(np.sort(rng.choice(V, int(rng.integers(5, 80)), replace=False)))
    s = _sets_of(recs, V)
    for t in (0.7, 0.9):
        ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
        assert st["results"] > 50
        for method in ("plain", "batched"):
            _check_same(ctx.selfjoin(s, t, method=method), ref, st)


@pytest.mark.parametrize("t", [0.6, 0.8])
def test_heavy_tailed_records_vs_oracle(ctx, t):
    """The heavy-tailed generator (lognormal sizes, near-duplicate clusters) at a small size."""
    s = ctx.tokenize(datagen.heavy(4000, seed=9), **datagen.TITLE_TOK)
    ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
    for method in ("plain", "batched"):
        _check_same(ctx.selfjoin(s, t, method=method), ref, st)


@pytest.mark.parametrize("filt", ["warp", "cta", "global"])
@pytest.mark.parametrize("t", [0.5, 0.8])
def test_filter_strategies_match_oracle(ctx, titles_sets, filt, t):
    """Every filter strategy of the batched method (a warp per query, a CTA per
    query, the global-memory accumulator for every query) gives the oracle's
    pairs and counters."""
    s = titles_sets
    got = ctx.selfjoin(s, t, method="batched", filter=filt)
    ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
    _check_same(got, ref, st)
    if filt == "global":
        assert got.stats["heavy_queries"] > 0


def test_global_accumulator_joins_of_different_sizes_in_turn():
    """The global-memory accumulator's per-source counters must be zero when a
    query starts, whatever join of whatever size used the scratch before: joins
    of 9,000, then 2,500, then 6,000 records in one context, each against the oracle."""
    with F.Context(device=0) as c2:
        for n, seed, t in ((9000, 41, 0.6), (2500, 42, 0.5), (6000, 43, 0.7)):
            s = c2.tokenize(datagen.titles(n, seed=seed), **datagen.TITLE_TOK)
            ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, t)
            for method, filt in (("batched", "global"), ("plain", "auto")):
                _check_same(c2.selfjoin(s, t, method=method, filter=filt), ref, st)


@pytest.mark.parametrize("filt", ["warp", "global"])
def test_filter_strategies_on_heavy_tailed_records(ctx, filt):
    s = ctx.tokenize(datagen.heavy(4000, seed=19), **datagen.TITLE_TOK)
    ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, 0.7)
    _check_same(ctx.selfjoin(s, 0.7, method="batched", filter=filt), ref, st)


def test_kmer_reads_vs_oracle(ctx):
    text = datagen.reads(3000, seed=3, genome_len=60000)
    s = ctx.tokenize(text, **datagen.READ_TOK)
    for method in ("plain", "batched"):
        got = ctx.selfjoin(s, 0.8, method=method)
        ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, 0.8)
        _check_same(got, ref, st)


def test_autotuner_picks_a_shape_and_caches_it(tmp_path, titles_sets):
    path = tmp_path / "tune.json"
    with F.Context(device=0, tune_cache_path=str(path)) as c2:
        best = c2.autotune(titles_sets, 0.7, reps=1)
        assert best["threads"] in (32, 64, 128, 256) and best["ms"] > 0
        assert best["filter"] in ("warp", "cta", "global")
        got = c2.selfjoin(titles_sets, 0.7, method="batched")
    ref, st = O.join(titles_sets.pos, titles_sets.len, titles_sets.tokens, titles_sets.n_terms, 0.7)
    _check_same(got, ref, st)
    txt = path.read_text()
    assert best["key"] in txt
    with F.Context(device=0, tune_cache_path=str(path)) as c3:  # reloads the cache
        got = c3.selfjoin(titles_sets, 0.7, method="batched")
        _check_same(got, ref, st)


@pytest.mark.parametrize("method", ["plain", "batched"])
def test_query_range_shards_reassemble_the_join(ctx, titles_sets, method):
    """A join split into query ranges (the multi-GPU sharding) gives the same pairs and counters."""
    from new_fgssjoin_b200.shard import shard_ranges
    s = titles_sets
    ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, 0.7)
    parts = [ctx.selfjoin(s, 0.7, method=method, query_range=r) for r in shard_ranges(s.len, 3)]
    assert np.array_equal(np.concatenate([p.q for p in parts]), ref["q"])
    assert np.array_equal(np.concatenate([p.s for p in parts]), ref["s"])
    assert sum(p.stats["candidates"] for p in parts) == st["candidates"]
    assert sum(p.stats["intersections"] for p in parts) == st["intersections"]


def test_query_costs_are_the_batched_work_estimates(ctx, titles_sets):
    """Without the model a query's cost is its window entries plus its size: the
    costs sum to the batched join's window-entry counter plus the record sizes."""
    s = titles_sets
    cost = ctx.query_costs(s, 0.7, use_model=False)
    got = ctx.selfjoin(s, 0.7, method="batched")
    assert len(cost) == s.n_sets and cost.dtype == np.uint64
    assert int(cost.sum()) == got.stats["window_entries"] + int(s.len.astype(np.uint64).sum())


def test_cost_balanced_shards_reassemble_the_join(ctx, titles_sets):
    """Query ranges cut by the learned cost estimates (as on several GPUs) give the full join."""
    from new_fgssjoin_b200.shard import shard_ranges
    s = titles_sets
    ctx.model_train([s], [0.7], epochs=50, lr=0.01, seed=3)
    cost = ctx.query_costs(s, 0.7, use_model=True)
    ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, 0.7)
    parts = [ctx.selfjoin(s, 0.7, method="batched", query_range=r, use_model=True)
             for r in shard_ranges(s.len, 4, cost)]
    assert np.array_equal(np.concatenate([p.q for p in parts]), ref["q"])
    assert np.array_equal(np.concatenate([p.s for p in parts]), ref["s"])
    assert sum(p.stats["candidates"] for p in parts) == st["candidates"]


def _device_view(sets):
    import torch
    from new_fgssjoin_b200.binding import _View
    arrs = [torch.from_numpy(a.view(np.int32)).cuda() for a in (sets.id, sets.pos, sets.len, sets.tokens)]
    v = _View()
    v.id, v.pos, v.len, v.tokens = [t.data_ptr() for t in arrs]
    v.n_sets, v.n_tokens, v.n_terms, v.on_device = sets.n_sets, sets.n_tokens, sets.n_terms, 1
    return v, arrs


def test_graph_replay_matches_and_follows_new_contents(ctx):
    """Batched joins on device inputs are captured into a CUDA graph on the first
    call and replayed on the next ones: same pairs, and a replay after the input
    contents changed (same pointers, same sizes) still gives the right pairs."""
    import torch
    a = ctx.tokenize(_titles(4000, 71), **datagen.TITLE_TOK)
    v, arrs = _device_view(a)
    ts = [0.6, 0.8]
    refs = [O.join(a.pos, a.len, a.tokens, a.n_terms, t) for t in ts]
    for call in range(3):  # record + capture, then two replays
        outs = ctx.selfjoin_batch([v, v], ts)
        for got, (ref, st) in zip(outs, refs):
            _check_same(got, ref, st)
    # new contents in the same buffers: term ids permuted, each record re-sorted
    perm = np.random.default_rng(5).permutation(a.n_terms).astype(np.uint32)
    tok = perm[a.tokens]
    for i in range(a.n_sets):
        tok[a.pos[i]:a.pos[i] + a.len[i]] = np.sort(tok[a.pos[i]:a.pos[i] + a.len[i]])
    arrs[3].copy_(torch.from_numpy(tok.view(np.int32)))
    c = F.Sets(a.id, a.pos, a.len, tok, a.n_terms)
    refs2 = [O.join(c.pos, c.len, c.tokens, c.n_terms, t) for t in ts]
    outs = ctx.selfjoin_batch([v, v], ts)
    for got, (ref, st) in zip(outs, refs2):
        _check_same(got, ref, st)


def test_graph_replay_with_results_beyond_capture_capacity(ctx):
    """When new contents produce more pairs than the captured capacity, the call
    falls back to the exact eager path."""
    import torch
    n, L = 3000, 12
    rng = np.random.default_rng(8)
    tok = np.concatenate([np.sort(rng.choice(5000, L, replace=False)) for _ in range(n)]).astype(np.uint32)
    s = F.Sets(np.arange(1, n + 1), np.arange(n) * L, np.full(n, L), tok, 5000)
    v, arrs = _device_view(s)
    ref, st = O.join(s.pos, s.len, s.tokens, s.n_terms, 0.9)
    for _ in range(2):
        _check_same(ctx.selfjoin_batch([v], [0.9])[0], ref, st)
    same = np.tile(tok[:L], n)  # every record identical: n(n-1)/2 results
    arrs[3].copy_(torch.from_numpy(same.view(np.int32)))
    s2 = F.Sets(s.id, s.pos, s.len, same, 5000)
    ref2, st2 = O.join(s2.pos, s2.len, s2.tokens, s2.n_terms, 0.9)
    got = ctx.selfjoin_batch([v], [0.9])[0]
    _check_same(got, ref2, st2)
    assert len(got) == n * (n - 1) // 2
    # the fallback recorded the batch again in the same buffers: later calls replay it
    for _ in range(2):
        got = ctx.selfjoin_batch([v], [0.9])[0]
        _check_same(got, ref2, st2)
        assert got.stats["overflow_retries"] == 0


def test_graph_captured_after_first_call_overflowed(ctx):
    """A first call whose presized result buffers overflow re-runs the join
    exactly and still captures the batch, with the exact capacity: the replays
    give the same pairs without a re-run."""
    a = ctx.tokenize(_titles(3000, 73), **datagen.TITLE_TOK)
    v, arrs = _device_view(a)
    ts = [0.5, 0.7, 0.9]
    refs = [O.join(a.pos, a.len, a.tokens, a.n_terms, t) for t in ts]
    first = ctx.selfjoin_batch([v] * 3, ts, result_capacity=1)
    for got, (ref, st) in zip(first, refs):
        _check_same(got, ref, st)
    assert sum(o.stats["overflow_retries"] for o in first) >= 1
    for _ in range(2):
        outs = ctx.selfjoin_batch([v] * 3, ts, result_capacity=1)
        for got, (ref, st) in zip(outs, refs):
            _check_same(got, ref, st)
            assert got.stats["overflow_retries"] == 0


@pytest.mark.parametrize("shards", [1, 5])
def test_streamed_output_equals_the_pairs(ctx, titles_sets, tmp_path, shards):
    """fgss_selfjoin_to_file: the text file equals the printed pairs line for line,
    the binary file holds the same (id, id, sim) records, the counters add up."""
    s = titles_sets
    ref = ctx.selfjoin(s, 0.7, method="batched")
    st = ctx.selfjoin_to_file(s, 0.7, str(tmp_path / "p.txt"), fmt="text", shards=shards)
    assert (tmp_path / "p.txt").read_text().splitlines() == ref.lines()
    for k in ("candidates", "intersections", "results"):
        assert st[k] == ref.stats[k]
    ctx.selfjoin_to_file(s, 0.7, str(tmp_path / "p.bin"), fmt="binary", shards=shards, method="plain")
    rec = np.fromfile(tmp_path / "p.bin", dtype=np.dtype([("q", "<u4"), ("s", "<u4"), ("sim", "<f4")]))
    assert np.array_equal(rec["q"], ref.id_q) and np.array_equal(rec["s"], ref.id_s)
    assert np.array_equal(rec["sim"], ref.sim)
