"""GPU: the reference's own join kernels (oracle/_ref/ref_join, its sources
compiled unchanged and driven with one tile) against the oracle and this
library: the pairs with their overlaps and the reference's counters.  This
pins the oracle's join on reference code, and times the reference's GPU path
on the 18,000-title configuration (printed)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
import new_fgssjoin_b200 as F
from new_fgssjoin_b200 import datagen
from oracle import oracle as O
from test_ref_join import REF_JOIN, run_ref_join

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(REF_JOIN), reason="reference join harness not built")]


@pytest.mark.parametrize("t", ["0.5", "0.59", "0.7", "0.9"])
def test_reference_kernels_give_the_golden_fixture_pairs(tmp_path, t):
    path = os.path.join(GOLDEN, "small.txt.3gram.bin")
    p, r = run_ref_join(path, t, str(tmp_path / "o"))
    assert p.returncode == 0, p.stderr
    s = F.ppjoin_format(path)
    lines = ["%d %d %f" % (s.id[q], s.id[w], np.float32(o) / np.float32(s.len[q] + s.len[w] - o))
             for q, w, o in r["pairs"]]
    assert sorted(lines) == json.load(open(os.path.join(GOLDEN, "small_pairs.json")))[t]


@pytest.mark.parametrize("n,t", [(18_000, 0.9), (5_000, 0.6), (5_000, 0.8)])
def test_reference_kernels_equal_oracle_and_library(ctx, tmp_path, n, t):
    """The 18,000-title configuration (t = 0.9; the pair set must equal the
    reference's) and the float32-boundary thresholds 0.6 / 0.8."""
    sets = ctx.tokenize(datagen.titles(n, seed=1), **datagen.TITLE_TOK)
    path = str(tmp_path / "titles.bin")
    sets.to_bin(path)
    p, r = run_ref_join(path, t, str(tmp_path / "o"))
    assert p.returncode == 0, p.stderr
    ref, st = O.join(sets.pos, sets.len, sets.tokens, sets.n_terms, t)
    got = ctx.selfjoin(sets, t, method="batched")
    pr = r["pairs"]
    assert np.array_equal(pr[:, 0], ref["q"]) and np.array_equal(pr[:, 1], ref["s"])
    assert np.array_equal(pr[:, 2], ref["overlap"])
    assert np.array_equal(got.q, ref["q"]) and np.array_equal(got.s, ref["s"])
    assert r["candidates"] == st["candidates"] == got.stats["candidates"]
    assert r["intersections"] == st["intersections"] == got.stats["intersections"]
    print("reference kernels, %d titles, t = %.2f: %.1f ms (prepare + index + filter + verify + results); "
          "results paired as the reference prints them: %d of %d"
          % (n, t, r["ms"], r["paired_results"], len(pr)))
