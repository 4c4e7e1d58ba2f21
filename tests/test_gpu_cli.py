"""The fgssjoin command line (both argument forms, and the R-S form) on a B200."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN
from new_fgssjoin_b200 import datagen
from oracle import oracle as O
from rs_util import split_titles, oracle_dual

pytestmark = pytest.mark.gpu

CLI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "new_fgssjoin_b200", "_lib",
                   "fgssjoin")


def _run(args):
    p = subprocess.run([CLI] + args, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    counters = {k: int(v) for k, v in re.findall(r"# (Candidates|Intersections|Results): (\d+)", p.stderr)}
    return [x for x in p.stdout.splitlines() if x], counters


def test_reference_argument_form_prints_the_golden_pairs():
    for t in ("0.5", "0.7", "0.9"):
        lines, _ = _run([os.path.join(GOLDEN, "small.txt.3gram.bin"), t])
        assert sorted(lines) == json.load(open(os.path.join(GOLDEN, "small_pairs.json")))[t]


def test_text_form_matches_oracle(tmp_path):
    text = datagen.titles(3000, seed=21)
    f = tmp_path / "titles.txt"
    f.write_bytes(text)
    ids, lens, tok, loc, nt = O.tokenize(text, q=3, pad=True, suffix=False)
    mid, mpos, mlen, mtok = O.file_to_memory(ids, lens, tok)
    ref, st = O.join(mpos, mlen, mtok, nt, 0.8)
    want = ["%d %d %f" % (mid[q], mid[s], x) for q, s, x in zip(ref["q"], ref["s"], ref["sim"])]
    for extra in (["--method", "plain"], []):
        lines, cnt = _run(["-f", str(f), "-q", "3", "-t", "0.8", "--pad", "--distinct"] + extra)
        assert lines == want
        assert cnt == {"Candidates": st["candidates"], "Intersections": st["intersections"],
                       "Results": st["results"]}


def test_rs_form_matches_oracle(tmp_path):
    tr, ts = split_titles(3000, 22)
    (tmp_path / "r.txt").write_bytes(tr)
    (tmp_path / "s.txt").write_bytes(ts)
    (rid, rp, rl, rt), (sid, sp, sl, stk), nt = oracle_dual(tr, ts, q=3, pad=True, suffix=False)
    ref, st = O.rsjoin((rp, rl, rt), (sp, sl, stk), nt, 0.7)
    want = ["%d %d %f" % (rid[r], sid[s], x) for r, s, x in zip(ref["r"], ref["s"], ref["sim"])]
    lines, cnt = _run(["-f", str(tmp_path / "r.txt"), "-s", str(tmp_path / "s.txt"), "-q", "3", "-t", "0.7",
                       "--pad", "--distinct", "--method", "batched"])
    assert len(want) > 0 and lines == want
    assert cnt["Results"] == st["results"] and cnt["Candidates"] == st["candidates"]


def test_streamed_output_file(tmp_path):
    text = datagen.titles(3000, seed=23)
    f = tmp_path / "titles.txt"
    f.write_bytes(text)
    lines, cnt = _run(["-f", str(f), "-q", "3", "-t", "0.7", "--pad", "--distinct"])
    out = tmp_path / "pairs.txt"
    none, cnt2 = _run(["-f", str(f), "-q", "3", "-t", "0.7", "--pad", "--distinct", "--out", str(out),
                       "--shards", "3", "--method", "batched"])
    assert none == [] and len(lines) > 0
    assert out.read_text().splitlines() == lines and cnt2 == cnt


PRE = os.path.join(os.path.dirname(CLI), "preprocess")


def test_preprocess_selfjoin_writes_the_reference_fixture(tmp_path):
    """`preprocess selfjoin small.txt 3` (the reference's command) prints its
    counts and writes the reference's own fixture files byte for byte."""
    src = tmp_path / "small.txt"
    src.write_bytes(open(os.path.join(GOLDEN, "small.txt"), "rb").read())
    p = subprocess.run([PRE, "selfjoin", str(src), "3"], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert "Number of tokens: 88" in p.stdout and "Number of terms: 42" in p.stdout
    assert (tmp_path / "small.txt.3gram.bin").read_bytes() == \
        open(os.path.join(GOLDEN, "small.txt.3gram.bin"), "rb").read()
    assert (tmp_path / "small.txt.3gram.bin.loc").read_bytes() == \
        open(os.path.join(GOLDEN, "small.txt.3gram.bin.loc"), "rb").read()
    # and the join reads what it wrote
    lines, _ = _run([str(tmp_path / "small.txt.3gram.bin"), "0.7"])
    assert sorted(lines) == json.load(open(os.path.join(GOLDEN, "small_pairs.json")))["0.7"]


def test_preprocess_dualjoin_writes_both_files_over_one_vocabulary(tmp_path):
    """dualjoin tokenizes both files over one vocabulary (document frequency over
    both) and writes each as a .bin in file order, equal to the oracle's."""
    text_r, text_s = split_titles(2000, 31)
    fr, fs = tmp_path / "r.txt", tmp_path / "s.txt"
    fr.write_bytes(text_r)
    fs.write_bytes(text_s)
    p = subprocess.run([PRE, "dualjoin", str(fr), str(fs), "3", "--pad", "--distinct"], capture_output=True,
                       text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    r, s, nt = oracle_dual(text_r, text_s, **datagen.TITLE_TOK)
    assert "Number of terms: %d" % nt in p.stdout
    for path, (ids, pos, lens, toks) in ((fr, r), (fs, s)):
        order = range(len(ids))[::-1]  # file order: memory order reversed
        want = (np.asarray(ids)[::-1], np.asarray(lens)[::-1],
                np.concatenate([toks[pos[i]:pos[i] + lens[i]] for i in order]))
        got = O.decode_bin(open(str(path) + ".3gram.bin", "rb").read())
        for g, w_ in zip(got, want):
            assert np.array_equal(g, np.asarray(w_, dtype=np.uint32))
