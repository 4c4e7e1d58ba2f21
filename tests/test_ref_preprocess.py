"""CPU: token and term counts pinned against the reference's own preprocess
binary (built from its sources by oracle/ref_build.sh into oracle/_ref/).
Skipped where the reference checkout or the binary is absent."""
import os
import re
import subprocess

import pytest

from conftest import GOLDEN, REFERENCE, ROOT
from oracle import oracle as O

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "preprocess")
DBLP = os.path.join(REFERENCE, "test", "data", "string", "dblp_t_18k.txt")


def _sdbm(b):
    h = 0
    for c in b:
        h = (c + (h << 6) + (h << 16) - h) & 0xFFFFFFFFFFFFFFFF
    return h


def _ref_counts(path):
    out = subprocess.run([REF_BIN, "selfjoin", path, "3"], capture_output=True, text=True, timeout=120).stdout
    return (int(re.search(r"Number of tokens: (\d+)", out).group(1)),
            int(re.search(r"Number of terms: (\d+)", out).group(1)))


def _last_hash_is_singleton(text):
    """The reference's Df loop (preprocess_cli.cpp:293-306) folds the last sorted
    hash into the previous term when it occurs once; its term count is then one
    short."""
    hs = {}
    for line in text.split(b"\n"):
        if not line:
            continue
        s = bytes(c + 32 if 65 <= c <= 90 else c for c in line)
        occ = {}
        for p in range(len(s) - 2):
            g = s[p:p + 3]
            o = occ.get(g, -1) + 1
            occ[g] = o
            h = _sdbm(g + str(o).encode())
            hs[h] = hs.get(h, 0) + 1
    return hs[max(hs)] == 1


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference preprocess binary not built")
@pytest.mark.parametrize("path", [os.path.join(GOLDEN, "small.txt"), DBLP])
def test_counts_match_reference_binary(path):
    if not os.path.exists(path):
        pytest.skip("reference data file absent")
    text = open(path, "rb").read()
    ids, lens, tok, loc, nterms = O.tokenize(text, q=3, pad=False, suffix=True, lower=True)
    ref_tokens, ref_terms = _ref_counts(path)
    assert len(tok) == ref_tokens
    assert nterms == ref_terms + (1 if _last_hash_is_singleton(text) else 0)
