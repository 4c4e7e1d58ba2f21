"""Helpers of the R-S join tests: two title files over one vocabulary, split
by the oracle the way fgss_tokenize_dual splits them."""
import numpy as np

from new_fgssjoin_b200 import datagen
from oracle import oracle as O


def split_titles(n, seed):
    """n title records dealt alternately into an R text and an S text (the
    generator's perturbed copies then give pairs across)."""
    lines = datagen.titles(n, seed=seed).split(b"\n")[:-1]
    return b"\n".join(lines[0::2]) + b"\n", b"\n".join(lines[1::2]) + b"\n"


def oracle_dual(text_r, text_s, **tok):
    """Oracle tokenization of R's text then S's text as one input, split into
    the two sides: ((id, pos, len, tokens) of R, same of S, n_terms)."""
    if text_r and not text_r.endswith(b"\n"):
        text_r = text_r + b"\n"
    nr = sum(1 for x in text_r.split(b"\n") if x)
    ids, lens, tok, loc, nt = O.tokenize(text_r + text_s, **tok)
    mid, mpos, mlen, mtok = O.file_to_memory(ids, lens, tok)

    def side(mask, shift):
        ln = mlen[mask]
        t = np.concatenate([mtok[p:p + n] for p, n in zip(mpos[mask], ln)]) if len(ln) else np.zeros(0, np.uint32)
        p = np.concatenate([[0], np.cumsum(ln[:-1])]).astype(np.uint32) if len(ln) else np.zeros(0, np.uint32)
        return mid[mask] - shift, p, ln, t.astype(np.uint32)
    return side(mid <= nr, 0), side(mid > nr, nr), nt
