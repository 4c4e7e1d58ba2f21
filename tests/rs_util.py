"""Helpers of the R-S join tests."""
from new_fgssjoin_b200 import datagen
from oracle import oracle as O


def split_titles(n, seed):
    """n title records dealt alternately into an R text and an S text (the
    generator's perturbed copies then give pairs across)."""
    lines = datagen.titles(n, seed=seed).split(b"\n")[:-1]
    return b"\n".join(lines[0::2]) + b"\n", b"\n".join(lines[1::2]) + b"\n"


def oracle_dual(text_r, text_s, **tok):
    return O.tokenize_dual(text_r, text_s, **tok)
