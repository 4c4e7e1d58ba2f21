"""CPU check of the overlap bound behind the fused kernel's bitmap filter: for
token sets x, y hashed into B-bit bitmaps by the kernel's hash (top bits of
x * 0x9E3779B1), |x & y| <= (|x| + |y| - popcount(b(x) ^ b(y))) / 2, so a
candidate whose bound is below floor(min overlap) can skip its merge."""
import numpy as np
import pytest


def _bitmap(tokens, bits):
    shift = 32 - int(np.log2(bits))
    h = ((np.asarray(tokens, dtype=np.uint64) * 0x9E3779B1) & 0xFFFFFFFF) >> shift
    b = np.zeros(bits, dtype=bool)
    b[h.astype(np.int64)] = True
    return b


@pytest.mark.parametrize("bits", [256, 512])
def test_bound_never_below_the_overlap(bits):
    rng = np.random.default_rng(bits)
    for _ in range(3000):
        n = int(rng.integers(1, 400))
        vocab = int(rng.choice([50, 500, 100000]))
        x = rng.choice(vocab, size=min(n, vocab), replace=False)
        share = rng.random()
        y = np.unique(np.concatenate([x[rng.random(len(x)) < share],
                                      rng.choice(vocab, size=int(rng.integers(0, 400)))]))
        o = len(np.intersect1d(x, y))
        pc = int(np.count_nonzero(_bitmap(x, bits) ^ _bitmap(y, bits)))
        assert 2 * o <= len(x) + len(y) - pc
