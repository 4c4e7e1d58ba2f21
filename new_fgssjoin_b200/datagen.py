"""Seeded synthetic workloads standing in for the reference's DBLP-title data.

The reference measured on DBLP titles (test/data/string/dblp_t_18k.txt and
larger files not shipped, .MISSING_LARGE_BLOBS); the workloads here are
seeded synthetic text of the same shape, generated with numpy:

- ``titles``: records of 5-15 words drawn Zipf(s=1.1) from a vocabulary of
  50,000 lowercase words of 3-10 letters, space-joined; a fraction of the
  records are copies of earlier records with 1-3 random character edits
  (config "18k/100k titles", t = 0.5 ... 0.9).
- ``heavy``: word counts lognormal(mu=2.5, sigma=1.0) clipped to 2-600, with
  5 % of the records in near-duplicate clusters of 2-20 perturbed copies
  (config "1M heavy-tailed records", t = 0.7).
- ``reads``: 150-base reads sampled from a seeded random 5 Mbp genome with a
  0.5 % substitution rate, one read per line, for canonical 16-mer sets.

Every generator returns ``bytes`` (lines separated by '\\n') and is
deterministic in its seed.
"""
import numpy as np

LETTERS = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz", dtype=np.uint8)


def _vocab(rng, n_words=50000, lo=3, hi=10):
    lens = rng.integers(lo, hi + 1, n_words)
    chars = LETTERS[rng.integers(0, 26, (n_words, hi))]
    return chars, lens


def _zipf_ids(rng, n, n_words, s):
    ranks = np.arange(1, n_words + 1, dtype=np.float64)
    w = ranks ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return np.searchsorted(cdf, rng.random(n), side="right").clip(0, n_words - 1)


def _render(chars, lens, word_ids, words_per_rec):
    """Word ids + words per record -> list of per-record byte strings (space-joined)."""
    wl = lens[word_ids]
    # per word: its letters followed by a separator (space, or newline at record end)
    tot = wl + 1
    out_len = int(tot.sum())
    starts = np.zeros(len(word_ids) + 1, dtype=np.int64)
    np.cumsum(tot, out=starts[1:])
    buf = np.empty(out_len, dtype=np.uint8)
    # letter positions
    rep_w = np.repeat(np.arange(len(word_ids)), wl)
    # within-word offset = global letter index - first letter index of its word
    first_letter = np.zeros(len(word_ids) + 1, dtype=np.int64)
    np.cumsum(wl, out=first_letter[1:])
    within = np.arange(int(wl.sum())) - np.repeat(first_letter[:-1], wl)
    buf[np.repeat(starts[:-1], wl) + within] = chars[word_ids[rep_w], within]
    sep = starts[1:] - 1
    buf[sep] = ord(" ")
    rec_end = np.cumsum(words_per_rec) - 1
    buf[sep[rec_end]] = ord("\n")
    text = buf.tobytes()
    lines = text.split(b"\n")[:-1]
    return lines


def _perturb(rng, line, n_edits):
    b = bytearray(line)
    for _ in range(n_edits):
        op = rng.integers(0, 3)
        if len(b) <= 1:
            op = 2
        p = int(rng.integers(0, max(1, len(b))))
        c = int(LETTERS[rng.integers(0, 26)])
        if op == 0:
            b[p] = c
        elif op == 1:
            del b[p]
        else:
            b.insert(p, c)
    return bytes(b)


def titles(n_records, seed=0, n_words=50000, zipf_s=1.1, min_words=5, max_words=15, dup_frac=0.10):
    """Title-like records; ``dup_frac`` of them are 1-3-edit copies of earlier records."""
    rng = np.random.default_rng(seed)
    chars, lens = _vocab(rng, n_words)
    wpr = rng.integers(min_words, max_words + 1, n_records)
    ids = _zipf_ids(rng, int(wpr.sum()), n_words, zipf_s)
    lines = _render(chars, lens, ids, wpr)
    n_dup = int(round(dup_frac * n_records))
    if n_dup and n_records > 1:
        targets = rng.choice(np.arange(1, n_records), size=min(n_dup, n_records - 1), replace=False)
        for i in np.sort(targets):
            j = int(rng.integers(0, i))
            lines[i] = _perturb(rng, lines[j], int(rng.integers(1, 4)))
    return b"\n".join(lines) + b"\n"


def heavy(n_records, seed=0, n_words=50000, zipf_s=1.1, mu=2.5, sigma=1.0, lo=2, hi=600, cluster_frac=0.05):
    """Heavy-tailed record sizes with near-duplicate clusters of 2-20 copies."""
    rng = np.random.default_rng(seed)
    chars, lens = _vocab(rng, n_words)
    wpr = np.clip(np.round(rng.lognormal(mu, sigma, n_records)), lo, hi).astype(np.int64)
    ids = _zipf_ids(rng, int(wpr.sum()), n_words, zipf_s)
    lines = _render(chars, lens, ids, wpr)
    # clusters: pick bases, overwrite following random records with perturbed copies
    want = int(round(cluster_frac * n_records))
    placed = 0
    free = rng.permutation(n_records)
    k = 0
    while placed < want and k + 1 < n_records:
        size = int(rng.integers(2, 21))
        base = int(free[k]); k += 1
        for _ in range(size - 1):
            if k >= n_records or placed >= want:
                break
            dst = int(free[k]); k += 1
            lines[dst] = _perturb(rng, lines[base], int(rng.integers(1, 4)))
            placed += 1
        placed += 1
    return b"\n".join(lines) + b"\n"


def reads(n_reads, seed=0, genome_len=5_000_000, read_len=150, sub_rate=0.005):
    """Reads of ``read_len`` bases from a random genome, with substitutions."""
    rng = np.random.default_rng(seed)
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    genome = rng.integers(0, 4, genome_len, dtype=np.uint8)
    starts = rng.integers(0, genome_len - read_len + 1, n_reads)
    idx = starts[:, None] + np.arange(read_len)[None, :]
    r = genome[idx]
    mask = rng.random(r.shape) < sub_rate
    shift = rng.integers(1, 4, r.shape, dtype=np.uint8)
    r = np.where(mask, (r + shift) % 4, r).astype(np.uint8)
    out = np.empty((n_reads, read_len + 1), dtype=np.uint8)
    out[:, :read_len] = acgt[r]
    out[:, read_len] = ord("\n")
    return out.tobytes()


def batch_sizes(n_joins=256, lo=1000, hi=200000, seed=0):
    """Log-uniform join sizes and thresholds of the 256-join batch workload."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), n_joins)).astype(np.int64)
    ts = rng.choice(np.array([0.6, 0.7, 0.8, 0.9, 0.95]), n_joins)
    return sizes, ts


# tokenization of the workloads: padded lower-case 3-grams, distinct per record
TITLE_TOK = dict(q=3, mode="qgram", pad=True, suffix=False, lower=True)
READ_TOK = dict(q=16, mode="kmer", pad=False, suffix=False, lower=True)


def main(argv=None):
    """Writes one of the synthetic workloads' texts to a file (one record per line):
    python -m new_fgssjoin_b200.datagen heavy|titles <records> [--seed S] --out <path>."""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m new_fgssjoin_b200.datagen")
    ap.add_argument("kind", choices=["heavy", "titles"])
    ap.add_argument("records", type=int)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    text = (heavy if a.kind == "heavy" else titles)(a.records, seed=a.seed)
    with open(a.out, "wb") as f:
        f.write(text if isinstance(text, (bytes, bytearray)) else text.encode())


if __name__ == "__main__":
    main()
