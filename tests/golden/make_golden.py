"""Regenerates the golden fixtures under tests/golden/ (run in a checkout that
has the reference project next to it; the GPU tests only read the copies).

- small.txt, small.txt.3gram.bin, small.txt.3gram.bin.loc: copied verbatim from
  the reference's test/data/string/ (its only known-answer fixture for the
  tokenizer and the .bin format).
- small_pairs.json: the golden pairs of that fixture at several thresholds,
  computed by brute force over the decoded .bin (every pair, exact overlap,
  the reference's final float test) -- the expected stdout of
  ``fgssjoin small.txt.3gram.bin <t>`` as sorted "id id sim" lines.
"""
import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FGSS_REFERENCE", "/root/reference")


def main():
    src = os.path.join(REF, "test", "data", "string")
    for f in ("small.txt", "small.txt.3gram.bin", "small.txt.3gram.bin.loc"):
        shutil.copyfile(os.path.join(src, f), os.path.join(HERE, f))
    raw = open(os.path.join(HERE, "small.txt.3gram.bin"), "rb").read()
    a = np.frombuffer(raw, dtype="<i4")
    recs = []
    i = 0
    while i < len(a):
        n = int(a[i + 1]); recs.append((int(a[i]), [int(x) for x in a[i + 2:i + 2 + n]])); i += 2 + n
    mem = recs[::-1]                      # data.cu:97-113: memory order is the file reversed
    out = {}
    for t in (0.5, 0.59, 0.6, 0.7, 0.75, 0.8, 0.9):
        tf = np.float32(t)
        lines = []
        for qi in range(len(mem)):
            for si in range(qi + 1, len(mem)):
                x, y = mem[qi][1], mem[si][1]
                o = len(set(x) & set(y))
                if o == 0:
                    continue
                mo = np.float32(np.float32(tf / np.float32(1 + tf)) * np.float32(len(x) + len(y)))
                if o < int(np.floor(mo)):
                    continue
                sim = np.float32(np.float32(o) / np.float32(len(x) + len(y) - o))
                if sim >= tf:
                    lines.append("%d %d %f" % (mem[qi][0], mem[si][0], float(sim)))
        out["%g" % t] = sorted(lines)
    with open(os.path.join(HERE, "small_pairs.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
