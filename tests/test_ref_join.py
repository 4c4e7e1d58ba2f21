"""The reference's own GPU join (oracle/_ref/ref_join: its kernels compiled
unchanged, driven with one tile).

CPU: the harness refuses, before any CUDA call, the inputs its reading showed
unsafe (more than 46,340 records; an empty record).  GPU: on the fixture and
on the 18,000-title configuration its pairs and counters equal the oracle's
and this library's.  Skipped where the harness was not built."""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from oracle import oracle as O

REF_JOIN = os.path.join(ROOT, "oracle", "_ref", "ref_join")
needs_harness = pytest.mark.skipif(not os.path.exists(REF_JOIN), reason="reference join harness not built")


def run_ref_join(path, t, out):
    p = subprocess.run([REF_JOIN, path, repr(float(t)), out], capture_output=True, text=True, timeout=600)
    if p.returncode != 0:
        return p, None
    raw = open(out, "rb").read()
    n, cand, inter, paired = struct.unpack("<4Q", raw[:32])
    ms = struct.unpack("<d", raw[32:40])[0]
    tri = np.frombuffer(raw[40:], dtype="<u4").reshape(-1, 3)
    assert len(tri) == n
    return p, {"pairs": tri, "candidates": cand, "intersections": inter, "paired_results": paired, "ms": ms}


@needs_harness
def test_harness_refuses_more_than_46340_records(tmp_path):
    n = 46341
    rec = np.zeros((n, 3), dtype="<i4")
    rec[:, 0] = np.arange(1, n + 1)
    rec[:, 1] = 1
    rec[:, 2] = np.arange(n) % 7
    f = tmp_path / "many.bin"
    f.write_bytes(rec.tobytes())
    p, r = run_ref_join(str(f), 0.9, str(tmp_path / "o"))
    assert p.returncode == 2 and "refused" in p.stderr and r is None


@needs_harness
def test_harness_refuses_an_empty_record(tmp_path):
    raw = O.encode_bin(np.array([1, 2], np.uint32), np.array([0, 2], np.uint32), np.array([3, 5], np.uint32))
    f = tmp_path / "empty.bin"
    f.write_bytes(raw)
    p, r = run_ref_join(str(f), 0.5, str(tmp_path / "o"))
    assert p.returncode == 2 and "empty record" in p.stderr
