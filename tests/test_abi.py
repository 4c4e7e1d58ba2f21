"""CPU: the C-ABI library loads, exports what include/fgss.h declares, and its
host-side parts (bound tables, .bin I/O) agree with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
import new_fgssjoin_b200 as F
from oracle import oracle as O


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "fgss.h")).read()
    declared = set(re.findall(r"\b(fgss_[a-z0-9_]+)\s*\(", hdr))
    L = F.load_library()
    missing = [s for s in sorted(declared) if not hasattr(L, s)]
    assert not missing, missing
    assert declared == set(F.EXPORTED_SYMBOLS)


def test_version_and_strerror():
    L = F.load_library()
    assert L.fgss_version() == 1
    assert L.fgss_strerror(4) == b"malformed input"


@pytest.mark.parametrize("t", [0.5, 0.6, 0.7, 0.75, 0.8, 0.9, 0.95])
def test_bound_tables_match_oracle_float32(t):
    """similarity.cuh float32 expressions, tabulated by the library on the host."""
    maxlen = 4000
    probe, index, mins, maxs, need = F.bounds_table(t, maxlen)
    qp, ip, mn, mx = O.bounds_table(t, maxlen)
    assert np.array_equal(probe[1:], qp[1:]) and np.array_equal(index[1:], ip[1:])
    assert probe[0] == 0 and index[0] == 0  # an empty record has no prefix
    assert np.array_equal(mins, mn) and np.array_equal(maxs, mx)


@pytest.mark.parametrize("t", [0.5, 0.6, 0.7, 0.8, 0.9, 0.95])
def test_need_table_equals_final_float_test(t):
    """The integer overlap bound is exactly block.cu:190-193 + checking.cu:167."""
    L = O.lib()
    maxlen = 600
    *_, need = F.bounds_table(t, maxlen)
    ft = ctypes.c_float(t)
    rng = np.random.default_rng(0)
    for _ in range(3000):
        a = int(rng.integers(1, maxlen + 1)); b = int(rng.integers(1, maxlen + 1))
        for o in range(max(0, int(need[a + b]) - 2), min(a, b, int(need[a + b]) + 2) + 1):
            mo = L.orc_min_overlap(ft, a, b)
            accept = o > 0 and o >= int(np.floor(mo)) and L.orc_similarity(a, b, o) >= np.float32(t)
            assert accept == (o >= need[a + b]), (a, b, o)


def test_exact_bounds_are_rational():
    probe, index, mins, maxs, need = F.bounds_table(0.8, 200, bounds="exact")
    for n in range(1, 201):
        assert probe[n] == n - (-(-4 * n // 5)) + 1
        assert index[n] == n - (-(-8 * n // 9)) + 1
    for S in range(1, 401):
        assert need[S] == max(1, -(-4 * S // 9))


def test_bin_roundtrip_and_memory_order(tmp_path):
    s = F.ppjoin_format(os.path.join(GOLDEN, "small.txt.3gram.bin"))
    assert list(s.id) == [4, 2, 3, 1, 5] and list(s.len) == [24, 19, 18, 16, 11]
    assert s.n_terms == 42
    # loc in memory order: records reversed
    ids, lens, tok = O.decode_bin(open(os.path.join(GOLDEN, "small.txt.3gram.bin"), "rb").read())
    loc_file = np.fromfile(os.path.join(GOLDEN, "small.txt.3gram.bin.loc"), dtype="<u4")
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    s.loc = np.concatenate([loc_file[off[i]:off[i + 1]] for i in range(len(lens))[::-1]]).astype(np.uint32)
    out = tmp_path / "x.bin"
    s.to_bin(str(out), str(out) + ".loc")
    assert out.read_bytes() == open(os.path.join(GOLDEN, "small.txt.3gram.bin"), "rb").read()
    assert (tmp_path / "x.bin.loc").read_bytes() == open(os.path.join(GOLDEN, "small.txt.3gram.bin.loc"), "rb").read()


def test_truncated_bin_is_a_format_error(tmp_path):
    raw = open(os.path.join(GOLDEN, "small.txt.3gram.bin"), "rb").read()
    p = tmp_path / "t.bin"
    p.write_bytes(raw[:-8])
    with pytest.raises(F.FgssError) as e:
        F.ppjoin_format(str(p))
    assert e.value.status == 4


def test_missing_bin_is_an_io_error(tmp_path):
    with pytest.raises(F.FgssError) as e:
        F.ppjoin_format(str(tmp_path / "nope.bin"))
    assert e.value.status == 5
