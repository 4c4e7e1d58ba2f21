"""GPU scan and radix sort primitives against numpy."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 31, 4096, 4097, 100000, 3_000_001])
def test_exclusive_scan(ctx, n):
    rng = np.random.default_rng(n)
    a = rng.integers(0, 1000, n).astype(np.uint32)
    d_in = torch.from_numpy(a.view(np.int32)).cuda()
    d_out = torch.empty_like(d_in)
    ctx.dev_exclusive_scan_u32(d_in.data_ptr(), d_out.data_ptr(), n)
    incl = np.cumsum(a.astype(np.uint64))
    want = ((incl - a.astype(np.uint64)) & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    assert np.array_equal(d_out.cpu().numpy().view(np.uint32), want)


@pytest.mark.parametrize("n,bits", [(1, 8), (1000, 13), (70000, 64), (1_000_003, 40)])
def test_radix_sort_stable(ctx, n, bits):
    rng = np.random.default_rng(bits)
    k = rng.integers(0, 2 ** 63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
    if bits < 64:
        k &= np.uint64((1 << bits) - 1)
    k[::7] = k[0]  # duplicates to exercise stability
    v = np.arange(n, dtype=np.uint32)
    dk = torch.from_numpy(k.view(np.int64)).cuda()
    dv = torch.from_numpy(v.view(np.int32)).cuda()
    ctx.dev_sort_pairs_u64(dk.data_ptr(), dv.data_ptr(), n, 0, bits)
    order = np.argsort(k, kind="stable")
    assert np.array_equal(dk.cpu().numpy().view(np.uint64), k[order])
    assert np.array_equal(dv.cpu().numpy().view(np.uint32), v[order])
