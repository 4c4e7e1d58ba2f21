"""The allocation-free scan entry point, checked against the regular one.

fgss_dev_exclusive_scan_u32_noalloc exists for callers that cannot call
cudaMalloc -- a host that reserves all device memory up front, or a loop
where an allocation (and the device-wide synchronization of cudaFree) is not
acceptable.  It keeps its scratch in a fixed array inside the library.  This
file is named to be collected last, so a run that stops at the first failure
has already run every other test; it passes on its own and after the rest.
"""
import ctypes

import numpy as np
import pytest
import torch

import new_fgssjoin_b200 as F

pytestmark = pytest.mark.gpu


def _noalloc(L, d_in, d_out, n, stream):
    return L.fgss_dev_exclusive_scan_u32_noalloc(ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
                                                 n, ctypes.c_void_p(stream))


def _want(a):
    incl = np.cumsum(a.astype(np.uint64))
    return ((incl - a.astype(np.uint64)) & np.uint64(0xFFFFFFFF)).astype(np.uint32)  # wraps like uint32


def test_noalloc_scan_matches_regular_scan_twice():
    L = F.load_library()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream(0)
    with F.Context(device=0, stream=stream.cuda_stream) as ctx:
        rng = np.random.default_rng(2024)
        # two calls in a row, the second on a smaller input: it must not see the
        # first call's scratch contents
        for n in (9_000_000, 123_457):
            a = rng.integers(0, 1 << 10, n).astype(np.uint32)
            d_in = torch.from_numpy(a.view(np.int32)).cuda()
            ref = torch.empty_like(d_in)
            got = torch.full_like(d_in, -1)
            ctx.dev_exclusive_scan_u32(d_in.data_ptr(), ref.data_ptr(), n)
            assert _noalloc(L, d_in, got, n, stream.cuda_stream) == 0
            torch.cuda.synchronize()
            assert torch.equal(got, ref)  # integer scan: exact
            assert np.array_equal(got.cpu().numpy().view(np.uint32), _want(a))


def test_noalloc_scan_in_place():
    """out == in: the header allows it, so check it against numpy."""
    L = F.load_library()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream(0)
    rng = np.random.default_rng(7)
    for n in (5_000_001, 4096):
        a = rng.integers(0, 1 << 31, n).astype(np.uint32)
        buf = torch.from_numpy(a.view(np.int32)).cuda()
        assert _noalloc(L, buf, buf, n, stream.cuda_stream) == 0
        torch.cuda.synchronize()
        assert np.array_equal(buf.cpu().numpy().view(np.uint32), _want(a))


def test_noalloc_scan_allocates_no_device_memory():
    """After a first call, further calls leave the device's free memory as it was."""
    L = F.load_library()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream(0)
    n = 3_000_000
    a = np.arange(n, dtype=np.uint32) % 977
    d_in = torch.from_numpy(a.view(np.int32)).cuda()
    out = torch.empty_like(d_in)
    assert _noalloc(L, d_in, out, n, stream.cuda_stream) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        assert _noalloc(L, d_in, out, n, stream.cuda_stream) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    assert np.array_equal(out.cpu().numpy().view(np.uint32), _want(a))


def test_noalloc_scan_rejects_sizes_beyond_its_scratch():
    L = F.load_library()
    torch.cuda.set_device(0)
    small = torch.zeros(16, dtype=torch.int32, device="cuda")
    # the size check comes before any kernel is queued, so nothing reads past `small`
    st = L.fgss_dev_exclusive_scan_u32_noalloc(ctypes.c_void_p(small.data_ptr()), ctypes.c_void_p(small.data_ptr()),
                                               65536 * 4096 + 1, None)
    assert st == 8  # FGSS_ERR_CAPACITY
    assert b"exceeds the fixed scratch limit" in L.fgss_last_error(None)
