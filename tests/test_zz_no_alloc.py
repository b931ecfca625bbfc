"""The allocation-free scan entry point matches the pooled one.

shn_exclusive_scan_u32_noalloc serves callers that cannot take a device
allocation on their hot path (an engine that has pre-claimed device memory
for its own allocator, a loop with an already-committed memory budget): its
look-back scratch is a fixed static device array instead of a pool
allocation.  This file is collected last on purpose, so a failure here
cannot hide the results of the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scan_both(shn, torch, x):
    lib = shn._abi.load()
    ctx = shn.default_context()
    d_in = torch.from_numpy(x.view(np.int32)).cuda()
    ref = torch.empty(x.size + 1, dtype=torch.int32, device="cuda")
    out = torch.full((x.size + 1,), -1, dtype=torch.int32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = lib.shn_exclusive_scan_u32(ctx.handle, C.c_void_p(d_in.data_ptr()), C.c_void_p(ref.data_ptr()),
                                    x.size, stream)
    assert st == 0
    st = lib.shn_exclusive_scan_u32_noalloc(C.c_void_p(d_in.data_ptr()), C.c_void_p(out.data_ptr()),
                                            x.size, stream)
    assert st == 0
    torch.cuda.synchronize()
    return ref.cpu().numpy().view(np.uint32), out.cpu().numpy().view(np.uint32)


def _status(shn, torch):
    lib = shn._abi.load()
    return lib.shn_exclusive_scan_u32_noalloc_status(C.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_noalloc_scan_matches_pooled_scan_twice(gpu):
    import torch

    import shinobi_b200 as shn
    rng = np.random.default_rng(7)
    # two calls in a row with different sizes: the second must not see the
    # first call's leftovers in the shared scratch array
    for n in (3_000_017, 1_234_567):
        x = rng.integers(0, 1000, size=n, dtype=np.uint32)
        ref, out = _scan_both(shn, torch, x)
        assert np.array_equal(out, ref)
        assert out[-1] == np.uint32(x.astype(np.uint64).sum() & 0xFFFFFFFF)
        assert _status(shn, torch) == 0


@pytest.mark.parametrize("n", [0, 1, 2047, 2048, 2049, 1 << 24])
def test_noalloc_scan_boundary_sizes(gpu, n):
    """Empty input, one element, one tile and a bit more, and the maximum size
    (all 8192 tiles of the fixed array)."""
    import torch

    import shinobi_b200 as shn
    rng = np.random.default_rng(n + 3)
    x = rng.integers(0, 50, size=n, dtype=np.uint32)
    ref, out = _scan_both(shn, torch, x)
    assert np.array_equal(out, ref)
    assert _status(shn, torch) == 0


def test_noalloc_scan_reports_a_wait_that_gave_up(gpu):
    """A call whose first tile is withheld: the other tiles' bounded look-back
    waits run out and shn_exclusive_scan_u32_noalloc_status reports it; the
    report clears the error, and the next call is correct."""
    import torch

    import shinobi_b200 as shn
    lib = shn._abi.load()
    rng = np.random.default_rng(11)
    x = rng.integers(0, 1000, size=100_000, dtype=np.uint32)
    assert lib.shn_debug_force_lookback_timeout(shn._abi.SHN_FORCE_NOALLOC_SCAN, None, None) == 0
    _scan_both(shn, torch, x)
    assert _status(shn, torch) == shn._abi.SHN_ERR_TIMEOUT
    ref, out = _scan_both(shn, torch, x)
    assert np.array_equal(out, ref)
    assert _status(shn, torch) == 0


def test_noalloc_scan_rejects_sizes_beyond_the_maximum(gpu):
    import torch

    import shinobi_b200 as shn
    lib = shn._abi.load()
    d = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib.shn_exclusive_scan_u32_noalloc(C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()),
                                            (1 << 24) + 1, None)
    assert st == 1  # SHN_ERR_INVALID, nothing launched
