"""Allocation-free tile-count scan against the workspace entry point.

``r2s_scan_tile_counts_noalloc`` keeps its scratch in a static device array;
``r2s_scan_tile_counts`` takes a caller workspace. Both must give the same
int64 inclusive prefix sums (bit-exact: integer work), on two calls in a row,
since the second call reuses the static scratch the first one left behind.
"""

import gc

import pytest
import torch

from r2splat_b200.cuda import _backend

pytestmark = pytest.mark.gpu


def _stream(device):
    return torch.cuda.current_stream(device).cuda_stream


def _scan_with_workspace(counts):
    n = counts.numel()
    lib = _backend.library()
    ws = torch.empty(int(lib.r2s_isect_count_workspace(n)), dtype=torch.uint8, device=counts.device)
    cum = torch.empty(n, dtype=torch.int64, device=counts.device)
    _backend.call("r2s_scan_tile_counts", counts.data_ptr(), n, cum.data_ptr(), ws.data_ptr(), ws.numel(),
                  _stream(counts.device))
    return cum


def _scan_no_alloc(counts, cum):
    _backend.call("r2s_scan_tile_counts_noalloc", counts.data_ptr(), counts.numel(), cum.data_ptr(),
                  _stream(counts.device))


@pytest.mark.parametrize("n", [1, 4096, 4097, 1_000_003, 1 << 25])
def test_no_alloc_scan_matches_workspace_scan_twice(device, n):
    limit = int(_backend.library().r2s_scan_tile_counts_noalloc_max())
    assert limit == 1 << 25
    gen = torch.Generator(device="cpu").manual_seed(n)
    first = torch.randint(0, 65, (n,), generator=gen, dtype=torch.int32).to(device)
    second = torch.randint(0, 3, (n,), generator=gen, dtype=torch.int32).to(device)
    for counts in (first, second):
        expected = _scan_with_workspace(counts)
        cum = torch.full((n,), -1, dtype=torch.int64, device=device)
        gc.collect()
        torch.cuda.synchronize(device)
        allocations = torch.cuda.memory_stats(device).get("allocation.all.allocated", 0)
        _scan_no_alloc(counts, cum)
        torch.cuda.synchronize(device)
        # The cumulative allocation count of the caching allocator must not move.
        assert torch.cuda.memory_stats(device).get("allocation.all.allocated", 0) == allocations
        assert torch.equal(cum, expected)
        assert torch.equal(cum, torch.cumsum(counts.to(torch.int64), 0))


def test_no_alloc_scan_rejects_sizes_beyond_its_scratch(device):
    limit = int(_backend.library().r2s_scan_tile_counts_noalloc_max())
    # Buffers large enough for the claimed size, so the call is in bounds even
    # though the host check refuses it before any launch.
    counts = torch.zeros(limit + 1, dtype=torch.int32, device=device)
    cum = torch.full((limit + 1,), -7, dtype=torch.int64, device=device)
    with pytest.raises(RuntimeError, match="exceeds the static scratch limit"):
        _backend.call("r2s_scan_tile_counts_noalloc", counts.data_ptr(), limit + 1, cum.data_ptr(),
                      _stream(device))
    torch.cuda.synchronize(device)
    assert bool((cum == -7).all())
    # The entry point stays usable after a rejected call.
    small = torch.arange(10, dtype=torch.int32, device=device)
    out = torch.empty(10, dtype=torch.int64, device=device)
    _scan_no_alloc(small, out)
    assert torch.equal(out, torch.cumsum(small.to(torch.int64), 0))
