"""The allocation-free entry point, bg_traversal_counts_noalloc.

It is for callers that cannot let this library allocate device memory: an
application that reserves the device's memory for its own pool up front, or a
profiling harness whose measurements cudaFree's implicit synchronisation would
disturb.  It must give the same node and triangle counts as
bg_traversal_counts (integer counts of the same traversal: exact equality), on
two calls in a row (the static scratch keeps the previous call's contents, so
the second call checks that the counters are cleared), and reject ray counts
beyond its static scratch with a clear error.  With the library's allocation
cap at zero (bg_alloc_limit) it must still work -- it allocates nothing --
while the allocating entry point is refused.  Kept in a file of its own that
is collected last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_counts_match_allocating_entry_point():
    import torch
    from banshee_b200 import capi, scenes

    ctx = capi.Context(0)
    gs = capi.GpuScene(ctx, scenes.soup(50_000, seed=21))
    for any_hit in (False, True):
        rays = scenes.soup_rays(200_000, "incoherent", seed=22, any_hit=any_hit)
        dr = torch.from_numpy(rays.view(np.uint8)).cuda()
        torch.cuda.synchronize()
        want = gs.traversal_counts(dr.data_ptr(), rays.shape[0], any_hit=any_hit)
        assert want[0] > 0 and want[1] > 0
        first = gs.traversal_counts_noalloc(dr.data_ptr(), rays.shape[0], any_hit=any_hit)
        second = gs.traversal_counts_noalloc(dr.data_ptr(), rays.shape[0], any_hit=any_hit)
        assert first == want, (first, want)
        assert second == want, (second, want)
    # a ragged, smaller call after a larger one: counters restart from zero
    sub = dr[: 1001 * 32]
    assert gs.traversal_counts_noalloc(sub.data_ptr(), 1001, any_hit=True) == \
        gs.traversal_counts(sub.data_ptr(), 1001, any_hit=True)
    assert gs.error_flags() == 0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from banshee_b200 import capi, scenes

    ctx = capi.Context(0)
    gs = capi.GpuScene(ctx, scenes.soup(1000, seed=3))
    limit = ((16 << 20) - 256) // 16          # closest-hit rays that fit the 16 MiB scratch
    buf = torch.zeros(32 * 8, dtype=torch.uint8, device="cuda")
    with pytest.raises(capi.BansheeError) as ei:
        gs.traversal_counts_noalloc(buf.data_ptr(), limit + 1, any_hit=False)
    assert ei.value.code == -1 and "limit" in str(ei.value)


def test_noalloc_allocates_nothing():
    """Under a zero allocation cap the allocation-free entry point still gives
    the allocating entry point's counts, the allocation counter does not move,
    and the allocating entry point is refused with BG_ERR_OOM."""
    import torch
    from banshee_b200 import capi, scenes

    ctx = capi.Context(0)
    gs = capi.GpuScene(ctx, scenes.soup(20_000, seed=5))
    rays = scenes.soup_rays(1 << 16, "coherent", seed=6)
    dr = torch.from_numpy(rays.view(np.uint8)).cuda()
    torch.cuda.synchronize()
    want = gs.traversal_counts(dr.data_ptr(), rays.shape[0])
    gs.traversal_counts_noalloc(dr.data_ptr(), rays.shape[0])       # the device's scratch address is looked up
    before = capi.alloc_stats()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]      # the device's free memory, whoever allocates
    capi.alloc_limit(0)
    try:
        for _ in range(2):
            assert gs.traversal_counts_noalloc(dr.data_ptr(), rays.shape[0]) == want
        assert torch.cuda.mem_get_info()[0] == free_before
        after = capi.alloc_stats()
        assert after["calls"] == before["calls"] and after["bytes"] == before["bytes"]
        with pytest.raises(capi.BansheeError) as ei:
            gs.traversal_counts(dr.data_ptr(), rays.shape[0])
        assert ei.value.code == -3                                   # BG_ERR_OOM
        assert capi.alloc_stats()["refused"] == after["refused"] + 1
    finally:
        capi.alloc_limit(None)
    assert gs.traversal_counts(dr.data_ptr(), rays.shape[0]) == want
